// Stand-in for CUDA's OpenGL interop header in the headless reference build
// (oracle/_ref): the real one includes GL/gl.h, which this image lacks. Only
// declarations are needed; the harness never calls the interop paths.
#pragma once
#include <glad/glad.h>
#include <cuda_runtime_api.h>
extern "C" {
extern __host__ cudaError_t CUDARTAPI cudaGraphicsGLRegisterImage(struct cudaGraphicsResource **resource,
                                                                  GLuint image, GLenum target, unsigned int flags);
extern __host__ cudaError_t CUDARTAPI cudaGraphicsGLRegisterBuffer(struct cudaGraphicsResource **resource,
                                                                   GLuint buffer, unsigned int flags);
}
