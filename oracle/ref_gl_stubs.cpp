// GL entry points for the headless reference build (oracle/_ref): the
// reference's scene loader creates a VAO/VBO per mesh through ImGui's GL
// loader table (Src/Core/scene.cpp:485-498). Here that table holds no-op
// functions, so no GL library is loaded or called. Test infrastructure only.
#include <imgui_impl_opengl3_loader.h>

union ImGL3WProcs imgl3wProcs;

namespace {
void APIENTRY gen(GLsizei n, GLuint *ids) {
    for (GLsizei i = 0; i < n; ++i) ids[i] = 0;
}
void APIENTRY bind1(GLuint) {}
void APIENTRY bind2(GLenum, GLuint) {}
void APIENTRY data(GLenum, GLsizeiptr, const void *, GLenum) {}
void APIENTRY enable(GLuint) {}
void APIENTRY attrib(GLuint, GLint, GLenum, GLboolean, GLsizei, const void *) {}
}  // namespace

extern "C" void refr_install_gl_stubs(void) {
    imgl3wProcs.gl.GenVertexArrays = gen;
    imgl3wProcs.gl.GenBuffers = gen;
    imgl3wProcs.gl.BindVertexArray = bind1;
    imgl3wProcs.gl.BindBuffer = bind2;
    imgl3wProcs.gl.BufferData = data;
    imgl3wProcs.gl.EnableVertexAttribArray = enable;
    imgl3wProcs.gl.VertexAttribPointer = attrib;
}
