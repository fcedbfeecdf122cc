// Host-side scene description produced by the JSON/OBJ/HDR loader
// (scene_load.cpp) and consumed by the device upload (render.cu).
#pragma once
#include <map>
#include <string>
#include <vector>
#include <cstdint>

namespace crt {

// Material types of Src/Core/material.h:6-12.
enum MatType : int { MAT_LIGHT = 0, MAT_DIFFUSE = 1, MAT_PBR = 2, MAT_DIELECTRIC = 3, MAT_SUBSURFACE = 4 };
enum LightType : int { LIGHT_AREA = 0, LIGHT_POINT = 1, LIGHT_ENV = 2 };

// Device material record (64 B). Field defaults follow Src/Core/material.h
// and the per-type parsing of Src/Core/scene.cpp:283-378.
struct DMaterial {
    int type;
    float base[3];
    float ke[3];
    float roughness;
    float metallic;
    float transmission;
    float scatter[3];
    float ior;
    int tex;  // diffuse texture index or -1
    int pad;
};

// Device mesh record (Src/Core/triangle.h:62-74 minus host-only fields).
struct DMesh {
    int material;
    int light;   // index into lights or -1
    int start;   // first primitive in scene order
    int count;
    float area;  // sum of triangle areas in primitive order
    int pad[3];
};

// Device light record (Src/Core/light.h:18-44).
struct DLight {
    int type;
    int mesh;
    float emission[3];
    int pad[3];
};

// Orbit camera state (CameraParam, Src/Core/camera.h:11-46).
struct CameraState {
    float target[3];
    float distance, theta, phi, fovy;
    int width, height;
    float position[3], lookat[3], up[3];
    float u[3], v[3], w[3], du[3], dv[3], left_down[3];
    float focal, ratio;
};

// A decoded diffuse texture: 8-bit RGBA, rows top-down.
struct HostTexture {
    std::string name;
    int width = 0, height = 0;
    std::vector<uint8_t> rgba;
};

struct HostScene {
    // camera block
    std::string camera_type = "pinhole";
    int width = 0, height = 0;
    float fovy = 40.f;
    int max_bounces = 5;
    float rr = 0.8f;
    int spp = 16;
    float direction[3] = {0.f, 0.f, -1.f};
    bool denoise = false;
    // geometry in scene (primitive) order
    std::vector<float> verts;    // 9 per triangle
    std::vector<float> normals;  // 9 per triangle (per-vertex)
    std::vector<float> uvs;      // 6 per triangle
    std::vector<int> prim_mesh;  // mesh per triangle
    std::vector<DMesh> meshes;
    std::vector<std::string> mesh_names;
    std::vector<DMaterial> materials;
    std::vector<std::string> material_names;
    std::vector<DLight> lights;
    std::vector<HostTexture> textures;
    int env_light = -1;
    // environment map (RGBA float, top row first)
    int env_w = 0, env_h = 0;
    std::vector<float> env;
    std::vector<std::string> warnings;
};

// Parses a scene JSON with the reference's schema and semantics
// (Src/Core/scene.cpp:129-252, :254-396, :398-537, :539-616; OBJ import
// Src/Utils/objloader.cpp:66-210; HDR via the Radiance format).
void load_scene_json(const std::string &path, HostScene &out);

// Decodes a texture image file (PNG or binary PPM) to 8-bit RGBA (image.cpp).
void load_texture_image(const std::string &path, HostTexture &out);

// Triangle area and unit face normal exactly as Triangle::Triangle
// (Src/Core/triangle.cu:3-10).
float triangle_area(const float *v);

// Unit face normal of a triangle (9 floats) as the OBJ import computes it
// for faces without vertex normals (Src/Utils/objloader.cpp:192-198).
void face_normal(const float *v, float *n);

// Material record with the defaults of Src/Core/material.h before any
// per-type field is parsed.
DMaterial default_material_record();

}  // namespace crt
