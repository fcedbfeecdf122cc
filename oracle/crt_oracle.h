/* CPU restatement of the reference's render-path arithmetic (test
 * infrastructure: used only by tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg, never by the product path). */
#ifndef CRT_ORACLE_H
#define CRT_ORACLE_H
#include <stdint.h>

/* rays: n x 8 floats (o, tmin, d, tmax); out: n x 4 (t, prim bits, b1, b2). */
void oracle_trace_brute(const float *verts, long ntris, const float *rays, long n, float *out, int nthreads);
/* FP64 intersector: out_t (double), out_prim. Same acceptance predicate. */
void oracle_trace_fp64(const float *verts, long ntris, const float *rays, long n, double *out_t, int32_t *out_prim,
                       int nthreads);
/* Light::Visible for n queries (n x 12 floats); occluded[i] = !visible. */
void oracle_visible(const float *verts, long ntris, const float *q, long n, uint8_t *occluded, int nthreads);
/* Single-triangle test: returns 1 if accepted with *t < closest. */
int oracle_tri_isect(const float *v, const float *o, const float *d, float closest, float *t, float *b1, float *b2);

/* Closest hit by brute force in index order (ties -> lowest index); o, d
 * are 3 floats. Returns the primitive or -1; t, b1, b2 of the hit. */
int oracle_closest_brute(const float *verts, long ntris, const float *o, const float *d, float tmax, float *t,
                         float *b1, float *b2);
/* Light::Visible for one query of 12 floats; 1 = visible. */
int oracle_visible_one(const float *verts, long ntris, const float *q);

/* Scene arrays for the oracle renderer (tables as exported by the library:
 * materials 16 floats, meshes 8, lights 8 per entry). */
typedef struct oracle_scene {
    const float *verts, *normals, *uvs;
    const int32_t *prim_mesh;
    long ntris;
    const float *meshes, *materials, *lights;
    int nmeshes, nmaterials, nlights;
    int env_light;
    const float *env; /* RGBA, top row first */
    int env_w, env_h;
    float cam_pos[3], cam_ld[3], cam_du[3], cam_dv[3];
    int width, height;
    int max_bounces;
    float rr;
    int rr_start;
    unsigned long long seed;
    /* diffuse textures: RGBA bytes, top row first (material entry 14 = index) */
    int ntex;
    const unsigned char *const *tex;
    const int *tex_w, *tex_h;
} oracle_scene;

/* Path-traces samples [first_sample, first_sample + spp) of every pixel and
 * adds them to direct/indirect (w*h*4 floats) and sumsq (may be NULL). */
void oracle_render(const oracle_scene *s, int first_sample, int spp, float *direct, float *indirect, float *sumsq,
                   int nthreads);
/* Environment-map CDFs (u: w*h, v: h) and alias tables (2 floats/entry). */
void oracle_env_tables(const float *env, int w, int h, float *ucdf, float *vcdf, float *row_alias, float *col_alias);

#endif
