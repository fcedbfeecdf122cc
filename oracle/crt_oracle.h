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

#endif
