/* Minimal dynamic parallel-for over [0, n) on POSIX threads (this toolchain
 * has no OpenMP runtime). Work is handed out in chunks through an atomic
 * counter. Test infrastructure only. */
#ifndef CRT_PAR_H
#define CRT_PAR_H
#include <pthread.h>
#include <stdatomic.h>
#include <unistd.h>

typedef void (*par_body_fn)(long i, void *ctx);

typedef struct {
    atomic_long next;
    long n, chunk;
    par_body_fn fn;
    void *ctx;
} par_job;

static void *par_worker(void *arg) {
    par_job *j = (par_job *)arg;
    for (;;) {
        long b = atomic_fetch_add(&j->next, j->chunk);
        if (b >= j->n) break;
        long e = b + j->chunk < j->n ? b + j->chunk : j->n;
        for (long i = b; i < e; ++i) j->fn(i, j->ctx);
    }
    return 0;
}

static inline int par_default_threads(void) {
    long c = sysconf(_SC_NPROCESSORS_ONLN);
    return c > 0 ? (int)c : 1;
}

static inline void par_for(long n, long chunk, int nthreads, par_body_fn fn, void *ctx) {
    if (nthreads <= 0) nthreads = par_default_threads();
    if (nthreads > 256) nthreads = 256;
    par_job j;
    atomic_init(&j.next, 0);
    j.n = n;
    j.chunk = chunk > 0 ? chunk : 1;
    j.fn = fn;
    j.ctx = ctx;
    if (nthreads == 1 || n <= j.chunk) {
        par_worker(&j);
        return;
    }
    pthread_t th[256];
    int started = 0;
    for (int t = 1; t < nthreads; ++t)
        if (pthread_create(&th[started], 0, par_worker, &j) == 0) ++started;
    par_worker(&j);
    for (int t = 0; t < started; ++t) pthread_join(th[t], 0);
}

#endif
