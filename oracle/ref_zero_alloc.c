/* Test infrastructure: LD_PRELOAD shim for running the reference `curc -c`
 * (built with the shared CUDA runtime) when generating golden archives and
 * in the benchmark's reference arm.
 *
 * The reference's k-mer indexes count bucket sizes in non-atomic uint8
 * counters (compress.cu:381/404, 720/739), so a slot of pos_array can stay
 * unwritten.  RefMatcher::match_binary_dest (compress.cu:760-770) then reads
 * the reference at pos_array[j]*5 with no upper bound; an uninitialised slot
 * can hold any value and the read can leave the allocation.  Zero-filling
 * every device allocation turns such a slot into position 0, which is in
 * bounds, and changes nothing else: every other buffer is written before it
 * is read.
 *
 * The fill costs a cudaMemset and a device synchronisation per allocation.
 * When CURC_SHIM_LOG names a file, the shim appends to it at exit one line
 * "<allocations> <seconds>": the number of filled allocations and the wall
 * time spent in the fills, so that the cost can be reported beside the
 * reference's own time. */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <pthread.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <time.h>

typedef int cudaError_t;
typedef cudaError_t (*malloc_fn)(void**, size_t);
extern cudaError_t cudaMemset(void* p, int v, size_t n);
extern cudaError_t cudaDeviceSynchronize(void);

static double g_fill_s = 0.0;
static unsigned long g_fills = 0;
static pthread_mutex_t g_mu = PTHREAD_MUTEX_INITIALIZER;

static double now_s(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

__attribute__((destructor)) static void report(void) {
    const char* path = getenv("CURC_SHIM_LOG");
    if (!path) return;
    FILE* f = fopen(path, "a");
    if (!f) return;
    fprintf(f, "%lu %.6f\n", g_fills, g_fill_s);
    fclose(f);
}

cudaError_t cudaMalloc(void** p, size_t n) {
    static malloc_fn real = 0;
    if (!real) real = (malloc_fn)dlsym(RTLD_NEXT, "cudaMalloc");
    cudaError_t e = real(p, n);
    if (e == 0 && n) {
        const double t = now_s();
        e = cudaMemset(*p, 0, n);
        if (e == 0) e = cudaDeviceSynchronize();
        const double dt = now_s() - t;
        /* the reference allocates from several host threads */
        pthread_mutex_lock(&g_mu);
        g_fill_s += dt;
        ++g_fills;
        pthread_mutex_unlock(&g_mu);
    }
    return e;
}
