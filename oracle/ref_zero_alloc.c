/* Test infrastructure: LD_PRELOAD shim for running the reference `curc -c`
 * (built with the shared CUDA runtime) when generating golden archives.
 *
 * The reference's k-mer indexes count bucket sizes in non-atomic uint8
 * counters (compress.cu:381/404, 720/739), so a slot of pos_array can stay
 * unwritten.  RefMatcher::match_binary_dest (compress.cu:760-770) then reads
 * the reference at pos_array[j]*5 with no upper bound; an uninitialised slot
 * can hold any value and the read can leave the allocation.  Zero-filling
 * every device allocation turns such a slot into position 0, which is in
 * bounds, and changes nothing else: every other buffer is written before it
 * is read. */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <stddef.h>

typedef int cudaError_t;
typedef cudaError_t (*malloc_fn)(void**, size_t);
extern cudaError_t cudaMemset(void* p, int v, size_t n);
extern cudaError_t cudaDeviceSynchronize(void);

cudaError_t cudaMalloc(void** p, size_t n) {
    static malloc_fn real = 0;
    if (!real) real = (malloc_fn)dlsym(RTLD_NEXT, "cudaMalloc");
    cudaError_t e = real(p, n);
    if (e == 0 && n) {
        e = cudaMemset(*p, 0, n);
        if (e == 0) e = cudaDeviceSynchronize();
    }
    return e;
}
