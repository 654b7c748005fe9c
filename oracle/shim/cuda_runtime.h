/*
 * Host emulation of the few CUDA runtime names the reference sources use.
 *
 * TEST INFRASTRUCTURE ONLY. This header lets oracle/Makefile compile the
 * reference's HCGrid/gridding.cu, healpix.cu, helpers.cu and gmap.cpp with
 * g++ for the host, so the reference's own algorithm (including the body of
 * its `hcgrid` kernel) runs on CPU cores as the parity checker and the
 * timed CPU baseline. Nothing in the product includes it.
 *
 * Device memory is host memory, `__constant__` symbols are plain globals,
 * the legacy texture reference is a pointer wrapper, and a kernel launch is
 * a loop over (block, thread) with OpenMP across blocks
 * (HCG_EMU_LAUNCH below). The reference kernel has no inter-thread
 * communication (its only __syncthreads() is after all work), so the
 * emulation is exact.
 */
#ifndef HCG_SHIM_CUDA_RUNTIME_H
#define HCG_SHIM_CUDA_RUNTIME_H

#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#define __host__
#define __device__
#define __global__
#define __constant__
#define __shared__
#define __forceinline__ inline

struct uint3 { unsigned int x, y, z; };
struct dim3 {
    unsigned int x, y, z;
    dim3(unsigned int a = 1, unsigned int b = 1, unsigned int c = 1) : x(a), y(b), z(c) {}
};

extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

inline void __syncthreads() {}

typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 };
inline const char *cudaGetErrorString(cudaError_t e) { return e == 0 ? "no error" : "emulated error"; }

enum cudaMemcpyKind {
    cudaMemcpyHostToHost = 0,
    cudaMemcpyHostToDevice = 1,
    cudaMemcpyDeviceToHost = 2,
    cudaMemcpyDeviceToDevice = 3
};

inline cudaError_t cudaMalloc(void **p, size_t n) {
    *p = malloc(n ? n : 1);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
inline cudaError_t cudaMallocHost(void **p, size_t n) { return cudaMalloc(p, n); }
inline cudaError_t cudaFree(void *p) { free(p); return cudaSuccess; }
inline cudaError_t cudaFreeHost(void *p) { free(p); return cudaSuccess; }
inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind) {
    memcpy(d, s, n);
    return cudaSuccess;
}
template <class T>
inline cudaError_t cudaMemcpyToSymbol(T &symbol, const void *src, size_t n) {
    memcpy((void *)&symbol, src, n);
    return cudaSuccess;
}
inline cudaError_t cudaDeviceReset() { return cudaSuccess; }
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }

/* Legacy 1-D texture reference over linear memory. */
template <class T>
struct texture {
    const T *ptr = nullptr;
};
template <class T, class I>
inline T tex1Dfetch(const texture<T> &t, I i) { return t.ptr[i]; }
template <class T>
inline cudaError_t cudaBindTexture(size_t *, texture<T> &t, const void *p, size_t) {
    t.ptr = (const T *)p;
    return cudaSuccess;
}
template <class T>
inline cudaError_t cudaUnbindTexture(texture<T> &t) { t.ptr = nullptr; return cudaSuccess; }

/* Events: wall-clock stand-ins so the reference's own timing printouts work. */
struct hcg_emu_event { double t; };
typedef hcg_emu_event *cudaEvent_t;
double hcg_emu_now_ms();
inline cudaError_t cudaEventCreate(cudaEvent_t *e) { *e = new hcg_emu_event{0.0}; return cudaSuccess; }
inline cudaError_t cudaEventRecord(cudaEvent_t e, int = 0) { e->t = hcg_emu_now_ms(); return cudaSuccess; }
inline cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
inline cudaError_t cudaEventElapsedTime(float *ms, cudaEvent_t a, cudaEvent_t b) {
    *ms = (float)(b->t - a->t);
    return cudaSuccess;
}
inline cudaError_t cudaEventDestroy(cudaEvent_t e) { delete e; return cudaSuccess; }

/* Kernel launch: every (block, thread) in order inside a block, blocks spread
 * over OpenMP threads. Used via HCG_EMU_LAUNCH, which the build recipe puts in
 * place of the reference's `kernel<<<grid, block>>>(args)` launch line. */
template <class F>
void hcg_emu_launch(dim3 g, dim3 b, F f) {
    long nblk = (long)g.x * g.y * g.z;
#pragma omp parallel for schedule(dynamic, 8)
    for (long blk = 0; blk < nblk; ++blk) {
        gridDim = g;
        blockDim = b;
        blockIdx.x = (unsigned)(blk % g.x);
        blockIdx.y = (unsigned)((blk / g.x) % g.y);
        blockIdx.z = (unsigned)(blk / ((long)g.x * g.y));
        for (unsigned tz = 0; tz < b.z; ++tz)
            for (unsigned ty = 0; ty < b.y; ++ty)
                for (unsigned tx = 0; tx < b.x; ++tx) {
                    threadIdx.x = tx; threadIdx.y = ty; threadIdx.z = tz;
                    f();
                }
    }
}
#define HCG_EMU_LAUNCH(g, b, kern, ...) hcg_emu_launch(dim3(g), dim3(b), [&]() { kern(__VA_ARGS__); })

#endif
