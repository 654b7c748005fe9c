// Dec-band sharding: the samples a band of target rows needs.
//
// Output pixels are independent, and a pixel only reads the samples of the
// rings its disc covers (the reference's uring..dring, gridding.cu:306-323).
// Each ring's window is formed from that ring's samples alone (the window
// search and walk stay inside the ring, gridding.cu:326-374), so a field made
// of the complete rings [rlo, rhi] that the band's pixels visit grids those
// pixels with the same candidates, in the same order, as the whole field.
// One more sample goes in front of ring rlo: the reference's search never
// grids the first used ring of a field (its start index underflows,
// gridding.cu:326,363-367), and that sample's ring, which no pixel of the
// band visits, takes that place; the band's rings keep theirs. When rlo is
// the field's own first ring there is no such sample, and the band's field
// starts where the whole one does.
//
// A rank of a sharded job takes the sorted positions [s0, s1) (the field's
// sorted order, hcg_field_sorted), builds a field of those samples and their
// spectra, and grids its rows: no sample exchange beyond that range and no
// reduction.
#include <cuda_runtime.h>

#include <climits>
#include <mutex>
#include <string>

#include "hcg_internal.h"
#include "hcg_kernels.cuh"

namespace hcg {
namespace {

// Smallest first ring and largest end ring (relative to firstring) over the
// pixels [p0, p1) that see any ring; rr[0] starts at UINT_MAX, rr[1] at 0.
__global__ void k_band_rings(HpxParams h, uint64_t firstring, uint64_t usedrings, double disc,
                             const double *__restrict__ X, const double *__restrict__ Y, uint64_t p0, uint64_t p1,
                             unsigned int *rr, DevStats *stats) {
    const uint64_t p = p0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    unsigned int lo = UINT_MAX, hi = 0;
    if (p < p1) {
        PixPrep P;
        prep_item(h, firstring, usedrings, disc, X + p, Y + p, &P, stats, 0);
        if (P.nr > 0) {
            lo = (unsigned int)P.ur;
            hi = (unsigned int)(P.ur + P.nr);
        }
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if ((threadIdx.x & 31) == 0) {
        if (lo != UINT_MAX) atomicMin(&rr[0], lo);
        if (hi) atomicMax(&rr[1], hi);
    }
}

}  // namespace
}  // namespace hcg

using namespace hcg;

extern "C" hcg_status hcg_field_band_samples(hcg_context *ctx, const hcg_field *field, const hcg_target *target,
                                             uint32_t y0, uint32_t y1, uint64_t *s0, uint64_t *s1) {
    if (!ctx || !field || !target || !s0 || !s1) return HCG_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (y0 > y1 || y1 > target->ny) {
        ctx->err = "hcg_field_band_samples: rows [" + std::to_string(y0) + ", " + std::to_string(y1) +
                   ") outside the target's " + std::to_string(target->ny);
        return HCG_EINVAL;
    }
    *s0 = *s1 = 0;
    if (y0 == y1) return HCG_OK;
    cudaStream_t s = ctx->stream;
    unsigned int *rr = nullptr;
    const unsigned int init[2] = {UINT_MAX, 0};
    unsigned int got[2] = {UINT_MAX, 0};
    uint32_t lut[2] = {0, 0};
    const uint64_t p0 = (uint64_t)y0 * target->nx, p1 = (uint64_t)y1 * target->nx;
    cudaError_t e = dalloc(&rr, sizeof init, s, ctx->pool);
    if (e == cudaSuccess) e = cudaMemcpyAsync(rr, init, sizeof init, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && p1 > p0) {
        k_band_rings<<<(unsigned)((p1 - p0 + 255) / 256), 256, 0, s>>>(
            field->hpx, field->firstring, field->usedrings, field->disc_size, target->d_x, target->d_y, p0, p1, rr,
            ctx->d_stats);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(got, rr, sizeof got, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && got[0] != UINT_MAX) {
        // LUT[k]: first sorted position of relative ring k; LUT[usedrings] = n
        const uint64_t rlo = got[0], rend = got[1] <= field->usedrings ? got[1] : field->usedrings;
        e = cudaMemcpyAsync(&lut[0], field->d_lut + rlo, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&lut[1], field->d_lut + rend, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e == cudaSuccess && lut[1] > lut[0]) {
            *s0 = lut[0] > 0 ? lut[0] - 1 : 0;  // the sample in front of ring rlo
            *s1 = lut[1];
        }
    }
    if (rr) cudaFreeAsync(rr, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ctx->err = std::string("hcg_field_band_samples: ") + cudaGetErrorString(e);
        return HCG_EDEVICE;
    }
    return HCG_OK;
}
