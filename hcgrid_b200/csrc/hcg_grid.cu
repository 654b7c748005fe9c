// Gather gridding on the device (replaces the `hcgrid` kernel,
// HCGrid/gridding.cu:277-403, and the host normalisation,
// HCGrid/gmap.cpp:306-312).
//
// Selection follows the reference exactly: per target pixel the ring range
// [uring, dring] from the disc around its centre, per ring the HEALPix pixel
// window [lpix, rpix] at phi -/+ disc_size (not scaled by 1/cos(dec)), the
// polar whole-ring rule, the first-used-ring skip of the reference's search
// (start_int - 1 underflow) and a strict distance < sphere_radius cutoff.
// Rings whose window edge falls outside the ring -- where the reference's
// loop would never advance -- are skipped and counted instead.
//
// Geometry (ring windows, great-circle distance, cutoff, Gaussian weight)
// is FP64. Channel sums are FP32 (multi-channel) or FP64 (single channel);
// weight sums are FP64.
//
// Kernels
//   k_pixel_prep     per pixel: ring range and the phi half of loc2pix
//   k_grid_1chan     one warp per pixel, candidates spread over lanes, FP64
//   k_group<COUNT>   one warp per 2x2 pixel group: candidate count (COUNT)
//                    or FP64 weights written as compact (sample, w[4]) entries
//   k_group_accum    one warp per group: FP32 channel accumulation from the
//                    entries, 4 channels per lane, normalised on store
#include <cuda_runtime.h>

#include <algorithm>
#include <utility>
#include <vector>

#include "hcg_internal.h"
#include "hcg_kernels.cuh"
#include "hcg_wcs.cuh"

namespace hcg {
namespace {

// ---------------------------------------------------------------------------
// Single-job kernels: one launch per phase, thread/warp/block indices map
// directly onto pixels, groups and tiles.

__global__ void k_pixel_prep(HpxParams h, uint64_t firstring, uint64_t usedrings, double disc, uint64_t npixmap,
                             const double *__restrict__ X, const double *__restrict__ Y, PixPrep *__restrict__ out,
                             DevStats *stats) {
    uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (p < npixmap) prep_item(h, firstring, usedrings, disc, X, Y, out, stats, p);
}

// GEN: fields whose kernel is not GAUSS1D
template <bool GEN>
__global__ void __launch_bounds__(256) k_grid_1chan(GridArgs a, uint64_t npixmap, const float *__restrict__ data,
                                                    uint32_t cstride, float *__restrict__ out,
                                                    float *__restrict__ wout) {
    uint64_t p = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    if (p < npixmap) grid1_item<GEN>(a, data, cstride, out, wout, p);
}

// GEN: fields whose kernel is not GAUSS1D; PACK: entries as 16-bit hi/lo
// pairs for the tensor-core builders (1) or as FP32 weights (0)
template <bool COUNT, bool GEN = false, int PACK = 0>
__global__ void __launch_bounds__(256, 3) k_group(GridArgs a, GroupArgs g, uint32_t *__restrict__ cap,
                                               const unsigned long long *__restrict__ off,
                                               uint32_t *__restrict__ e_idx, float4 *__restrict__ e_w,
                                               uint32_t *__restrict__ cnt, double *__restrict__ wsum,
                                               TileArgs tiles) {
    __shared__ PixPrep s_prep[8][4];
    __shared__ PixHalf s_half[8][4];
    int warp = threadIdx.x >> 5;
    uint64_t grp = g.g0 + blockIdx.x * 8ull + warp;
    if (grp < g.g1)
        group_item<COUNT, GEN, PACK>(a, g, cap, off, e_idx, e_w, cnt, wsum, tiles, grp, s_prep[warp], s_half[warp]);
}

__global__ void __launch_bounds__(256) k_group_accum(GroupArgs g, const unsigned long long *__restrict__ off,
                                                     const uint32_t *__restrict__ cnt,
                                                     const uint32_t *__restrict__ e_idx,
                                                     const float4 *__restrict__ e_w, const double *__restrict__ wsum,
                                                     const float *__restrict__ spec, uint32_t nchan,
                                                     uint32_t cstride, float *__restrict__ out, uint32_t ostride,
                                                     float *__restrict__ wout) {
    uint64_t grp = g.g0 + blockIdx.x * 8ull + (threadIdx.x >> 5);
    if (grp < g.g1)
        group_accum_item(g, off, cnt, e_idx, e_w, wsum, spec, nchan, cstride, out, ostride, wout, grp);
}

__global__ void __launch_bounds__(256) k_tile_rings(GridArgs a, GroupArgs g, TileArgs T) {
    tile_rings_item(a, g, T, T.t0 + blockIdx.x);
}

__global__ void __launch_bounds__(kTileThreads, kAccumCtas) k_tile_accum(GroupArgs g, TileArgs T,
                                                            const unsigned long long *__restrict__ off,
                                                            const uint32_t *__restrict__ cnt,
                                                            const uint32_t *__restrict__ e_slot,
                                                            const float4 *__restrict__ e_w,
                                                            const double *__restrict__ wsum,
                                                            const float *__restrict__ spec, uint32_t nchan,
                                                            uint32_t cstride, float *__restrict__ out,
                                                            uint32_t ostride, float *__restrict__ wout,
                                                            unsigned long long *timeouts) {
    // slices of a tile are adjacent blocks: they run together and share the
    // tile's entries through L2
    tile_accum_item<kAccumBufs, kAccumRows, kAccumCpt, kAccumSlice>(g, T, off, cnt, e_slot, e_w, wsum, spec, nchan,
                                                                    cstride, out, ostride, wout, T.t0 + blockIdx.y,
                                                                    blockIdx.x * kAccumSlice, timeouts);
}

// Exclusive scan of n uint32 counts into uint64 offsets (out[n] = total),
// one block of 1024 threads.
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(const uint32_t *__restrict__ in, uint64_t n,
                                                            uint32_t parts, unsigned long long *__restrict__ psum) {
    scan_sums_item(in, n, parts, psum, blockIdx.x);
}
__global__ void __launch_bounds__(kScanThreads) k_scan_psum(unsigned long long *__restrict__ psum, uint32_t parts) {
    scan_psum_item(psum, parts);
}
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const uint32_t *__restrict__ in, uint64_t n,
                                                             uint32_t parts, const unsigned long long *__restrict__ psum,
                                                             unsigned long long *__restrict__ out) {
    scan_apply_item(in, n, parts, psum, out, blockIdx.x);
}


// Entry offsets at the first group of every tile row (and the total).
__global__ void k_row_offsets(const unsigned long long *__restrict__ off, uint64_t ngroups, uint64_t groups_per_row,
                              uint32_t nrows, unsigned long long *__restrict__ out) {
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r > nrows) return;
    uint64_t g0 = min((uint64_t)r * groups_per_row, ngroups);
    out[r] = off[g0];
}

// Coarsening: pixel p of row-run [lead, lead + factor) takes the ring range,
// the phi halves of its windows and the polar rule of the run's first pixel
// (HCGrid/gridding.cu:284-308: the disc of l1[0], b1[0]); its own l1, b1,
// cb1 stay for distance and weight. Leaders are only read, so in place.
__global__ void k_coarsen(PixPrep *__restrict__ prep, uint32_t nx, uint64_t npix, uint32_t factor) {
    const uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (p >= npix) return;
    const uint32_t x = (uint32_t)(p % nx), back = x % factor;
    if (back == 0) return;
    const PixPrep L = prep[p - back];
    PixPrep &P = prep[p];
    for (int e = 0; e < 2; ++e) {
        P.tt[e] = L.tt[e];
        P.t1[e] = L.t1[e];
        P.tp[e] = L.tp[e];
    }
    P.ur = L.ur;
    P.nr = L.nr;
    P.polar = L.polar;
}

// Target pixel centres of a SIN header, one thread per pixel.
__global__ void k_sin_coords(SinWcs w, uint32_t nx, uint64_t npix, double *__restrict__ X, double *__restrict__ Y) {
    uint64_t o = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (o >= npix) return;
    double x, y;
    sin_pix2world(w, (double)(o % nx) + 1.0, (double)(o / nx) + 1.0, x, y);
    X[o] = x;
    Y[o] = y;
}

}  // namespace

cudaError_t coarsen_prep(PixPrep *prep, uint32_t nx, uint64_t npix, uint32_t factor, cudaStream_t s) {
    if (factor <= 1 || npix == 0) return cudaSuccess;
    k_coarsen<<<(unsigned)((npix + 255) / 256), 256, 0, s>>>(prep, nx, npix, factor);
    return cudaGetLastError();
}

cudaError_t sin_coords_device(const SinWcs &w, uint32_t nx, uint32_t ny, double *d_x, double *d_y, cudaStream_t s) {
    uint64_t n = (uint64_t)nx * ny;
    k_sin_coords<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(w, nx, n, d_x, d_y);
    return cudaGetLastError();
}

cudaError_t grid_field(hcg_context *ctx, const hcg_field *f, const hcg_target *t, float *d_cube, int layout,
                       float *d_wts, int engine, std::string &why) {
    // engine: HCG_ENGINE_FP32 or a tensor-core engine whose split the field holds
    const bool tc = (engine == HCG_ENGINE_TC_BF16 || engine == HCG_ENGINE_TC_F16) && f->nchan > 1;
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    const uint64_t P = (uint64_t)t->nx * t->ny;
    if ((e = cudaMemsetAsync(&ctx->d_stats->timeouts, 0, 2 * sizeof(unsigned long long), s)) != cudaSuccess) return e;
    PixPrep *prep = (PixPrep *)ctx->scratch.get(0, P * sizeof(PixPrep), s, e);
    if (e != cudaSuccess) return e;
    cudaEventRecord(ctx->ev0, s);
    k_pixel_prep<<<(unsigned)((P + 255) / 256), 256, 0, s>>>(f->hpx, f->firstring, f->usedrings, f->disc_size, P,
                                                              t->d_x, t->d_y, prep, ctx->d_stats);
    if ((e = coarsen_prep(prep, t->nx, P, ctx->factor, s)) != cudaSuccess) return e;
    cudaEventRecord(ctx->evp[0], s);
    const GridArgs a = grid_args(f, prep, ctx->d_stats);
    if (f->nchan == 1) {
        cudaEventRecord(ctx->evp[1], s);
        cudaEventRecord(ctx->evp[2], s);
        const unsigned nblk = (unsigned)((P * 32 + 255) / 256);
        if (f->kernel_type == HCG_GAUSS1D)
            k_grid_1chan<false><<<nblk, 256, 0, s>>>(a, P, f->d_spec, f->cstride, d_cube, d_wts);
        else
            k_grid_1chan<true><<<nblk, 256, 0, s>>>(a, P, f->d_spec, f->cstride, d_cube, d_wts);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    } else {
        GroupArgs g;
        g.nx = t->nx;
        g.ny = t->ny;
        g.gx = (t->nx + 1) / 2;
        g.ngroups = (uint64_t)g.gx * ((t->ny + 1) / 2);
        uint32_t *cap = (uint32_t *)ctx->scratch.get(1, g.ngroups * sizeof(uint32_t), s, e);
        unsigned long long *off =
            (unsigned long long *)ctx->scratch.get(2, (g.ngroups + 1) * sizeof(unsigned long long), s, e);
        uint32_t *cnt = (uint32_t *)ctx->scratch.get(3, g.ngroups * sizeof(uint32_t), s, e);
        double *wsum = (double *)ctx->scratch.get(4, P * sizeof(double), s, e);
        if (e != cudaSuccess) return e;
        g.g0 = 0;
        g.g1 = g.ngroups;
        g.ebase = 0;
        unsigned gblocks = (unsigned)((g.ngroups + 7) / 8);
        // tile table (union of ring windows per 16x8-pixel tile)
        TileArgs T{};
        T.ntx = (t->nx + kTileX - 1) / kTileX;
        T.nty = (t->ny + kTileY - 1) / kTileY;
        T.t0 = 0;
        const uint64_t ntiles = (uint64_t)T.ntx * T.nty;
        T.r0 = (int *)ctx->scratch.get(8, ntiles * sizeof(int), s, e);
        T.nr = (int *)ctx->scratch.get(9, ntiles * sizeof(int), s, e);
        T.U = (uint32_t *)ctx->scratch.get(10, ntiles * sizeof(uint32_t), s, e);
        T.ulo = (uint32_t *)ctx->scratch.get(11, ntiles * kTileMaxRings * sizeof(uint32_t), s, e);
        T.base = (uint32_t *)ctx->scratch.get(12, ntiles * (kTileMaxRings + 1) * sizeof(uint32_t), s, e);
        T.ring_idx = (uint16_t *)ctx->scratch.get(14, ntiles * kTileMaxSpan * sizeof(uint16_t), s, e);
        unsigned long long *rowoff =
            (unsigned long long *)ctx->scratch.get(13, (T.nty + 4) * sizeof(unsigned long long), s, e);
        const uint32_t parts = (uint32_t)std::min<uint64_t>(1024, (g.ngroups + 4095) / 4096 + 1);
        unsigned long long *psum =
            (unsigned long long *)ctx->scratch.get(15, (parts + 1) * sizeof(unsigned long long), s, e);
        T.cap = cap;  // the tile pass counts each group's candidates
        {
            // the tile pass keeps each group's windows for the weight pass (up to 4 GiB of them)
            const size_t wbytes = (size_t)ntiles * kWinSpan * kTileGroups * 2 * sizeof(uint4);
            cudaError_t ew = cudaSuccess;
            T.win = wbytes <= (4ull << 30) ? (uint4 *)ctx->scratch.get(18, wbytes, s, ew) : nullptr;
            if (ew != cudaSuccess) {
                cudaGetLastError();
                T.win = nullptr;
            }
        }
        T.overflow = &ctx->d_stats->overflow;
        T.pad = tc ? 8 : 1;  // the tensor-core engine loads ring runs as boxes of 8 samples
        T.ustat = ctx->d_stats->ustat;
        if (e != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(T.overflow, 0, 3 * sizeof(unsigned long long), s)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(T.ustat, 0, 2 * sizeof(unsigned long long), s)) != cudaSuccess) return e;
        k_tile_rings<<<(unsigned)ntiles, 256, 0, s>>>(a, g, T);
        TileArgs none{};
        // groups of tiles whose ring span exceeds the table (cap unknown) are counted here
        k_group<true><<<gblocks, 256, 0, s>>>(a, g, cap, nullptr, nullptr, nullptr, nullptr, nullptr, none);
        k_scan_sums<<<parts, kScanThreads, 0, s>>>(cap, g.ngroups, parts, psum);
        k_scan_psum<<<1, kScanThreads, 0, s>>>(psum, parts);
        k_scan_apply<<<parts, kScanThreads, 0, s>>>(cap, g.ngroups, parts, psum, off);
        // entry offsets at tile-row boundaries: the work is split into runs of
        // tile rows whose entries fit the context's entry budget
        const uint64_t groups_per_row = (uint64_t)(kTileY / 2) * g.gx;
        k_row_offsets<<<(T.nty + 1 + 255) / 256, 256, 0, s>>>(off, g.ngroups, groups_per_row, T.nty, rowoff);
        if ((e = cudaMemcpyAsync(rowoff + T.nty + 1, T.overflow, sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                 s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(rowoff + T.nty + 2, T.ustat, 2 * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
            return e;
        cudaEventRecord(ctx->evp[1], s);
        std::vector<unsigned long long> ro(T.nty + 4);
        if ((e = cudaMemcpyAsync(ro.data(), rowoff, ro.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                 s)) != cudaSuccess)
            return e;
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
        const bool tiled = ro[T.nty + 1] == 0;  // every tile's ring span fits the tile table
        if (tc && !tiled && !f->d_spec) {
            why = "a tile spans more than " + std::to_string(kTileMaxSpan) + " rings or holds samples in more than " +
                  std::to_string(kTileMaxRings) + ": the FP32 fallback needs the FP32 spectra";
            return cudaErrorInvalidValue;
        }
        const uint32_t ostride = layout == HCG_LAYOUT_CHANNEL_MAJOR ? 0 : f->nchan;  // 0: [channel][pixel]
        if (tc && tiled && tc_use_weights(ctx, f, ro[T.nty + 2], ro[T.nty], ntiles)) {
            // dense tiles: the tensor-core kernel evaluates the weights itself (no entries)
            cudaEventRecord(ctx->evp[2], s);
            if ((e = tc_weights(ctx, f, a, g, T, ntiles, d_cube, ostride, d_wts, why)) != cudaSuccess) return e;
            cudaEventRecord(ctx->ev1, s);
            return cudaGetLastError();
        }
        const unsigned long long budget = ctx->entry_budget / (sizeof(uint32_t) + sizeof(float4));
        std::vector<std::pair<uint32_t, uint32_t>> chunks;
        unsigned long long most = 1;
        for (uint32_t ra = 0; ra < T.nty;) {
            uint32_t rb = ra + 1;
            // a run fits the entry budget and the 65535 limit of the grid's y dimension
            while (rb < T.nty && ro[rb + 1] - ro[ra] <= budget && (uint64_t)(rb + 1 - ra) * T.ntx <= 65535) ++rb;
            chunks.push_back({ra, rb});
            most = std::max(most, ro[rb] - ro[ra]);
            ra = rb;
        }
        uint32_t *e_idx = (uint32_t *)ctx->scratch.get(5, (most + 1) * sizeof(uint32_t), s, e);
        float4 *e_w = (float4 *)ctx->scratch.get(6, (most + 1) * sizeof(float4), s, e);
        if (e != cudaSuccess) {
            why = "entry buffer of " + std::to_string(most) + " candidates";
            return e;
        }
        float *dst = d_cube;
        const int smem = kAccumBufs * kAccumRows * kAccumSlice * (int)sizeof(float);
        static bool attr_set = false;
        if (tiled && !attr_set) {
            if ((e = cudaFuncSetAttribute(k_tile_accum, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) !=
                cudaSuccess)
                return e;
            attr_set = true;
        }
        bool first = true;
        for (auto &ch : chunks) {
            GroupArgs gc = g;
            if (tiled && tc) {  // the tensor-core builders take packed hi/lo weights
                gc.pack = 1;
                tc_entry_format(f, gc.fmt, gc.wscale);
            }
            gc.g0 = std::min<uint64_t>((uint64_t)ch.first * groups_per_row, g.ngroups);
            gc.g1 = std::min<uint64_t>((uint64_t)ch.second * groups_per_row, g.ngroups);
            gc.ebase = ro[ch.first];
            if (gc.g1 <= gc.g0) continue;
            unsigned cb = (unsigned)((gc.g1 - gc.g0 + 7) / 8);
            const TileArgs &tt = tiled ? T : none;
            if (f->kernel_type == HCG_GAUSS1D) {
                if (gc.pack)
                    k_group<false, false, 1><<<cb, 256, 0, s>>>(a, gc, nullptr, off, e_idx, e_w, cnt, wsum, tt);
                else
                    k_group<false, false, 0><<<cb, 256, 0, s>>>(a, gc, nullptr, off, e_idx, e_w, cnt, wsum, tt);
            } else {
                if (gc.pack)
                    k_group<false, true, 1><<<cb, 256, 0, s>>>(a, gc, nullptr, off, e_idx, e_w, cnt, wsum, tt);
                else
                    k_group<false, true, 0><<<cb, 256, 0, s>>>(a, gc, nullptr, off, e_idx, e_w, cnt, wsum, tt);
            }
            if (first) cudaEventRecord(ctx->evp[2], s);  // phase marks are exact for a single chunk
            first = false;
            if (tiled && tc) {
                TileArgs Tc = T;
                Tc.t0 = (uint64_t)ch.first * T.ntx;
                e = tc_accum(ctx, f, gc, Tc, (uint64_t)(ch.second - ch.first) * T.ntx, off, cnt, e_idx, e_w, wsum, dst,
                             ostride, d_wts, ro[T.nty + 3], why);
                if (e != cudaSuccess) return e;
            } else if (tiled) {
                TileArgs Tc = T;
                Tc.t0 = (uint64_t)ch.first * T.ntx;
                dim3 grid((f->cstride + kAccumSlice - 1) / kAccumSlice,
                          (unsigned)((uint64_t)(ch.second - ch.first) * T.ntx));
                k_tile_accum<<<grid, kTileThreads, smem, s>>>(gc, Tc, off, cnt, e_idx, e_w, wsum, f->d_spec,
                                                               f->nchan, f->cstride, dst, ostride, d_wts,
                                                               &ctx->d_stats->timeouts);
            } else {
                k_group_accum<<<cb, 256, 0, s>>>(gc, off, cnt, e_idx, e_w, wsum, f->d_spec, f->nchan, f->cstride,
                                                 dst, ostride, d_wts);
            }
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        if (first) cudaEventRecord(ctx->evp[2], s);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    cudaEventRecord(ctx->ev1, s);
    return cudaGetLastError();
}

}  // namespace hcg
