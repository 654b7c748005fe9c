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
#include "hcg_wcs.cuh"

namespace hcg {
namespace {

__device__ __forceinline__ uint32_t lower_bound_u64(const uint64_t *__restrict__ a, uint32_t lo, uint32_t hi,
                                                    uint64_t key) {
    while (lo < hi) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if (__ldg(a + mid) < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}
__device__ __forceinline__ uint32_t upper_bound_u64(const uint64_t *__restrict__ a, uint32_t lo, uint32_t hi,
                                                    uint64_t key) {
    while (lo < hi) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if (__ldg(a + mid) <= key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void k_pixel_prep(HpxParams h, uint64_t firstring, uint64_t usedrings, double disc, uint64_t npixmap,
                             const double *__restrict__ X, const double *__restrict__ Y, PixPrep *__restrict__ out,
                             DevStats *stats) {
    uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (p >= npixmap) return;
    PixPrep P;
    double x = X[p], y = Y[p];
    P.l1 = dmul(x, kDeg2Rad);
    P.b1 = dmul(y, kDeg2Rad);
    P.cb1 = cos(P.b1);
    P.pad = 0;
    if (!isfinite(x) || !isfinite(y)) {
        P.ur = 0; P.nr = 0; P.polar = 0;
        for (int e = 0; e < 2; ++e) P.tt[e] = P.t1[e] = P.tp[e] = 0.0;
        out[p] = P;
        return;
    }
    // gridding.cu:306-323
    double disc_theta = dsub(kHalfPi, P.b1);
    double disc_phi = P.l1;
    double utheta = dsub(disc_theta, disc);
    if (dmul(utheta, kRad2Deg) < 0) utheta = 0;
    int hard1, hard2;
    uint64_t uring = pix2ring(h, ang2pix(h, utheta, disc_phi, hard1));
    if (uring < firstring) uring = firstring;
    utheta = dadd(disc_theta, disc);
    uint64_t dring = pix2ring(h, ang2pix(h, utheta, disc_phi, hard2));
    if (dring >= firstring + usedrings) dring = firstring + usedrings - 1;
    if (hard1 | hard2) atomicAdd(&stats->hard_roundings, 1ULL);
    P.ur = (int)(uring - firstring);
    P.nr = (dring >= uring) ? (int)(dring - uring + 1) : 0;
    double dt = dmul(disc_theta, kRad2Deg);
    P.polar = (dt <= kNorthB || dt >= kSouthB);
    double ns = u2d(h.nside);
    double phis[2] = {dsub(disc_phi, disc), dadd(disc_phi, disc)};
    for (int e = 0; e < 2; ++e) {
        double tt = fmodulo(dmul(phis[e], kInvHalfPi), 4.0);
        P.tt[e] = tt;
        P.t1[e] = dmul(ns, dadd(0.5, tt));
        P.tp[e] = dsub(tt, u2d(d2u(tt)));
    }
    out[p] = P;
}

// loc2pix(z_ring, phi_edge) from its ring half and phi half.
__device__ __forceinline__ uint64_t edge_pix(const HpxParams &h, const RingRec &R, const PixPrep &P, int e) {
    if (R.eq) {
        uint64_t nl4 = 4 * h.nside;
        uint64_t jp = d2u(dsub(P.t1[e], R.t2));
        uint64_t jm = d2u(dadd(P.t1[e], R.t2));
        uint64_t ir = h.nside + 1 + jp - jm;
        uint64_t kshift = 1 - (ir & 1);
        uint64_t t1 = jp + jm + kshift + 1 + nl4 + nl4 - h.nside;
        uint64_t ip = (h.order > 0) ? ((t1 >> 1) & (nl4 - 1)) : ((t1 >> 1) % nl4);
        return h.ncap + (ir - 1) * nl4 + ip;
    }
    uint64_t jp = d2u(dmul(P.tp[e], R.t2));
    uint64_t jm = d2u(dmul(dsub(1.0, P.tp[e]), R.t2));
    uint64_t ir = jp + jm + 1;
    uint64_t ip = d2u(dmul(P.tt[e], u2d(ir)));
    return R.zpos ? 2 * ir * (ir - 1) + ip : h.npix - 2 * ir * (ir + 1) + ip;
}

// Candidate interval [lo, hi) of one ring for one pixel
// (gridding.cu:329-367). Returns false where the reference would spin.
__device__ __forceinline__ bool ring_window(const HpxParams &h, const RingRec &R, const PixPrep &P,
                                            const uint64_t *__restrict__ keys, uint32_t &lo, uint32_t &hi) {
    lo = hi = 0;
    uint64_t lpix = P.polar ? R.startpix : edge_pix(h, R, P, 0);
    if (!(lpix >= R.startpix && lpix < R.startpix + R.npr)) return false;
    uint64_t rpix = P.polar ? R.startpix + R.npr - 1 : edge_pix(h, R, P, 1);
    if (!(rpix >= R.startpix && rpix < R.startpix + R.npr)) return false;
    if (R.lut_lo == 0) return true;  // first used ring: the reference's search returns "none"
    lo = lower_bound_u64(keys, R.lut_lo, R.lut_hi, lpix);
    hi = upper_bound_u64(keys, lo, R.lut_hi, rpix);
    return true;
}

// helpers.cu:128-130 (degrees), with cos(b1), cos(b2) precomputed.
__device__ __forceinline__ double dist_deg(double l1, double b1, double cb1, double l2, double b2, double cb2) {
    double sb = sin((b1 - b2) * 0.5);
    double sl = sin((l1 - l2) * 0.5);
    return 2.0 * asin(sqrt(sb * sb + cb1 * cb2 * (sl * sl))) * kRad2Deg;
}

// Lane of the warp whose inclusive prefix `incl` first exceeds t.
__device__ __forceinline__ int owner_lane(uint32_t incl, uint32_t t) {
    int lo = 0;
#pragma unroll
    for (int step = 16; step; step >>= 1) {
        uint32_t v = __shfl_sync(0xffffffffu, incl, lo + step - 1);
        if (v <= t) lo += step;
    }
    return lo;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct GridArgs {
    HpxParams h;
    const RingRec *rings;
    const PixPrep *prep;
    const uint64_t *keys;
    const double *l2, *b2, *cb2, *w;
    double sphere_radius, p0;
    DevStats *stats;
};

// Single channel: one warp per pixel, FP64 throughout.
__global__ void __launch_bounds__(256) k_grid_1chan(GridArgs a, uint64_t npixmap, const float *__restrict__ data,
                                                    uint32_t cstride, float *__restrict__ out,
                                                    float *__restrict__ wout) {
    uint64_t p = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (p >= npixmap) return;
    const PixPrep P = a.prep[p];
    double acc = 0.0, ws = 0.0;
    unsigned long long cand = 0, within = 0, skips = 0;
    for (int rb = 0; rb < P.nr; rb += 32) {
        int r = rb + lane;
        uint32_t lo = 0, hi = 0;
        if (r < P.nr) {
            if (!ring_window(a.h, a.rings[P.ur + r], P, a.keys, lo, hi)) ++skips;
        }
        uint32_t len = hi > lo ? hi - lo : 0;
        uint32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        for (uint32_t tb = 0; tb < total; tb += 32) {
            uint32_t t = tb + lane;
            int src = owner_lane(incl, t);
            uint32_t s_lo = __shfl_sync(0xffffffffu, lo, src);
            uint32_t s_incl = __shfl_sync(0xffffffffu, incl, src);
            uint32_t s_len = __shfl_sync(0xffffffffu, len, src);
            if (t < total) {
                uint32_t idx = s_lo + (t - (s_incl - s_len));
                double d = dist_deg(P.l1, P.b1, P.cb1, __ldg(a.l2 + idx), __ldg(a.b2 + idx), __ldg(a.cb2 + idx));
                ++cand;
                if (d < a.sphere_radius) {
                    double wt = __ldg(a.w + idx) * exp(-d * d * a.p0);
                    acc += (double)__ldg(data + (uint64_t)idx * cstride) * wt;
                    ws += wt;
                    ++within;
                }
            }
        }
    }
    acc = warp_sum(acc);
    ws = warp_sum(ws);
    cand = warp_sum_u64(cand);
    within = warp_sum_u64(within);
    skips = warp_sum_u64(skips);
    if (lane == 0) {
        out[p] = (float)(acc / ws);
        if (wout) wout[p] = (float)ws;
        if (cand) atomicAdd(&a.stats->pairs_candidate, cand);
        if (within) atomicAdd(&a.stats->pairs_within, within);
        if (skips) atomicAdd(&a.stats->ring_skips, skips);
    }
}

struct GroupArgs {
    uint32_t nx, ny, gx;
    uint64_t ngroups;
    uint64_t g0, g1;             // groups handled by this launch
    unsigned long long ebase;    // entry offset of group g0 in the entry buffer
};

// Tiles of kTileX x kTileY pixels (kTileX/2 x kTileY/2 groups) whose union of
// ring windows is staged in shared memory by k_tile_accum. Per tile: first
// ring, ring count (0 = no samples), union size U and, per ring j, the union
// interval start ulo[j] and its slot base[j] in the staged list.
constexpr int kTileX = 16, kTileY = 8, kTileMaxRings = 256;
struct TileArgs {
    uint32_t ntx, nty;
    uint64_t t0;  // first tile of this launch
    int *r0, *nr;
    uint32_t *U, *ulo, *base;  // ulo: [tile][kTileMaxRings], base: [tile][kTileMaxRings + 1]
    unsigned long long *overflow;
};

// One warp per 2x2 pixel group. COUNT: number of union candidates (upper
// bound of the entries). Otherwise: FP64 weights of every union candidate
// for the 4 pixels, compacted to entries with any non-zero weight.
// With a tile table (`tiles.ulo` set) the entries hold the sample's slot in
// its tile's staged list instead of the sample index.
template <bool COUNT>
__global__ void __launch_bounds__(256) k_group(GridArgs a, GroupArgs g, uint32_t *__restrict__ cap,
                                               const unsigned long long *__restrict__ off,
                                               uint32_t *__restrict__ e_idx, float4 *__restrict__ e_w,
                                               uint32_t *__restrict__ cnt, double *__restrict__ wsum,
                                               TileArgs tiles) {
    __shared__ PixPrep s_prep[8][4];
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint64_t grp = g.g0 + blockIdx.x * 8ull + warp;
    if (grp >= g.g1) return;
    uint32_t gyi = (uint32_t)(grp / g.gx), gxi = (uint32_t)(grp % g.gx);
    uint64_t pix[4];
    bool valid[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint32_t xx = 2 * gxi + (q & 1), yy = 2 * gyi + (q >> 1);
        valid[q] = xx < g.nx && yy < g.ny;
        pix[q] = (uint64_t)yy * g.nx + xx;
    }
    if (lane < 4 && valid[lane]) s_prep[warp][lane] = a.prep[pix[lane]];
    __syncwarp();
    int R0 = 1 << 30, R1 = -1;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (valid[q] && s_prep[warp][q].nr > 0) {
            R0 = min(R0, s_prep[warp][q].ur);
            R1 = max(R1, s_prep[warp][q].ur + s_prep[warp][q].nr - 1);
        }
    }
    unsigned lt = (1u << lane) - 1u;
    unsigned long long count = 0, cand = 0, within = 0, skips = 0;
    uint32_t base = 0;
    double ws[4] = {0.0, 0.0, 0.0, 0.0};
    const unsigned long long eoff = COUNT ? 0 : off[grp] - g.ebase;
    const bool slots = !COUNT && tiles.ulo != nullptr;
    uint64_t tile = 0;
    int tr0 = 0;
    if (slots) {
        tile = (uint64_t)(gyi / (kTileY / 2)) * tiles.ntx + gxi / (kTileX / 2);
        tr0 = tiles.r0[tile];
    }
    for (int rb = R0; rb <= R1; rb += 32) {
        int k = rb + lane;
        uint32_t lo[4] = {0, 0, 0, 0}, hi[4] = {0, 0, 0, 0};
        uint32_t glo = 0xffffffffu, ghi = 0;
        long long slot_shift = 0;  // slot = idx + slot_shift for this lane's ring
        if (slots && k <= R1) {
            uint64_t j = tile * kTileMaxRings + (uint64_t)(k - tr0);
            slot_shift = (long long)tiles.base[tile * (kTileMaxRings + 1) + (k - tr0)] - (long long)tiles.ulo[j];
        }
        if (k <= R1) {
            const RingRec R = a.rings[k];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const PixPrep &P = s_prep[warp][q];
                if (valid[q] && k >= P.ur && k < P.ur + P.nr) {
                    if (!ring_window(a.h, R, P, a.keys, lo[q], hi[q])) {
                        ++skips;
                    } else if (hi[q] > lo[q]) {
                        glo = min(glo, lo[q]);
                        ghi = max(ghi, hi[q]);
                    }
                }
            }
        }
        uint32_t len = glo < ghi ? ghi - glo : 0;
        if (COUNT) {
            count += len;
            continue;
        }
        uint32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        for (uint32_t tb = 0; tb < total; tb += 32) {
            uint32_t t = tb + lane;
            int src = owner_lane(incl, t);
            uint32_t s_glo = __shfl_sync(0xffffffffu, glo, src);
            uint32_t s_excl = __shfl_sync(0xffffffffu, incl - len, src);
            long long s_shift = __shfl_sync(0xffffffffu, slot_shift, src);
            uint32_t s_lo[4], s_hi[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                s_lo[q] = __shfl_sync(0xffffffffu, lo[q], src);
                s_hi[q] = __shfl_sync(0xffffffffu, hi[q], src);
            }
            float wq[4] = {0.f, 0.f, 0.f, 0.f};
            uint32_t idx = 0;
            bool any = false;
            if (t < total) {
                idx = s_glo + (t - s_excl);
                double l2 = __ldg(a.l2 + idx), b2 = __ldg(a.b2 + idx), cb2 = __ldg(a.cb2 + idx);
                double win = __ldg(a.w + idx);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (idx >= s_lo[q] && idx < s_hi[q]) {
                        const PixPrep &P = s_prep[warp][q];
                        double d = dist_deg(P.l1, P.b1, P.cb1, l2, b2, cb2);
                        ++cand;
                        if (d < a.sphere_radius) {
                            double wt = win * exp(-d * d * a.p0);
                            ws[q] += wt;
                            wq[q] = (float)wt;
                            any = true;
                            ++within;
                        }
                    }
                }
            }
            unsigned ball = __ballot_sync(0xffffffffu, any);
            if (any) {
                unsigned long long pos = eoff + base + __popc(ball & lt);
                e_idx[pos] = slots ? (uint32_t)((long long)idx + s_shift) : idx;
                e_w[pos] = make_float4(wq[0], wq[1], wq[2], wq[3]);
            }
            base += __popc(ball);
        }
    }
    count = warp_sum_u64(count);
    cand = warp_sum_u64(cand);
    within = warp_sum_u64(within);
    skips = warp_sum_u64(skips);
    if (COUNT) {
        if (lane == 0) cap[grp] = (uint32_t)count;
        return;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) ws[q] = warp_sum(ws[q]);
    if (lane == 0) {
        cnt[grp] = base;
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (valid[q]) wsum[pix[q]] = ws[q];
        if (cand) atomicAdd(&a.stats->pairs_candidate, cand);
        if (within) atomicAdd(&a.stats->pairs_within, within);
        if (skips) atomicAdd(&a.stats->ring_skips, skips);
    }
}

// FP32 channel accumulation of a group's entries; lane owns 4 channels per
// 128-channel pass. Output [pixel][channel] with row stride `ostride`.
__global__ void __launch_bounds__(256) k_group_accum(GroupArgs g, const unsigned long long *__restrict__ off,
                                                     const uint32_t *__restrict__ cnt,
                                                     const uint32_t *__restrict__ e_idx,
                                                     const float4 *__restrict__ e_w, const double *__restrict__ wsum,
                                                     const float *__restrict__ spec, uint32_t nchan,
                                                     uint32_t cstride, float *__restrict__ out, uint32_t ostride,
                                                     float *__restrict__ wout) {
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint64_t grp = g.g0 + blockIdx.x * 8ull + warp;
    if (grp >= g.g1) return;
    uint32_t gyi = (uint32_t)(grp / g.gx), gxi = (uint32_t)(grp % g.gx);
    uint64_t pix[4];
    bool valid[4];
    float inv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint32_t xx = 2 * gxi + (q & 1), yy = 2 * gyi + (q >> 1);
        valid[q] = xx < g.nx && yy < g.ny;
        pix[q] = (uint64_t)yy * g.nx + xx;
        double w = valid[q] ? wsum[pix[q]] : 1.0;
        inv[q] = (float)(1.0 / w);
        if (valid[q] && wout && lane == 0) wout[pix[q]] = (float)w;
    }
    const unsigned long long e0 = off[grp] - g.ebase;
    const uint32_t ne = cnt[grp];
    for (uint32_t c0 = 0; c0 < nchan; c0 += 128) {
        uint32_t c = c0 + 4 * lane;
        float4 acc[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[q] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c < cstride) {
            const float *sp = spec + c;
            uint32_t e = 0;
            for (; e + 4 <= ne; e += 4) {
                uint32_t id[4];
                float4 w[4], s[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    id[u] = __ldg(e_idx + e0 + e + u);
                    w[u] = __ldg(e_w + e0 + e + u);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) s[u] = __ldg(reinterpret_cast<const float4 *>(sp + (uint64_t)id[u] * cstride));
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const float wv[4] = {w[u].x, w[u].y, w[u].z, w[u].w};
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        acc[q].x = fmaf(wv[q], s[u].x, acc[q].x);
                        acc[q].y = fmaf(wv[q], s[u].y, acc[q].y);
                        acc[q].z = fmaf(wv[q], s[u].z, acc[q].z);
                        acc[q].w = fmaf(wv[q], s[u].w, acc[q].w);
                    }
                }
            }
            for (; e < ne; ++e) {
                uint32_t id = __ldg(e_idx + e0 + e);
                float4 w = __ldg(e_w + e0 + e);
                float4 s = __ldg(reinterpret_cast<const float4 *>(sp + (uint64_t)id * cstride));
                const float wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    acc[q].x = fmaf(wv[q], s.x, acc[q].x);
                    acc[q].y = fmaf(wv[q], s.y, acc[q].y);
                    acc[q].z = fmaf(wv[q], s.z, acc[q].z);
                    acc[q].w = fmaf(wv[q], s.w, acc[q].w);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (!valid[q]) continue;
            float *o = out + pix[q] * ostride;
            float v[4] = {acc[q].x * inv[q], acc[q].y * inv[q], acc[q].z * inv[q], acc[q].w * inv[q]};
            if (c + 3 < nchan && (ostride & 3) == 0) {
                *reinterpret_cast<float4 *>(o + c) = make_float4(v[0], v[1], v[2], v[3]);
            } else {
                for (int j = 0; j < 4; ++j)
                    if (c + j < nchan) o[c + j] = v[j];
            }
        }
    }
}

// Union of the ring windows of all pixels of one tile, per ring, and the
// slot each ring's union starts at in the tile's staged list.
__global__ void __launch_bounds__(256) k_tile_rings(GridArgs a, GroupArgs g, TileArgs T) {
    __shared__ PixPrep s_prep[kTileX * kTileY];
    __shared__ uint32_t s_lo[kTileMaxRings], s_hi[kTileMaxRings];
    __shared__ int s_r0, s_r1;
    const uint64_t tile = T.t0 + blockIdx.x;
    const uint32_t tx0 = (uint32_t)(tile % T.ntx) * kTileX, ty0 = (uint32_t)(tile / T.ntx) * kTileY;
    const int tid = threadIdx.x;
    if (tid == 0) { s_r0 = 1 << 30; s_r1 = -1; }
    __syncthreads();
    if (tid < kTileX * kTileY) {
        uint32_t xx = tx0 + tid % kTileX, yy = ty0 + tid / kTileX;
        PixPrep P;
        if (xx < g.nx && yy < g.ny) {
            P = a.prep[(uint64_t)yy * g.nx + xx];
        } else {
            P.nr = 0;
            P.ur = 0;
        }
        s_prep[tid] = P;
        if (P.nr > 0) {
            atomicMin(&s_r0, P.ur);
            atomicMax(&s_r1, P.ur + P.nr - 1);
        }
    }
    __syncthreads();
    const int r0 = s_r0, nrt = s_r1 - s_r0 + 1;
    if (nrt <= 0 || nrt > kTileMaxRings) {
        if (tid == 0) {
            T.r0[tile] = 0;
            T.nr[tile] = 0;
            T.U[tile] = 0;
            if (nrt > kTileMaxRings) atomicAdd(T.overflow, 1ULL);
        }
        return;
    }
    for (int j = tid; j < nrt; j += blockDim.x) { s_lo[j] = 0xffffffffu; s_hi[j] = 0; }
    __syncthreads();
    const int npx = kTileX * kTileY;
    for (int i = tid; i < npx * nrt; i += blockDim.x) {
        int p = i % npx, j = i / npx;
        const PixPrep &P = s_prep[p];
        int k = r0 + j;
        if (P.nr > 0 && k >= P.ur && k < P.ur + P.nr) {
            uint32_t lo, hi;
            if (ring_window(a.h, a.rings[k], P, a.keys, lo, hi) && hi > lo) {
                atomicMin(&s_lo[j], lo);
                atomicMax(&s_hi[j], hi);
            }
        }
    }
    __syncthreads();
    if (tid < 32) {  // one warp: prefix sums of the union lengths
        uint32_t run = 0;
        for (int jb = 0; jb < nrt; jb += 32) {
            int j = jb + tid;
            uint32_t len = (j < nrt && s_lo[j] < s_hi[j]) ? s_hi[j] - s_lo[j] : 0;
            uint32_t incl = len;
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
                if (tid >= o) incl += v;
            }
            if (j < nrt) {
                T.ulo[tile * kTileMaxRings + j] = (s_lo[j] < s_hi[j]) ? s_lo[j] : 0;
                T.base[tile * (kTileMaxRings + 1) + j] = run + incl - len;
            }
            run += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (tid == 0) {
            T.base[tile * (kTileMaxRings + 1) + nrt] = run;
            T.r0[tile] = r0;
            T.nr[tile] = nrt;
            T.U[tile] = run;
        }
    }
}

// Channel sums of one tile for one slice of kSlice channels: the tile's
// union of candidate spectra (slots) is staged in shared memory chunk by
// chunk; 16 threads per 2x2 group each own 4 channels of the slice, so a
// staged value is used for 4 pixels. Output [pixel][channel].
constexpr int kSlice = 64, kTileThreads = (kTileX / 2) * (kTileY / 2) * (kSlice / 4);
constexpr int kStageSlots = 768;
__global__ void __launch_bounds__(kTileThreads) k_tile_accum(GroupArgs g, TileArgs T,
                                                            const unsigned long long *__restrict__ off,
                                                            const uint32_t *__restrict__ cnt,
                                                            const uint32_t *__restrict__ e_slot,
                                                            const float4 *__restrict__ e_w,
                                                            const double *__restrict__ wsum,
                                                            const float *__restrict__ spec, uint32_t nchan,
                                                            uint32_t cstride, float *__restrict__ out,
                                                            uint32_t ostride, float *__restrict__ wout) {
    extern __shared__ float4 s_spec[];  // [kStageSlots][kSlice / 4]
    __shared__ uint32_t s_ulo[kTileMaxRings], s_base[kTileMaxRings + 1];
    const uint64_t tile = T.t0 + blockIdx.x;
    const uint32_t c0 = blockIdx.y * kSlice;
    const int tid = threadIdx.x, q = tid & (kSlice / 4 - 1), gl = tid / (kSlice / 4);
    const int nrt = T.nr[tile];
    const uint32_t U = T.U[tile];
    for (int j = tid; j < nrt; j += kTileThreads) s_ulo[j] = T.ulo[tile * kTileMaxRings + j];
    for (int j = tid; j <= nrt; j += kTileThreads) s_base[j] = T.base[tile * (kTileMaxRings + 1) + j];
    const uint32_t gxi = (uint32_t)(tile % T.ntx) * (kTileX / 2) + gl % (kTileX / 2);
    const uint32_t gyi = (uint32_t)(tile / T.ntx) * (kTileY / 2) + gl / (kTileX / 2);
    const bool gvalid = gxi < g.gx && (uint64_t)gyi * g.gx + gxi < g.ngroups;
    const uint64_t grp = (uint64_t)gyi * g.gx + gxi;
    uint64_t e = 0, e_end = 0;
    if (gvalid) {
        e = off[grp] - g.ebase;
        e_end = e + cnt[grp];
    }
    float4 acc[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    for (uint32_t cs = 0; cs < U; cs += kStageSlots) {
        const uint32_t ce = min(U, cs + kStageSlots);
        // stage rows [cs, ce): 16 threads per row, one float4 each
        for (uint32_t i = tid; i < (ce - cs) * (kSlice / 4); i += kTileThreads) {
            uint32_t row = i / (kSlice / 4), part = i % (kSlice / 4);
            uint32_t slot = cs + row;
            int lo = 0, hi = nrt;  // ring j with base[j] <= slot < base[j+1]
            while (hi - lo > 1) {
                int mid = (lo + hi) >> 1;
                if (s_base[mid] <= slot) lo = mid; else hi = mid;
            }
            uint32_t idx = s_ulo[lo] + (slot - s_base[lo]);
            uint32_t c = c0 + 4 * part;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (c < cstride) v = __ldg(reinterpret_cast<const float4 *>(spec + (uint64_t)idx * cstride + c));
            s_spec[row * (kSlice / 4) + part] = v;
        }
        __syncthreads();
        for (; e + 4 <= e_end; e += 4) {
            uint32_t sl[4];
            float4 w[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                sl[u] = __ldg(e_slot + e + u);
                w[u] = __ldg(e_w + e + u);
            }
            if (sl[3] >= ce) break;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const float4 sv = s_spec[(sl[u] - cs) * (kSlice / 4) + q];
                const float wv[4] = {w[u].x, w[u].y, w[u].z, w[u].w};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    acc[k].x = fmaf(wv[k], sv.x, acc[k].x);
                    acc[k].y = fmaf(wv[k], sv.y, acc[k].y);
                    acc[k].z = fmaf(wv[k], sv.z, acc[k].z);
                    acc[k].w = fmaf(wv[k], sv.w, acc[k].w);
                }
            }
        }
        for (; e < e_end; ++e) {
            uint32_t sl = __ldg(e_slot + e);
            if (sl >= ce) break;
            const float4 w = __ldg(e_w + e);
            const float4 sv = s_spec[(sl - cs) * (kSlice / 4) + q];
            const float wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                acc[k].x = fmaf(wv[k], sv.x, acc[k].x);
                acc[k].y = fmaf(wv[k], sv.y, acc[k].y);
                acc[k].z = fmaf(wv[k], sv.z, acc[k].z);
                acc[k].w = fmaf(wv[k], sv.w, acc[k].w);
            }
        }
        __syncthreads();
    }
    if (!gvalid) return;
    const uint32_t c = c0 + 4 * q;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        uint32_t xx = 2 * gxi + (k & 1), yy = 2 * gyi + (k >> 1);
        if (xx >= g.nx || yy >= g.ny) continue;
        uint64_t p = (uint64_t)yy * g.nx + xx;
        double ws = wsum[p];
        float inv = (float)(1.0 / ws);
        if (wout && blockIdx.y == 0 && q == 0) wout[p] = (float)ws;
        float *o = out + p * ostride;
        float v[4] = {acc[k].x * inv, acc[k].y * inv, acc[k].z * inv, acc[k].w * inv};
        if (c + 3 < nchan && (ostride & 3) == 0) {
            *reinterpret_cast<float4 *>(o + c) = make_float4(v[0], v[1], v[2], v[3]);
        } else {
            for (int j = 0; j < 4; ++j)
                if (c + j < nchan) o[c + j] = v[j];
        }
    }
}

// Exclusive scan of n uint32 counts into uint64 offsets (out[n] = total),
// one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_scan_offsets(const uint32_t *__restrict__ in, uint64_t n,
                                                       unsigned long long *__restrict__ out) {
    __shared__ unsigned long long part[1024];
    uint64_t per = (n + 1023) / 1024;
    uint64_t b = threadIdx.x * per, e = min(n, b + per);
    unsigned long long s = 0;
    for (uint64_t i = b; i < e; ++i) s += in[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        unsigned long long v = (threadIdx.x >= o) ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    unsigned long long run = part[threadIdx.x] - s;
    for (uint64_t i = b; i < e; ++i) {
        out[i] = run;
        run += in[i];
    }
    if (threadIdx.x == 1023) out[n] = part[1023];
}

// [P][C] -> [C][P] transpose through shared memory.
__global__ void k_transpose(uint64_t P, uint32_t C, const float *__restrict__ in, float *__restrict__ out) {
    __shared__ float tile[32][33];
    uint64_t p0 = (uint64_t)blockIdx.x * 32;
    uint32_t c0 = blockIdx.y * 32;
    int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += 8) {
        uint64_t p = p0 + r;
        uint32_t c = c0 + tx;
        tile[r][tx] = (p < P && c < C) ? in[p * C + c] : 0.f;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        uint32_t c = c0 + r;
        uint64_t p = p0 + tx;
        if (p < P && c < C) out[(uint64_t)c * P + p] = tile[tx][r];
    }
}

// Entry offsets at the first group of every tile row (and the total).
__global__ void k_row_offsets(const unsigned long long *__restrict__ off, uint64_t ngroups, uint64_t groups_per_row,
                              uint32_t nrows, unsigned long long *__restrict__ out) {
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r > nrows) return;
    uint64_t g0 = min((uint64_t)r * groups_per_row, ngroups);
    out[r] = off[g0];
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

cudaError_t sin_coords_device(const SinWcs &w, uint32_t nx, uint32_t ny, double *d_x, double *d_y, cudaStream_t s) {
    uint64_t n = (uint64_t)nx * ny;
    k_sin_coords<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(w, nx, n, d_x, d_y);
    return cudaGetLastError();
}

cudaError_t grid_field(hcg_context *ctx, const hcg_field *f, const hcg_target *t, float *d_cube, int layout,
                       float *d_wts, int engine, std::string &why) {
    (void)engine;
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    const uint64_t P = (uint64_t)t->nx * t->ny;
    PixPrep *prep = (PixPrep *)ctx->scratch.get(0, P * sizeof(PixPrep), s, e);
    if (e != cudaSuccess) return e;
    cudaEventRecord(ctx->ev0, s);
    k_pixel_prep<<<(unsigned)((P + 255) / 256), 256, 0, s>>>(f->hpx, f->firstring, f->usedrings, ctx->disc_size, P,
                                                              t->d_x, t->d_y, prep, ctx->d_stats);
    cudaEventRecord(ctx->evp[0], s);
    GridArgs a{f->hpx, f->d_rings, prep, f->d_keys, f->d_l2, f->d_b2, f->d_cb2, f->d_w,
               ctx->sphere_radius, ctx->kparams[0], ctx->d_stats};
    if (f->nchan == 1) {
        cudaEventRecord(ctx->evp[1], s);
        cudaEventRecord(ctx->evp[2], s);
        k_grid_1chan<<<(unsigned)((P * 32 + 255) / 256), 256, 0, s>>>(a, P, f->d_spec, f->cstride, d_cube, d_wts);
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
        unsigned long long *rowoff =
            (unsigned long long *)ctx->scratch.get(13, (T.nty + 2) * sizeof(unsigned long long), s, e);
        T.overflow = &ctx->d_stats->overflow;
        if (e != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(T.overflow, 0, sizeof(unsigned long long), s)) != cudaSuccess) return e;
        k_tile_rings<<<(unsigned)ntiles, 256, 0, s>>>(a, g, T);
        TileArgs none{};
        k_group<true><<<gblocks, 256, 0, s>>>(a, g, cap, nullptr, nullptr, nullptr, nullptr, nullptr, none);
        k_scan_offsets<<<1, 1024, 0, s>>>(cap, g.ngroups, off);
        // entry offsets at tile-row boundaries: the work is split into runs of
        // tile rows whose entries fit the context's entry budget
        const uint64_t groups_per_row = (uint64_t)(kTileY / 2) * g.gx;
        k_row_offsets<<<(T.nty + 1 + 255) / 256, 256, 0, s>>>(off, g.ngroups, groups_per_row, T.nty, rowoff);
        if ((e = cudaMemcpyAsync(rowoff + T.nty + 1, T.overflow, sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                 s)) != cudaSuccess)
            return e;
        cudaEventRecord(ctx->evp[1], s);
        std::vector<unsigned long long> ro(T.nty + 2);
        if ((e = cudaMemcpyAsync(ro.data(), rowoff, ro.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                 s)) != cudaSuccess)
            return e;
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
        const bool tiled = ro[T.nty + 1] == 0;  // every tile's ring span fits the tile table
        const unsigned long long budget = ctx->entry_budget / (sizeof(uint32_t) + sizeof(float4));
        std::vector<std::pair<uint32_t, uint32_t>> chunks;
        unsigned long long most = 1;
        for (uint32_t ra = 0; ra < T.nty;) {
            uint32_t rb = ra + 1;
            while (rb < T.nty && ro[rb + 1] - ro[ra] <= budget) ++rb;
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
        if (layout == HCG_LAYOUT_CHANNEL_MAJOR) {
            dst = (float *)ctx->scratch.get(7, P * f->nchan * sizeof(float), s, e);
            if (e != cudaSuccess) return e;
        }
        const int smem = kStageSlots * kSlice * (int)sizeof(float);
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
            gc.g0 = std::min<uint64_t>((uint64_t)ch.first * groups_per_row, g.ngroups);
            gc.g1 = std::min<uint64_t>((uint64_t)ch.second * groups_per_row, g.ngroups);
            gc.ebase = ro[ch.first];
            if (gc.g1 <= gc.g0) continue;
            unsigned cb = (unsigned)((gc.g1 - gc.g0 + 7) / 8);
            k_group<false><<<cb, 256, 0, s>>>(a, gc, nullptr, off, e_idx, e_w, cnt, wsum, tiled ? T : none);
            if (first) cudaEventRecord(ctx->evp[2], s);  // phase marks are exact for a single chunk
            first = false;
            if (tiled) {
                TileArgs Tc = T;
                Tc.t0 = (uint64_t)ch.first * T.ntx;
                dim3 grid((unsigned)((uint64_t)(ch.second - ch.first) * T.ntx), (f->cstride + kSlice - 1) / kSlice);
                k_tile_accum<<<grid, kTileThreads, smem, s>>>(gc, Tc, off, cnt, e_idx, e_w, wsum, f->d_spec,
                                                               f->nchan, f->cstride, dst, f->nchan, d_wts);
            } else {
                k_group_accum<<<cb, 256, 0, s>>>(gc, off, cnt, e_idx, e_w, wsum, f->d_spec, f->nchan, f->cstride,
                                                 dst, f->nchan, d_wts);
            }
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        if (first) cudaEventRecord(ctx->evp[2], s);
        if (layout == HCG_LAYOUT_CHANNEL_MAJOR) {
            dim3 grid((unsigned)((P + 31) / 32), (f->nchan + 31) / 32);
            k_transpose<<<grid, dim3(32, 8), 0, s>>>(P, f->nchan, dst, d_cube);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    cudaEventRecord(ctx->ev1, s);
    return cudaGetLastError();
}

}  // namespace hcg
