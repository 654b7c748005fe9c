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

#include "hcg_internal.h"

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
};

// One warp per 2x2 pixel group. COUNT: number of union candidates (upper
// bound of the entries). Otherwise: FP64 weights of every union candidate
// for the 4 pixels, compacted to entries with any non-zero weight.
template <bool COUNT>
__global__ void __launch_bounds__(256) k_group(GridArgs a, GroupArgs g, uint32_t *__restrict__ cap,
                                               const unsigned long long *__restrict__ off,
                                               uint32_t *__restrict__ e_idx, float4 *__restrict__ e_w,
                                               uint32_t *__restrict__ cnt, double *__restrict__ wsum) {
    __shared__ PixPrep s_prep[8][4];
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint64_t grp = blockIdx.x * 8ull + warp;
    if (grp >= g.ngroups) return;
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
    const unsigned long long eoff = COUNT ? 0 : off[grp];
    for (int rb = R0; rb <= R1; rb += 32) {
        int k = rb + lane;
        uint32_t lo[4] = {0, 0, 0, 0}, hi[4] = {0, 0, 0, 0};
        uint32_t glo = 0xffffffffu, ghi = 0;
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
                e_idx[pos] = idx;
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
    uint64_t grp = blockIdx.x * 8ull + warp;
    if (grp >= g.ngroups) return;
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
    const unsigned long long e0 = off[grp];
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

}  // namespace

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
        unsigned gblocks = (unsigned)((g.ngroups + 7) / 8);
        k_group<true><<<gblocks, 256, 0, s>>>(a, g, cap, nullptr, nullptr, nullptr, nullptr, nullptr);
        k_scan_offsets<<<1, 1024, 0, s>>>(cap, g.ngroups, off);
        cudaEventRecord(ctx->evp[1], s);
        unsigned long long total = 0;
        if ((e = cudaMemcpyAsync(&total, off + g.ngroups, sizeof total, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
            return e;
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
        uint32_t *e_idx = (uint32_t *)ctx->scratch.get(5, (total + 1) * sizeof(uint32_t), s, e);
        float4 *e_w = (float4 *)ctx->scratch.get(6, (total + 1) * sizeof(float4), s, e);
        if (e != cudaSuccess) {
            why = "entry buffer of " + std::to_string(total) + " candidates";
            return e;
        }
        k_group<false><<<gblocks, 256, 0, s>>>(a, g, nullptr, off, e_idx, e_w, cnt, wsum);
        cudaEventRecord(ctx->evp[2], s);
        float *dst = d_cube;
        if (layout == HCG_LAYOUT_CHANNEL_MAJOR) {
            dst = (float *)ctx->scratch.get(7, P * f->nchan * sizeof(float), s, e);
            if (e != cudaSuccess) return e;
        }
        k_group_accum<<<gblocks, 256, 0, s>>>(g, off, cnt, e_idx, e_w, wsum, f->d_spec, f->nchan, f->cstride, dst,
                                              f->nchan, d_wts);
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
