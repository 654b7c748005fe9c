// Per-item device functions of the gridding kernels, shared by the
// single-job launches (hcg_grid.cu) and the batch engine (hcg_batch.cu), so
// both execute the same arithmetic. The method is described in hcg_grid.cu.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>

#include "hcg_internal.h"
#include "hcg_sm100.cuh"

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

__device__ __forceinline__ void prep_item(HpxParams h, uint64_t firstring, uint64_t usedrings, double disc,
                                          const double *__restrict__ X, const double *__restrict__ Y,
                                          PixPrep *__restrict__ out, DevStats *stats, uint64_t p) {
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

// Samples [lo, hi) of ring R whose pixels lie in [lpix, rpix].
__device__ __forceinline__ void pixel_window(const RingRec &R, uint64_t lpix, uint64_t rpix,
                                             const uint64_t *__restrict__ keys, const uint32_t *__restrict__ ptab,
                                             uint32_t &lo, uint32_t &hi) {
    if (R.span) {
        // the ring's pixel table gives the same bounds as the searches below
        const int64_t q0 = (int64_t)(lpix - R.startpix) - (int64_t)R.pmin;
        lo = q0 <= 0 ? R.lut_lo : (q0 >= (int64_t)R.span ? R.lut_hi : __ldg(ptab + R.tbl + q0));
        const int64_t q1 = (int64_t)(rpix - R.startpix) - (int64_t)R.pmin + 1;  // first pixel > rpix
        const uint32_t h1 = q1 <= 0 ? R.lut_lo : (q1 >= (int64_t)R.span ? R.lut_hi : __ldg(ptab + R.tbl + q1));
        hi = h1 > lo ? h1 : lo;
        return;
    }
    lo = lower_bound_u64(keys, R.lut_lo, R.lut_hi, lpix);
    hi = upper_bound_u64(keys, lo, R.lut_hi, rpix);
}

// Candidate interval [lo, hi) of one ring for one pixel
// (gridding.cu:329-367). Returns false where the reference would spin.
__device__ __forceinline__ bool ring_window(const HpxParams &h, const RingRec &R, const PixPrep &P,
                                            const uint64_t *__restrict__ keys, const uint32_t *__restrict__ ptab,
                                            uint32_t &lo, uint32_t &hi) {
    lo = hi = 0;
    uint64_t lpix = P.polar ? R.startpix : edge_pix(h, R, P, 0);
    if (!(lpix >= R.startpix && lpix < R.startpix + R.npr)) return false;
    uint64_t rpix = P.polar ? R.startpix + R.npr - 1 : edge_pix(h, R, P, 1);
    if (!(rpix >= R.startpix && rpix < R.startpix + R.npr)) return false;
    if (R.lut_lo == 0) return true;  // first used ring: the reference's search returns "none"
    pixel_window(R, lpix, rpix, keys, ptab, lo, hi);
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

// Four consecutive channels c..c+3 of pixel p into the cube: [pixel][channel]
// with row stride `ostride`, or [channel][pixel] (plane stride npix) when
// ostride is 0.
__device__ __forceinline__ void store_cube4(float *__restrict__ out, uint32_t ostride, uint64_t npix, uint64_t p,
                                            uint32_t c, uint32_t nchan, const float v[4]) {
    if (ostride) {
        float *o = out + p * ostride;
        if (c + 3 < nchan && (ostride & 3) == 0) {
            *reinterpret_cast<float4 *>(o + c) = make_float4(v[0], v[1], v[2], v[3]);
        } else {
            for (int j = 0; j < 4; ++j)
                if (c + j < nchan) o[c + j] = v[j];
        }
    } else {
        for (int j = 0; j < 4; ++j)
            if (c + j < nchan) out[(uint64_t)(c + j) * npix + p] = v[j];
    }
}

}  // namespace

// Geometry arguments of the gathering kernels (shared by several translation units).
struct GridArgs {
    HpxParams h;
    const RingRec *rings;
    const PixPrep *prep;
    const uint64_t *keys;
    const double *l2, *b2, *cb2, *w;
    double sphere_radius, p0;
    DevStats *stats;
    const double4 *half;  // per sorted sample: sin(l/2), cos(l/2), sin(b/2), cos(b/2)
    const uint32_t *ptab; // per-ring pixel tables (RingRec::tbl)
    double hlo, hhi;      // haversine thresholds bracketing sphere_radius (see pair_weight)
    int series;           // d^2 from the arcsine-squared series (small sphere_radius)
    double hpolar;        // haversine bound of every accepted pair (chord windows)
    float x2scale;        // 4 R2D^2 p0 log2(e): the FP32 Gaussian's exponent per unit of the series
    int series32;         // series && GAUSS1D: accepted pairs below the band take gauss_series_f32
    uint32_t ktype;       // HCG_GAUSS1D, HCG_GAUSS2D or HCG_TAPERED_SINC
    int ktaper;           // TAPERED_SINC with HCG_TAPER_FIX
    double kp1, kp2;      // second and third kernel parameters (p0 is the first)
};

namespace {

// Host: GridArgs of a field. The cutoff d < r (d = 2 asin(sqrt(h)) in degrees,
// helpers.cu:128-130) is decided from the haversine h alone when h is outside
// [h* (1 - 1e-9), h* (1 + 1e-9)], h* = sin^2(r / 2): the device's h and d carry
// relative errors below 1e-12 there, so the decision is the one the full
// formula takes. Inside the band the full formula decides.
inline GridArgs grid_args(const hcg_field *f, const PixPrep *prep, DevStats *stats) {
    GridArgs a{f->hpx, f->d_rings, prep, f->d_keys, f->d_l2, f->d_b2, f->d_cb2, f->d_w, f->sphere_radius,
               f->kparam0, stats, f->d_half, f->d_ptab, 0.0, 0.0, 0};
    const double s = std::sin(f->sphere_radius * kDeg2Rad * 0.5);
    const double hstar = s * s;
    a.hlo = hstar * (1.0 - 1e-9);
    a.hhi = hstar * (1.0 + 1e-9);
    a.series = hstar < 1e-3;
    a.hpolar = hstar * (1.0 + 1e-6);
    a.x2scale = (float)(4.0 * kRad2Deg * kRad2Deg * f->kparam0 * 1.4426950408889634);
    a.ktype = f->kernel_type;
    a.series32 = a.series && f->kernel_type == HCG_GAUSS1D;
    a.ktaper = f->taper_fix;
    a.kp1 = f->kparams[1];
    a.kp2 = f->kparams[2];
    return a;
}

// Candidate interval of the multi-channel path: the reference's window
// (gridding.cu:329-367; whole rings within 20 deg of a pole, 340-354)
// intersected with the pixels whose centres can hold a sample of the ring
// within the radius. An accepted pair has hav(d) < hpolar, and hav(d) =
// hav(db) + cos b_p cos b_s hav(dphi) with |db| >= the distance of b_p from
// the ring's latitude range and cos b_s >= the ring's smallest cos(lat), which
// bounds |dphi|; a sample lies within R.dphi of its pixel centre. The accepted
// pairs are the reference window's; only candidates beyond the radius are
// left out. Windows whose phi range wraps keep the reference's. `ref_len` is
// the reference window's length (its candidate count).
__device__ __forceinline__ bool ring_window_mc(const GridArgs &a, const RingRec &R, const PixPrep &P, uint32_t &lo,
                                               uint32_t &hi, uint32_t &ref_len) {
    ref_len = 0;
    if (!ring_window(a.h, R, P, a.keys, a.ptab, lo, hi)) return false;
    ref_len = hi > lo ? hi - lo : 0;
    if (R.lut_lo == 0 || hi <= lo) return true;
    // hav(db) >= y^2 (1 - y^2 / 3) with y = db / 2 (sin y >= y - y^3 / 6)
    const double y = 0.5 * fmax(0.0, fmax(R.bmin - P.b1, P.b1 - R.bmax));
    const double hb = y < 1.0 ? y * y * (1.0 - y * y * (1.0 / 3.0)) : 0.0;
    if (!(hb < a.hpolar)) {  // no sample of the ring within the radius
        hi = lo;
        return true;
    }
    const double H = (a.hpolar - hb) / (R.cbmin * P.cb1);
    if (!(H < 0.25)) return true;
    // |dphi| <= 2 asin(sqrt(H)) <= 2 sqrt(H / (1 - H)) (asin x = atan(x / sqrt(1 - x^2)) <= x / sqrt(1 - x^2))
    const double W = 2.0 * sqrt(H / (1.0 - H)) * (1.0 + 1e-9) + R.dphi + 1e-9;
    const double dp = 2.0 * kPi / (double)R.npr;
    const double lp = P.l1 - 2.0 * kPi * floor(P.l1 / (2.0 * kPi));
    const double jl = floor((lp - W - R.phi0) / dp), jh = ceil((lp + W - R.phi0) / dp);
    if (!(jl >= 0.0 && jh < (double)R.npr && jh - jl + 1.0 < (double)R.npr)) return true;
    uint32_t clo, chi;
    pixel_window(R, R.startpix + (uint64_t)jl, R.startpix + (uint64_t)jh, a.keys, a.ptab, clo, chi);
    lo = max(lo, clo);
    hi = max(lo, min(hi, chi));
    return true;
}

// 32-byte read-only load (no double4 overload of __ldg)
__device__ __forceinline__ double4 ldg4(const double4 *p) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// Pixel side of the pair test: half-angle sines and cosines.
struct PixHalf {
    double sl, cl, sb, cb;
};
__device__ __forceinline__ PixHalf pix_half(const PixPrep &P) {
    PixHalf q;
    sincos(P.l1 * 0.5, &q.sl, &q.cl);
    sincos(P.b1 * 0.5, &q.sb, &q.cb);
    return q;
}

// exp(-x) for the FP32 weights of the multi-channel path, x >= 0 from FP64:
// 2^(-x log2 e) with the exponent rounded once to FP32 and the hardware
// base-2 exponential (ex2.approx.ftz.f32, relative error about 2^-22). For
// x <= 4.5 (d <= 3 sigma) the result is within 5e-7 of exp(-x), relative.
__device__ __forceinline__ float gauss_f32(double x) {
    const float t = (float)(-x * 1.4426950408889634);  // log2(e)
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(t));
    return r;
}

// The same for an accepted pair whose cutoff FP64 has decided, from its
// haversine h < 1e-3: the arcsine-squared series (four terms) in FP32. The
// exponent's relative error stays below 3e-7, the weight's below 1.6e-6 at
// d = 3 sigma (x2scale = 4 R2D^2 p0 log2 e).
__device__ __forceinline__ float gauss_series_f32(double h, float x2scale) {
    const float hf = (float)h;
    const float t = -(hf * (1.f + hf * (1.f / 3.f + hf * (8.f / 45.f + hf * (4.f / 35.f))))) * x2scale;
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(t));
    return r;
}

// The grid kernels other than GAUSS1D (gridding.cu:242-256), FP64, for an
// accepted pair at d degrees: GAUSS2D (sigma_maj, sigma_min, PA) at the
// great-circle bearing of the sample seen from the pixel (helpers.cu:133-137),
// TAPERED_SINC (sigma, a, b) with sinc(x) = 1 for |x| < 1e-10
// (gridding.cu:229-235) and the taper exp(+(arg/a)^2) of the reference, or
// exp(-(arg/a)^2) with HCG_TAPER_FIX. Kept out of line: the GAUSS1D loops
// that inline pair_weight_s only branch to it.
__device__ __noinline__ double kernel_other(const GridArgs &a, const PixPrep &P, double d, double cb2,
                                            uint32_t idx) {
    const double p0 = a.p0, p1 = a.kp1, p2 = a.kp2;
    if (a.ktype == HCG_GAUSS2D) {
        double sdl, cdl;
        sincos(__ldg(a.l2 + idx) - P.l1, &sdl, &cdl);
        const double sb2 = sin(__ldg(a.b2 + idx)), sb1 = sin(P.b1);
        const double bear = atan2(cb2 * sdl, P.cb1 * sb2 - sb1 * cb2 * cdl);
        double sa, ca;
        sincos(bear - p2, &sa, &ca);
        const double ell = (p0 * p0) * (sa * sa) + (p1 * p1) * (ca * ca);
        const double q = d / p0 / p1;
        return exp(-((q * q) / 2. * ell));
    }
    const double arg = kPi * d / p0;
    const double x = arg / p2;
    const double s = fabs(x) < 1.e-10 ? 1. : sin(x) / x;
    const double t = (arg / p1) * (arg / p1);
    return s * exp(a.ktaper ? -t : t);
}

// Weight of sample idx for the pixel (0 outside sphere_radius): the
// haversine h = sin^2(db/2) + cos b1 cos b2 sin^2(dl/2) with the half-angle
// differences expanded from precomputed sines and cosines; d^2 for accepted
// pairs from asin^2(x) = sum_n (2x)^(2n) / (2 n^2 C(2n, n)) at x = sqrt(h)
// (five terms; used when h* < 1e-3, truncation below 1e-16 relative), else
// from asin itself. Pairs inside the threshold band take the full formula.
// GEN: the field's kernel may be other than GAUSS1D (kernel_other); without
// it the code is GAUSS1D's alone.
template <bool F32EXP = false, bool GEN = true>
__device__ __forceinline__ double pair_weight_s(const GridArgs &a, const PixPrep &P, const PixHalf &q,
                                                const double4 &s, double cb2, double win, uint32_t idx) {
    const double sb = q.sb * s.w - q.cb * s.z;  // sin((b1 - b2) / 2)
    const double sl = q.sl * s.y - q.cl * s.x;  // sin((l1 - l2) / 2)
    const double h = sb * sb + P.cb1 * cb2 * (sl * sl);
    if (h > a.hhi) return 0.0;
    if (F32EXP && h < a.hlo && a.series32) return win * (double)gauss_series_f32(h, a.x2scale);
    double d2;
    if (h < a.hlo) {
        if (a.series) {
            const double t = h * (1.0 + h * (1.0 / 3.0 + h * (8.0 / 45.0 + h * (4.0 / 35.0 + h * (128.0 / 1575.0)))));
            d2 = 4.0 * t * (kRad2Deg * kRad2Deg);
        } else {
            const double d = 2.0 * asin(sqrt(h)) * kRad2Deg;
            d2 = d * d;
        }
    } else {
        const double d = dist_deg(P.l1, P.b1, P.cb1, __ldg(a.l2 + idx), __ldg(a.b2 + idx), cb2);
        if (!(d < a.sphere_radius)) return 0.0;
        d2 = d * d;
    }
    if (GEN && a.ktype != HCG_GAUSS1D) {
        const double k = kernel_other(a, P, sqrt(d2), cb2, idx);
        return win * (F32EXP ? (double)(float)k : k);
    }
    // Multi-channel entries hold FP32 weights: the Gaussian is evaluated in
    // FP32 there (gauss_f32); distance and cutoff stay FP64.
    if (F32EXP) return win * (double)gauss_f32(d2 * a.p0);
    return win * exp(-d2 * a.p0);
}

template <bool GEN>
__device__ __forceinline__ double pair_weight(const GridArgs &a, const PixPrep &P, const PixHalf &q, uint32_t idx) {
    return pair_weight_s<false, GEN>(a, P, q, ldg4(a.half + idx), __ldg(a.cb2 + idx), __ldg(a.w + idx), idx);
}

// Single channel: one warp per pixel, FP64 throughout.
// Warp-collective: every lane passes the same pixel p. GEN as pair_weight_s.
template <bool GEN>
__device__ __forceinline__ void grid1_item(const GridArgs &a, const float *__restrict__ data, uint32_t cstride,
                                           float *__restrict__ out, float *__restrict__ wout, uint64_t p) {
    int lane = threadIdx.x & 31;
    const PixPrep P = a.prep[p];
    const PixHalf ph = pix_half(P);
    double acc = 0.0, ws = 0.0;
    unsigned long long cand = 0, within = 0, skips = 0;
    for (int rb = 0; rb < P.nr; rb += 32) {
        int r = rb + lane;
        uint32_t lo = 0, hi = 0;
        if (r < P.nr) {
            if (!ring_window(a.h, a.rings[P.ur + r], P, a.keys, a.ptab, lo, hi)) ++skips;
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
                const double wt = pair_weight<GEN>(a, P, ph, idx);
                ++cand;
                if (wt != 0.0) {
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

}  // namespace

// Launch arguments shared by the kernels of several translation units.
namespace {

// FP16 / BF16 halves of the tensor-core weight operand (fmt 0: FP16, 1: BF16).
__device__ __forceinline__ uint16_t tc_to16(float v, uint32_t fmt) {
    return fmt ? __bfloat16_as_ushort(__float2bfloat16_rn(v)) : __half_as_ushort(__float2half_rn(v));
}

__device__ __forceinline__ float tc_from16(uint16_t b, uint32_t fmt) {
    return fmt ? __bfloat162float(__ushort_as_bfloat16(b)) : __half2float(__ushort_as_half(b));
}

// hi/lo split of two weights at once (paired conversions): `hi` and `lo` hold
// the 16-bit values of a (low half) and b (high half), the same values as
// tc_to16 of each and of its remainder.
__device__ __forceinline__ void tc_split2(float a, float b, uint32_t fmt, uint32_t &hi, uint32_t &lo) {
    if (fmt) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        const float2 f = __bfloat1622float2(h);
        const __nv_bfloat162 l = __floats2bfloat162_rn(a - f.x, b - f.y);
        hi = *reinterpret_cast<const uint32_t *>(&h);
        lo = *reinterpret_cast<const uint32_t *>(&l);
    } else {
        const __half2 h = __floats2half2_rn(a, b);
        const float2 f = __half22float2(h);
        const __half2 l = __floats2half2_rn(a - f.x, b - f.y);
        hi = *reinterpret_cast<const uint32_t *>(&h);
        lo = *reinterpret_cast<const uint32_t *>(&l);
    }
}

}  // namespace

struct GroupArgs {
    uint32_t nx, ny, gx;
    uint64_t ngroups;
    uint64_t g0, g1;             // groups handled by this launch
    unsigned long long ebase;    // entry offset of group g0 in the entry buffer
    // entries for the tensor-core builders: the four weights times wscale as
    // 16-bit hi/lo pairs {hi(w0, w1), lo(w0, w1), hi(w2, w3), lo(w2, w3)}
    // (fmt 0: FP16, 1: BF16) instead of four FP32 weights
    uint32_t pack = 0, fmt = 0;
    float wscale = 1.f;
};

// Tiles of kTileX x kTileY pixels (kTileX/2 x kTileY/2 groups) whose union of
// ring windows is staged in shared memory by the accumulation kernels. Per
// tile: first ring r0 of its ring span, the number nr of rings of the span
// that hold union candidates (0 = no samples), the union size U and, per such
// ring c (in ring order), the union interval start ulo[c] and its slot
// base[c] in the staged list; ring_idx maps ring r0 + j of the span to c.
// Pixels much larger than the kernel give long spans with few occupied rings.
constexpr int kTileX = 16, kTileY = 8, kTileMaxRings = 1024, kTileMaxSpan = 4096;
constexpr uint32_t kCapUnknown = 0xffffffffu;
constexpr int kTileGroups = (kTileX / 2) * (kTileY / 2);
// Rings of a tile's span whose per-group windows the tile pass keeps for the
// weight pass (wider spans: the weight pass computes its windows itself).
// A kept window is (lo, hi); lo > hi marks a ring the reference would spin on.
constexpr int kWinSpan = 64;
struct TileArgs {
    uint32_t ntx, nty;
    uint64_t t0;  // first tile of this launch
    int *r0, *nr;
    uint32_t *U, *ulo, *base;  // ulo: [tile][kTileMaxRings], base: [tile][kTileMaxRings + 1]
    uint16_t *ring_idx;        // [tile][kTileMaxSpan]: index c of ring r0 + j (0xffff: no candidates)
    uint32_t *cap;             // per 2x2 group: union candidate count (kCapUnknown: left to k_group<true>)
    uint4 *win;                // [tile][kWinSpan][kTileGroups][2]: the group's 4 pixel windows per ring (or null)
    unsigned long long *overflow;
    uint32_t pad;  // ring runs take a multiple of `pad` slots (> 1: the tensor-core engine's 8-row boxes)
    unsigned long long *ustat;  // [0]: sum, [1]: largest of the tiles' staged slots U (or null)
};

// hcg_tc.cu: the tensor-core builders' entry format of a field with split
// spectra (GroupArgs::fmt and ::wscale).
void tc_entry_format(const hcg_field *f, uint32_t &fmt, float &wscale);
// hcg_tc.cu: tensor-core accumulation of `ntiles` tiles from T.t0, after
// k_group emitted the entries (slot mode, packed hi/lo weights) and the
// weight sums.
cudaError_t tc_accum(hcg_context *ctx, const hcg_field *f, const GroupArgs &g, const TileArgs &T, uint64_t ntiles,
                     const unsigned long long *off, const uint32_t *cnt, const uint32_t *e_slot, const float4 *e_w,
                     const double *wsum, float *out, uint32_t ostride, float *wout, unsigned long long umax,
                     std::string &why);
// hcg_tc.cu: tensor-core accumulation of `ntiles` tiles whose weights the
// kernel evaluates itself (dense tiles; no entries).
cudaError_t tc_weights(hcg_context *ctx, const hcg_field *f, const GridArgs &a, const GroupArgs &g,
                       const TileArgs &T, uint64_t ntiles, float *out, uint32_t ostride, float *wout,
                       std::string &why);

namespace {

// One warp per 2x2 pixel group. COUNT: number of union candidates (upper
// bound of the entries). Otherwise: FP64 weights of every union candidate
// for the 4 pixels, compacted to entries with any non-zero weight.
// With a tile table (`tiles.ulo` set) the entries hold the sample's slot in
// its tile's staged list instead of the sample index.
// Warp-collective: every lane passes the same group; s_prep is this warp's
// 4-entry shared-memory slot.
// PACK: 0 FP32 weights, 1 packed hi/lo pairs (GroupArgs::pack), 2 as g.pack says.
template <bool COUNT, bool GEN = false, int PACK = 2>  // GEN as pair_weight_s
__device__ __forceinline__ void group_item(const GridArgs &a, const GroupArgs &g, uint32_t *__restrict__ cap,
                                           const unsigned long long *__restrict__ off,
                                           uint32_t *__restrict__ e_idx, float4 *__restrict__ e_w,
                                           uint32_t *__restrict__ cnt, double *__restrict__ wsum,
                                           const TileArgs &tiles, uint64_t grp, PixPrep *s_prep, PixHalf *s_half) {
    int lane = threadIdx.x & 31;
    __syncwarp();
    if (COUNT && cap[grp] != kCapUnknown) return;  // counted by the tile pass
    uint32_t gyi = (uint32_t)(grp / g.gx), gxi = (uint32_t)(grp % g.gx);
    uint64_t pix[4];
    bool valid[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint32_t xx = 2 * gxi + (q & 1), yy = 2 * gyi + (q >> 1);
        valid[q] = xx < g.nx && yy < g.ny;
        pix[q] = (uint64_t)yy * g.nx + xx;
    }
    if (lane < 4 && valid[lane]) {
        s_prep[lane] = a.prep[pix[lane]];
        if (!COUNT) s_half[lane] = pix_half(s_prep[lane]);
    }
    __syncwarp();
    int R0 = 1 << 30, R1 = -1;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (valid[q] && s_prep[q].nr > 0) {
            R0 = min(R0, s_prep[q].ur);
            R1 = max(R1, s_prep[q].ur + s_prep[q].nr - 1);
        }
    }
    unsigned lt = (1u << lane) - 1u;
    unsigned long long count = 0, within = 0;
    uint32_t base = 0;
    double ws[4] = {0.0, 0.0, 0.0, 0.0};
    const unsigned long long eoff = COUNT ? 0 : off[grp] - g.ebase;
    bool slots = !COUNT && tiles.ulo != nullptr;
    uint64_t tile = 0;
    int tr0 = 0;
    if (slots) {
        tile = (uint64_t)(gyi / (kTileY / 2)) * tiles.ntx + gxi / (kTileX / 2);
        tr0 = tiles.r0[tile];
        slots = tiles.nr[tile] > 0;  // no ring table (tile without samples, or one spanning too many rings)
    }
    for (int rb = R0; rb <= R1; rb += 32) {
        int k = rb + lane;
        uint32_t lo[4] = {0, 0, 0, 0}, hi[4] = {0, 0, 0, 0};
        uint32_t glo = 0xffffffffu, ghi = 0;
        long long slot_shift = 0;  // slot = idx + slot_shift for this lane's ring
        if (slots && k <= R1) {
            const uint32_t c = tiles.ring_idx[tile * kTileMaxSpan + (uint64_t)(k - tr0)];
            if (c < kTileMaxRings)  // rings without tile candidates have none for the group either
                slot_shift = (long long)tiles.base[tile * (kTileMaxRings + 1) + c] -
                             (long long)tiles.ulo[tile * kTileMaxRings + c];
        }
        if (k <= R1 && !COUNT && slots && tiles.win && k - tr0 < kWinSpan) {
            // the tile pass kept this group's windows for the ring
            const uint4 *w = tiles.win + ((tile * kWinSpan + (uint64_t)(k - tr0)) * kTileGroups +
                                          (uint64_t)((gyi % (kTileY / 2)) * (kTileX / 2) + gxi % (kTileX / 2))) * 2;
            const uint4 w0 = __ldg(w), w1 = __ldg(w + 1);
            const uint32_t kl[4] = {w0.x, w0.z, w1.x, w1.z}, kh[4] = {w0.y, w0.w, w1.y, w1.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (kl[q] <= kh[q]) {  // lo > hi: a ring the reference would spin on
                    lo[q] = kl[q];
                    hi[q] = kh[q];
                    if (hi[q] > lo[q]) {
                        glo = min(glo, lo[q]);
                        ghi = max(ghi, hi[q]);
                    }
                }
            }
        } else if (k <= R1) {
            const RingRec R = a.rings[k];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const PixPrep &P = s_prep[q];
                if (valid[q] && k >= P.ur && k < P.ur + P.nr) {
                    uint32_t rl;
                    if (ring_window_mc(a, R, P, lo[q], hi[q], rl) && hi[q] > lo[q]) {
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
                const double4 hs = ldg4(a.half + idx);
                const double cb2 = __ldg(a.cb2 + idx), win = __ldg(a.w + idx);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (idx >= s_lo[q] && idx < s_hi[q]) {
                        const double wt = pair_weight_s<true, GEN>(a, s_prep[q], s_half[q], hs, cb2, win, idx);
                        if (wt != 0.0) {
                            ws[q] += wt;
                            wq[q] = (float)wt;
                            any = true;
                            ++within;
                        }
                    }
                }
                if (PACK == 1 || (PACK == 2 && g.pack)) {
                    // the four slots carry {hi(w0, w1), lo(w0, w1), hi(w2, w3), lo(w2, w3)}
                    uint32_t h01, l01, h23, l23;
                    tc_split2(wq[0] * g.wscale, wq[1] * g.wscale, g.fmt, h01, l01);
                    tc_split2(wq[2] * g.wscale, wq[3] * g.wscale, g.fmt, h23, l23);
                    wq[0] = __uint_as_float(h01);
                    wq[1] = __uint_as_float(l01);
                    wq[2] = __uint_as_float(h23);
                    wq[3] = __uint_as_float(l23);
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
    within = warp_sum_u64(within);
    if constexpr (COUNT) {
        if (lane == 0) cap[grp] = (uint32_t)count;
        return;
    } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) ws[q] = warp_sum(ws[q]);
        if (lane == 0) {
            cnt[grp] = base;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (valid[q]) wsum[pix[q]] = ws[q];
            if (within) atomicAdd(&a.stats->pairs_within, within);
        }
    }
}

// Exclusive scan of n u32 counts into u64 offsets (out[n] = the total), in
// three passes over `parts` contiguous parts of the input, each swept by a
// block of kScanThreads threads in coalesced rows: the part sums, a scan of
// the part sums (one block), then the scan of each part from its base.
constexpr int kScanThreads = 1024;

__device__ __forceinline__ void scan_part(uint64_t n, uint32_t parts, uint32_t p, uint64_t &b, uint64_t &e) {
    const uint64_t per = (n + parts - 1) / parts;
    b = min(n, (uint64_t)p * per);
    e = min(n, b + per);
}

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and sets `total`. Every thread of the block calls it.
__device__ __forceinline__ unsigned long long block_exclusive_scan(unsigned long long v, unsigned long long &total) {
    __shared__ unsigned long long s_warp[kScanThreads / 32];
    __shared__ unsigned long long s_total;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned long long incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    __syncthreads();  // the shared values of a previous call are no longer read
    if (lane == 31) s_warp[w] = incl;
    __syncthreads();
    if (w == 0) {
        const unsigned long long x = lane < nw ? s_warp[lane] : 0ULL;
        unsigned long long xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long t = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += t;
        }
        if (lane < nw) s_warp[lane] = xi - x;  // exclusive over the warps
        if (lane == 31) s_total = xi;
    }
    __syncthreads();
    total = s_total;
    return s_warp[w] + incl - v;
}

__device__ __forceinline__ void scan_sums_item(const uint32_t *__restrict__ in, uint64_t n, uint32_t parts,
                                               unsigned long long *__restrict__ psum, uint32_t p) {
    uint64_t b, e;
    scan_part(n, parts, p, b, e);
    unsigned long long v = 0;
    for (uint64_t i = b + threadIdx.x; i < e; i += blockDim.x) v += in[i];
    unsigned long long tot;
    block_exclusive_scan(v, tot);
    if (threadIdx.x == 0) psum[p] = tot;
}

// One block: psum[0..parts) -> exclusive prefix sums, psum[parts] = total.
__device__ __forceinline__ void scan_psum_item(unsigned long long *__restrict__ psum, uint32_t parts) {
    unsigned long long run = 0;
    for (uint32_t c = 0; c < parts; c += blockDim.x) {
        const uint32_t i = c + threadIdx.x;
        const unsigned long long v = i < parts ? psum[i] : 0ULL;
        unsigned long long tot;
        const unsigned long long ex = block_exclusive_scan(v, tot);
        if (i < parts) psum[i] = run + ex;
        run += tot;
    }
    if (threadIdx.x == 0) psum[parts] = run;
}

__device__ __forceinline__ void scan_apply_item(const uint32_t *__restrict__ in, uint64_t n, uint32_t parts,
                                                const unsigned long long *__restrict__ psum,
                                                unsigned long long *__restrict__ out, uint32_t p) {
    uint64_t b, e;
    scan_part(n, parts, p, b, e);
    unsigned long long run = psum[p];
    for (uint64_t c = b; c < e; c += blockDim.x) {
        const uint64_t i = c + threadIdx.x;
        const unsigned long long v = i < e ? in[i] : 0ULL;
        unsigned long long tot;
        const unsigned long long ex = block_exclusive_scan(v, tot);
        if (i < e) out[i] = run + ex;
        run += tot;
    }
    if (p == parts - 1 && threadIdx.x == 0) out[n] = psum[parts];
}

// FP32 channel accumulation of a group's entries; lane owns 4 channels per
// 128-channel pass. Output [pixel][channel] with row stride `ostride`.
// Warp-collective: every lane passes the same group.
__device__ __forceinline__ void group_accum_item(const GroupArgs &g, const unsigned long long *__restrict__ off,
                                                 const uint32_t *__restrict__ cnt, const uint32_t *__restrict__ e_idx,
                                                 const float4 *__restrict__ e_w, const double *__restrict__ wsum,
                                                 const float *__restrict__ spec, uint32_t nchan, uint32_t cstride,
                                                 float *__restrict__ out, uint32_t ostride,
                                                 float *__restrict__ wout, uint64_t grp) {
    int lane = threadIdx.x & 31;
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
            const float v[4] = {acc[q].x * inv[q], acc[q].y * inv[q], acc[q].z * inv[q], acc[q].w * inv[q]};
            store_cube4(out, ostride, (uint64_t)g.nx * g.ny, pix[q], c, nchan, v);
        }
    }
}

// Union of the ring windows of all pixels of one tile, per ring, and the
// slot each ring's union starts at in the tile's staged list.
// Block-collective (call with every thread of a 256-thread block).
__device__ __forceinline__ void tile_rings_item(const GridArgs &a, const GroupArgs &g, const TileArgs &T,
                                                uint64_t tile) {
    __shared__ PixPrep s_prep[kTileX * kTileY];
    __shared__ uint32_t s_lo[kTileMaxSpan], s_hi[kTileMaxSpan];
    __shared__ uint32_t s_cnt[kTileGroups];
    __shared__ int s_r0, s_r1;
    const uint32_t tx0 = (uint32_t)(tile % T.ntx) * kTileX, ty0 = (uint32_t)(tile / T.ntx) * kTileY;
    const int tid = threadIdx.x;
    __syncthreads();  // shared state of a previous item is no longer read
    if (tid == 0) { s_r0 = 1 << 30; s_r1 = -1; }
    if (tid < kTileGroups) s_cnt[tid] = 0;
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
    // candidate counts of the tile's 2x2 groups (the entries k_group<false> may emit)
    auto write_caps = [&](bool known) {
        if (!T.cap || tid >= kTileGroups) return;
        const uint32_t gxi = (uint32_t)(tile % T.ntx) * (kTileX / 2) + tid % (kTileX / 2);
        const uint32_t gyi = (uint32_t)(tile / T.ntx) * (kTileY / 2) + tid / (kTileX / 2);
        const uint64_t grp = (uint64_t)gyi * g.gx + gxi;
        if (gxi < g.gx && grp < g.ngroups) T.cap[grp] = known ? s_cnt[tid] : kCapUnknown;
    };
    // the candidate statistic: the reference windows' lengths (the pairs the
    // reference visits) of every (pixel, ring) of the tile, and the rings the
    // reference would spin on
    unsigned long long cand = 0, skips = 0;
    auto add_cand = [&]() {
        cand = warp_sum_u64(cand);
        skips = warp_sum_u64(skips);
        if ((tid & 31) == 0 && cand) atomicAdd(&a.stats->pairs_candidate, cand);
        if ((tid & 31) == 0 && skips) atomicAdd(&a.stats->ring_skips, skips);
    };
    if (nrt <= 0 || nrt > kTileMaxSpan) {
        if (tid == 0) {
            T.r0[tile] = 0;
            T.nr[tile] = 0;
            T.U[tile] = 0;
            if (nrt > kTileMaxSpan) atomicAdd(T.overflow, 1ULL);
        }
        write_caps(nrt <= 0);  // no samples: nothing to count
        if (nrt > 0 && tid < kTileX * kTileY) {
            const PixPrep &P = s_prep[tid];
            for (int k = P.ur; k < P.ur + P.nr; ++k) {
                uint32_t lo, hi, rl;
                if (ring_window_mc(a, a.rings[k], P, lo, hi, rl))
                    cand += rl;
                else
                    ++skips;
            }
        }
        add_cand();
        return;
    }
    for (int j = tid; j < nrt; j += blockDim.x) { s_lo[j] = 0xffffffffu; s_hi[j] = 0; }
    __syncthreads();
    // one (group, ring, pixel) triple per thread, the four pixels of a group in
    // consecutive lanes: each thread forms one window (its dependent loads run
    // beside the other lanes'), the quad's shuffles give the group's union
    // (group_item's count) and the tile union takes min / max over groups. The
    // loop runs whole warps (inactive lanes hold empty windows).
    const int total = 4 * kTileGroups * nrt;
    for (int ib = 0; ib < total; ib += blockDim.x) {
        const int i = ib + tid;
        const bool act = i < total;
        const int q = i & 3, quad = i >> 2;
        const int gq = quad % kTileGroups, j = quad / kTileGroups;
        const int k = r0 + j;
        uint32_t lo = 0, hi = 0;
        if (act) {
            const int p = (2 * (gq / (kTileX / 2)) + (q >> 1)) * kTileX + 2 * (gq % (kTileX / 2)) + (q & 1);
            const PixPrep &P = s_prep[p];
            if (P.nr > 0 && k >= P.ur && k < P.ur + P.nr) {
                uint32_t rl;
                if (!ring_window_mc(a, a.rings[k], P, lo, hi, rl)) {
                    lo = 1;  // lo > hi: the reference would spin on this ring
                    hi = 0;
                    ++skips;
                } else {
                    cand += rl;
                }
            }
        }
        uint32_t glo = hi > lo ? lo : 0xffffffffu, ghi = hi > lo ? hi : 0;
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) {
            glo = min(glo, __shfl_xor_sync(0xffffffffu, glo, o));
            ghi = max(ghi, __shfl_xor_sync(0xffffffffu, ghi, o));
        }
        if (!act) continue;
        if (T.win && j < kWinSpan)
            reinterpret_cast<uint2 *>(T.win + ((tile * kWinSpan + j) * kTileGroups + gq) * 2)[q] = make_uint2(lo, hi);
        if (q == 0 && glo < ghi) {
            atomicAdd(&s_cnt[gq], ghi - glo);
            atomicMin(&s_lo[j], glo);
            atomicMax(&s_hi[j], ghi);
        }
    }
    add_cand();
    __syncthreads();
    write_caps(true);
    if (tid < 32) {  // one warp: compaction of the occupied rings and prefix sums of their lengths
        uint32_t run = 0, count = 0;
        for (int jb = 0; jb < nrt; jb += 32) {
            const int j = jb + tid;
            const bool occ = j < nrt && s_lo[j] < s_hi[j];
            uint32_t len = occ ? s_hi[j] - s_lo[j] : 0;
            if (T.pad > 1) len = (len + T.pad - 1) / T.pad * T.pad;
            uint32_t incl = len;
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
                if (tid >= o) incl += v;
            }
            const unsigned ball = __ballot_sync(0xffffffffu, occ);
            const uint32_t c = count + __popc(ball & ((1u << tid) - 1u));
            if (j < nrt) T.ring_idx[tile * kTileMaxSpan + j] = (occ && c < kTileMaxRings) ? (uint16_t)c : 0xffff;
            if (occ && c < kTileMaxRings) {
                T.ulo[tile * kTileMaxRings + c] = s_lo[j];
                T.base[tile * (kTileMaxRings + 1) + c] = run + incl - len;
            }
            run += __shfl_sync(0xffffffffu, incl, 31);
            count += __popc(ball);
        }
        if (tid == 0) {
            if (count > kTileMaxRings) {  // more occupied rings than the table holds
                T.r0[tile] = 0;
                T.nr[tile] = 0;
                T.U[tile] = 0;
                atomicAdd(T.overflow, 1ULL);
            } else {
                T.base[tile * (kTileMaxRings + 1) + count] = run;
                T.r0[tile] = r0;
                T.nr[tile] = (int)count;
                T.U[tile] = run;
                if (T.ustat) {
                    atomicAdd(T.ustat, (unsigned long long)run);
                    atomicMax(T.ustat + 1, (unsigned long long)run);
                }
            }
        }
    }
}

// Channel sums of one tile for one slice of SL channels: the tile's union
// of candidate spectra (slots) is staged in shared memory chunk by chunk;
// SL / CPT threads per 2x2 group each own CPT channels of the slice, so a
// staged value is used for 4 pixels. A CTA has one thread per (group,
// channel part): tile_threads(CPT, SL).
constexpr int tile_threads(int cpt, int sl) { return (kTileX / 2) * (kTileY / 2) * (sl / cpt); }
// FP32 staging rings (buffers x rows of a slice), channels per thread and
// slice width, the same for k_tile_accum and the batch engine's kb_accum:
// 16 threads per 2x2 group, 8 channels each, over 128 channels (one
// 512-thread CTA per SM), so a group's entries are loaded once per 128
// channels; the ring is three 144-row buffers (216 KB): long chunks leave
// the warps a chunk of slack between barrier waits (measured on 4M x 1,024
// -> 1200^2: 96-row chunks x 4 buffers 34.3 ms, 128 x 3 31.8 ms, 144 x 3
// 30.5 ms).
constexpr int kAccumBufs = 3, kAccumRows = 144, kAccumCpt = 8, kAccumSlice = 128, kAccumCtas = 1;
constexpr int kBatchAccumBufs = kAccumBufs, kBatchAccumRows = kAccumRows, kBatchAccumCpt = kAccumCpt,
              kBatchSlice = kAccumSlice;
constexpr int kTileThreads = tile_threads(kAccumCpt, kAccumSlice);
constexpr int kBatchTileThreads = tile_threads(kBatchAccumCpt, kBatchSlice);

// 16-byte asynchronous global -> shared copy (zero-filled when !valid).
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool valid) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// One arrival on `bar` once all of this thread's earlier cp.async copies have
// landed (the barrier's count includes it).
__device__ __forceinline__ void cp_async_arrive(uint64_t *bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(sm100::smem_u32(bar)) : "memory");
}
constexpr uint64_t kTileWaitNs = 1000000000ull;  // bound of the FP32 staging ring's barrier waits
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Channel sums of one tile for one slice of SL channels. The tile's
// union of candidate spectra (its slots) is staged in shared memory in
// chunks of CH rows through a ring of NB buffers: every thread copies its
// share of a chunk with cp.async and arrives on the chunk's `full` barrier
// when its copies land; each warp arrives on the buffer's `empty` barrier
// when it has summed the chunk, and the chunk NB - 2 ahead is staged into a
// buffer only once every warp is done with that buffer's previous chunk. So a
// warp whose groups have many entries in one chunk holds the others back only
// two chunks later, not at every chunk. SL / CPT threads per 2x2 group
// each own CPT channels of the slice (float4 q, q + SL / CPT, ... of a
// row, so the group's loads of one row are contiguous), and a staged value
// feeds 4 pixels. Block-collective (every thread of a tile_threads(CPT, SL)
// block; NB * CH * SL floats of dynamic shared memory). A barrier wait
// that runs out (1 s) is counted in `timeouts` and the item winds down.
template <int NB, int CH, int CPT, int SL>
__device__ __forceinline__ void tile_accum_item(const GroupArgs &g, const TileArgs &T,
                                                const unsigned long long *__restrict__ off,
                                                const uint32_t *__restrict__ cnt,
                                                const uint32_t *__restrict__ e_slot,
                                                const float4 *__restrict__ e_w, const double *__restrict__ wsum,
                                                const float *__restrict__ spec, uint32_t nchan, uint32_t cstride,
                                                float *__restrict__ out, uint32_t ostride,
                                                float *__restrict__ wout, uint64_t tile, uint32_t c0,
                                                unsigned long long *timeouts) {
    static_assert(NB >= 3, "the chunk NB - 2 ahead is staged while one is summed");
    static_assert(CPT % 4 == 0 && SL % CPT == 0, "whole float4 channel quads per thread");
    constexpr int kThreads = tile_threads(CPT, SL), kWarps = kThreads / 32, kTpg = SL / CPT, kQ = CPT / 4;
    extern __shared__ float4 s_spec[];  // [NB][CH][SL / 4]
    __shared__ uint32_t s_ulo[kTileMaxRings], s_base[kTileMaxRings + 1];
    __shared__ uint64_t s_full[NB], s_empty[NB];
    __shared__ volatile int s_abort;
    __syncthreads();  // shared state of a previous item is no longer read
    const int tid = threadIdx.x, q = tid % kTpg, gl = tid / kTpg;
    const int nrt = T.nr[tile];
    const uint32_t U = T.U[tile];
    for (int j = tid; j < nrt; j += kThreads) s_ulo[j] = T.ulo[tile * kTileMaxRings + j];
    for (int j = tid; j <= nrt; j += kThreads) s_base[j] = T.base[tile * (kTileMaxRings + 1) + j];
    if (tid == 0) {
        for (int b = 0; b < NB; ++b) {
            sm100::mbar_init(&s_full[b], kThreads);
            sm100::mbar_init(&s_empty[b], kWarps);
        }
        s_abort = 0;
        sm100::mbar_fence_init();
    }
    const uint32_t gxi = (uint32_t)(tile % T.ntx) * (kTileX / 2) + gl % (kTileX / 2);
    const uint32_t gyi = (uint32_t)(tile / T.ntx) * (kTileY / 2) + gl / (kTileX / 2);
    const bool gvalid = gxi < g.gx && (uint64_t)gyi * g.gx + gxi < g.ngroups;
    const uint64_t grp = (uint64_t)gyi * g.gx + gxi;
    uint64_t e = 0, e_end = 0;
    if (gvalid) {
        e = off[grp] - g.ebase;
        e_end = e + cnt[grp];
    }
    float4 acc[4][kQ];  // [pixel of the group][channel quad of the thread]
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int j = 0; j < kQ; ++j) acc[k][j] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    // stage rows [cs, min(U, cs + CH)) into buffer b: each warp takes kRows
    // consecutive rows, its lane r finds row r's sample (the ring j with
    // base[j] <= slot < base[j+1]) once, and the warp's 16-byte copies take
    // their row's sample from that lane; the thread's arrival on full[b]
    // completes when its copies have landed
    constexpr uint32_t kRows = (CH + kWarps - 1) / kWarps, kParts = SL / 4;
    static_assert(kRows <= 32 && 32 % kParts == 0, "one lane per staged row of a warp, whole rows per pass");
    const uint32_t lane = tid & 31, warp = tid >> 5;
    const uint32_t pc = c0 + 4 * (lane % kParts);  // the channels of this lane's copies (32 % kParts == 0)
    const bool pok = pc < cstride;
    auto stage = [&](uint32_t cs, int b) {
        const uint32_t ce = min(U, cs + CH), r0 = cs + warp * kRows;
        const uint32_t nr = r0 < ce ? min(kRows, ce - r0) : 0;
        uint32_t idx = 0;
        if (lane < nr) {
            const uint32_t slot = r0 + lane;
            int lo = 0, hi = nrt;
            while (hi - lo > 1) {
                int mid = (lo + hi) >> 1;
                if (s_base[mid] <= slot) lo = mid; else hi = mid;
            }
            idx = s_ulo[lo] + (slot - s_base[lo]);
        }
        float4 *dst = s_spec + ((size_t)b * CH + (r0 - cs)) * kParts + lane % kParts;
        const float *src0 = spec + (pok ? pc : 0);
        for (uint32_t i0 = 0; i0 < nr * kParts; i0 += 32) {  // warp-uniform trip count
            const uint32_t row = (i0 + lane) / kParts;
            const uint32_t ri = __shfl_sync(0xffffffffu, idx, row & 31);
            if (i0 + lane < nr * kParts) cp_async16(dst + row * kParts, src0 + (uint64_t)ri * cstride, pok);
        }
        cp_async_arrive(&s_full[b]);
    };
    const uint32_t nchunks = (U + CH - 1) / CH;
    for (uint32_t k = 0; k < NB - 2 && k < nchunks; ++k) stage(k * CH, (int)k);
    for (uint32_t k = 0; k < nchunks; ++k) {
        const uint32_t cs = k * CH, ce = min(U, cs + CH);
        const int b = (int)(k % NB);
        // the chunk NB - 2 ahead, into the buffer of chunk k - 2 once every warp is done with it
        const uint32_t kn = k + NB - 2;
        if (kn < nchunks) {
            const int bn = (int)(kn % NB);
            if (kn >= (uint32_t)NB && !s_abort &&
                !sm100::mbar_wait(&s_empty[bn], ((kn / NB) - 1) & 1, kTileWaitNs)) {
                atomicAdd(timeouts, 1ULL);
                s_abort = 1;
            }
            stage(kn * CH, bn);
        }
        if (!s_abort && !sm100::mbar_wait(&s_full[b], (k / NB) & 1, kTileWaitNs)) {
            atomicAdd(timeouts, 1ULL);
            s_abort = 1;
        }
        if (s_abort) break;
        const float4 *buf = s_spec + (size_t)b * CH * (SL / 4) + q;
        auto fma_entry = [&](uint32_t sl, const float4 &w) {
            const float wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int j = 0; j < kQ; ++j) {
                const float4 sv = buf[(sl - cs) * (SL / 4) + j * kTpg];
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    acc[kk][j].x = fmaf(wv[kk], sv.x, acc[kk][j].x);
                    acc[kk][j].y = fmaf(wv[kk], sv.y, acc[kk][j].y);
                    acc[kk][j].z = fmaf(wv[kk], sv.z, acc[kk][j].z);
                    acc[kk][j].w = fmaf(wv[kk], sv.w, acc[kk][j].w);
                }
            }
        };
        // entries kSet at a time from two register sets in turn: the next set
        // is loaded while one is summed, and no set is copied
        // (one lane of the group also asks L1 for the entries kPrefetch ahead,
        // which the registers cannot hold: measured 29.1 against 30.5 ms of
        // channel sums on 4M x 1,024 -> 1200^2)
        constexpr int kSet = 3, kPrefetch = 24;
        auto load = [&](uint32_t *sl, float4 *w, uint64_t at) {
#pragma unroll
            for (int u = 0; u < kSet; ++u) {
                sl[u] = __ldg(e_slot + at + u);
                w[u] = __ldg(e_w + at + u);
            }
            if (q == 0) {  // the group's last entry at most
                const uint64_t pa = min(at + kPrefetch, e_end - 1);
                asm volatile("prefetch.global.L1 [%0];" ::"l"(e_w + pa));
                asm volatile("prefetch.global.L1 [%0];" ::"l"(e_slot + pa));
            }
        };
        auto sum = [&](const uint32_t *sl, const float4 *w) {
#pragma unroll
            for (int u = 0; u < kSet; ++u) fma_entry(sl[u], w[u]);
        };
        if (e + kSet <= e_end) {
            uint32_t sa[kSet], sb[kSet];
            float4 wa[kSet], wb[kSet];
            load(sa, wa, e);
            for (;;) {  // sa holds entries [e, e + kSet)
                const bool nb = e + 2 * kSet <= e_end;
                if (nb) load(sb, wb, e + kSet);
                if (sa[kSet - 1] >= ce) break;
                sum(sa, wa);
                e += kSet;
                if (!nb) break;
                const bool na = e + 2 * kSet <= e_end;  // sb holds entries [e, e + kSet)
                if (na) load(sa, wa, e + kSet);
                if (sb[kSet - 1] >= ce) break;
                sum(sb, wb);
                e += kSet;
                if (!na) break;
            }
        }
        for (; e < e_end; ++e) {
            uint32_t sl = __ldg(e_slot + e);
            if (sl >= ce) break;
            fma_entry(sl, __ldg(e_w + e));
        }
        __syncwarp();
        if ((tid & 31) == 0) sm100::mbar_arrive(&s_empty[b]);  // this warp is done with buffer b
    }
    cp_async_wait_all();  // no copy into the ring outlives the item
    if (!gvalid) return;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        uint32_t xx = 2 * gxi + (k & 1), yy = 2 * gyi + (k >> 1);
        if (xx >= g.nx || yy >= g.ny) continue;
        uint64_t p = (uint64_t)yy * g.nx + xx;
        double ws = wsum[p];
        float inv = (float)(1.0 / ws);
        if (wout && c0 == 0 && q == 0) wout[p] = (float)ws;
#pragma unroll
        for (int j = 0; j < kQ; ++j) {
            const float v[4] = {acc[k][j].x * inv, acc[k][j].y * inv, acc[k][j].z * inv, acc[k][j].w * inv};
            store_cube4(out, ostride, (uint64_t)g.nx * g.ny, p, c0 + 4 * (q + j * kTpg), nchan, v);
        }
    }
}

}  // namespace
}  // namespace hcg
