// Field construction on the device: HEALPix keys of the samples, a stable
// LSD radix sort of (key, original index), the permuted sample geometry,
// the two-level ring lookup table and the per-ring window table.
//
// Reference path replaced (HCGrid/gridding.cu:70-136, all host code there):
//   keys      theta = pi/2 - lat*D2R, phi = lon*D2R, h_ang2pix  (77-82)
//   sort      boost parallel_stable_sort of (hpx, inx) by hpx     (86-92)
//   permute   lons/lats/data gathered by the sorted order          (96-114)
//   LUT       h_start_ring[k] = first sample of ring firstring+k  (118-136)
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "hcg_internal.h"

namespace hcg {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;

struct KeyRange {
    unsigned long long kmin, kmax;
};

__global__ void k_sample_keys(HpxParams h, uint64_t n, const double *__restrict__ lon, const double *__restrict__ lat,
                              uint64_t *__restrict__ keys, uint32_t *__restrict__ idx, KeyRange *range,
                              DevStats *stats) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    unsigned long long kmin = ~0ULL, kmax = 0;
    if (i < n) {
        double lo = lon[i], la = lat[i];
        if (!isfinite(lo) || !isfinite(la) || fabs(la) > 90.0) atomicAdd(&stats->invalid_input, 1ULL);
        double theta = dsub(kHalfPi, dmul(kDeg2Rad, la));
        double phi = dmul(kDeg2Rad, lo);
        int hard;
        uint64_t k = ang2pix(h, theta, phi, hard);
        if (hard) atomicAdd(&stats->hard_roundings, 1ULL);
        keys[i] = k;
        idx[i] = (uint32_t)i;
        kmin = kmax = k;
    }
    // warp then block min/max
    for (int o = 16; o; o >>= 1) {
        kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
        kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&range->kmin, kmin);
        atomicMax(&range->kmax, kmax);
    }
}

__global__ void k_init_range(KeyRange *r) {
    r->kmin = ~0ULL;
    r->kmax = 0;
}

// Per-tile digit histogram, stored digit-major: hist[d * nblocks + b].
__global__ void __launch_bounds__(kSortThreads) k_rs_hist(const uint64_t *__restrict__ keys, uint64_t n, int shift,
                                                         uint64_t kmin, uint32_t *__restrict__ hist,
                                                         uint32_t nblocks) {
    __shared__ uint32_t h[8][256];
    int warp = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < 256 * 8; d += kSortThreads) (&h[0][0])[d] = 0;
    __syncthreads();
    uint64_t base = (uint64_t)blockIdx.x * kSortTile;
#pragma unroll 4
    for (int j = 0; j < kSortItems; ++j) {
        uint64_t i = base + (uint64_t)j * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[warp][((keys[i] - kmin) >> shift) & 255], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += kSortThreads) {
        uint32_t s = 0;
        for (int w = 0; w < 8; ++w) s += h[w][d];
        hist[(uint64_t)d * nblocks + blockIdx.x] = s;
    }
}

// In-place exclusive scan of n uint32 values by one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_scan_u32_1block(uint32_t *data, uint64_t n) {
    __shared__ uint32_t part[1024];
    uint64_t per = (n + 1023) / 1024;
    uint64_t b = threadIdx.x * per, e = min(n, b + per);
    uint32_t s = 0;
    for (uint64_t i = b; i < e; ++i) s += data[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        uint32_t v = (threadIdx.x >= o) ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = part[threadIdx.x] - s;
    for (uint64_t i = b; i < e; ++i) {
        uint32_t v = data[i];
        data[i] = run;
        run += v;
    }
}

// Stable scatter: items are ranked in index order (round, warp, lane), the
// rank among equal digits coming from __match_any_sync within a warp and a
// per-digit running count across warps and rounds.
__global__ void __launch_bounds__(kSortThreads) k_rs_scatter(const uint64_t *__restrict__ kin,
                                                            const uint32_t *__restrict__ vin,
                                                            uint64_t *__restrict__ kout, uint32_t *__restrict__ vout,
                                                            uint64_t n, int shift, uint64_t kmin,
                                                            const uint32_t *__restrict__ offs, uint32_t nblocks) {
    __shared__ uint32_t s_off[256];
    __shared__ uint32_t s_run[256];
    __shared__ uint32_t s_cnt[8][256];
    int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int d = tid; d < 256; d += kSortThreads) {
        s_off[d] = offs[(uint64_t)d * nblocks + blockIdx.x];
        s_run[d] = 0;
    }
    for (int d = tid; d < 8 * 256; d += kSortThreads) (&s_cnt[0][0])[d] = 0;
    __syncthreads();
    uint64_t base = (uint64_t)blockIdx.x * kSortTile;
    unsigned lt = (1u << lane) - 1u;
    for (int r = 0; r < kSortItems; ++r) {
        uint64_t i = base + (uint64_t)r * kSortThreads + tid;
        bool valid = i < n;
        uint64_t k = valid ? kin[i] : 0;
        uint32_t v = valid ? vin[i] : 0;
        uint32_t d = valid ? (uint32_t)(((k - kmin) >> shift) & 255) : 0x1000u;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        uint32_t rank = __popc(peers & lt);
        if (valid && rank == 0) s_cnt[warp][d] = __popc(peers);
        __syncthreads();
        if (tid < 256) {
            uint32_t run = s_run[tid];
            for (int w = 0; w < 8; ++w) {
                uint32_t c = s_cnt[w][tid];
                s_cnt[w][tid] = run;
                run += c;
            }
            s_run[tid] = run;
        }
        __syncthreads();
        if (valid) {
            uint32_t pos = s_off[d] + s_cnt[warp][d] + rank;
            kout[pos] = k;
            vout[pos] = v;
        }
        __syncthreads();
        if (tid < 256)
            for (int w = 0; w < 8; ++w) s_cnt[w][tid] = 0;
        __syncthreads();
    }
}

struct RingSpan {
    unsigned long long firstring, usedrings;
};

__global__ void k_ring_span(HpxParams h, uint64_t n, uint64_t *keys, RingSpan *span) {
    keys[n] = h.npix;  // sentinel (gridding.cu:100)
    uint64_t first = pix2ring(h, keys[0]);
    span->firstring = first;
    span->usedrings = (uint32_t)(1 + pix2ring(h, keys[n - 1]) - first);
}

__device__ __forceinline__ uint32_t lower_bound_u64(const uint64_t *a, uint32_t lo, uint32_t hi, uint64_t key) {
    while (lo < hi) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if (a[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// LUT[k] = number of samples with key < startpix(firstring + k): the value
// the reference's incremental search produces (gridding.cu:118-136).
__global__ void k_ring_lut(HpxParams h, uint64_t n, const uint64_t *__restrict__ keys, uint64_t firstring,
                           uint64_t usedrings, uint32_t *__restrict__ lut) {
    uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (k > usedrings) return;
    uint32_t v;
    if (k == 0)
        v = 0;
    else if (k == usedrings)
        v = (uint32_t)n;
    else {
        uint64_t sp, npr;
        ring_info(h, firstring + k, sp, npr);
        v = lower_bound_u64(keys, 0, (uint32_t)n, sp);
    }
    lut[k] = v;
}

// Ring half of loc2pix at each used ring's first pixel centre
// (gridding.cu:330-334: ring info, pix2ang of startpix, then the theta used
// by ang2pix for lpix and rpix).
__global__ void k_ring_table(HpxParams h, uint64_t firstring, uint64_t usedrings, const uint32_t *__restrict__ lut,
                             const uint64_t *__restrict__ keys, RingRec *__restrict__ rings, DevStats *stats) {
    uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (k >= usedrings) return;
    RingRec R;
    uint64_t ring = firstring + k;
    ring_info(h, ring, R.startpix, R.npr);
    double z, phi, sth;
    bool have;
    pix2loc(h, R.startpix, z, phi, sth, have);
    double theta = have ? atan2(sth, z) : acos(z);
    // ang2pix(theta, phi) as the kernel calls it: cos (and sin near the poles) of theta
    double s, c;
    int hard;
    sincos_cr(theta, s, c, hard);
    if (hard) atomicAdd(&stats->hard_roundings, 1ULL);
    bool use_sin = (theta < 0.01) || (theta > kPiMinus001);
    double za = fabs(c);
    double ns = u2d(h.nside);
    R.eq = za <= kTwoThird;
    R.zpos = c > 0;
    if (R.eq)
        R.t2 = dmul(dmul(ns, c), 0.75);
    else if ((za < 0.99) || !use_sin)
        R.t2 = dmul(ns, dsqrt(dmul(3., dsub(1., za))));
    else
        R.t2 = ddiv(dmul(ns, s), dsqrt(ddiv(dadd(1., za), 3.)));
    R.lut_lo = lut[k];
    R.lut_hi = lut[k + 1];
    R.phi0 = phi;
    R.dphi = 0.0;  // set by k_ring_phi
    R.cbmin = 1.0;
    R.bmin = 0.0;
    R.bmax = 0.0;
    // pixel range of the ring's samples; the table offsets are set on the host
    R.pmin = 0;
    R.span = 0;
    R.tbl = 0;
    if (R.lut_lo != 0 && R.lut_hi > R.lut_lo) {
        R.pmin = (uint32_t)(keys[R.lut_lo] - R.startpix);
        R.span = (uint32_t)(keys[R.lut_hi - 1] - keys[R.lut_lo] + 1);
    }
    rings[k] = R;
}

// Per ring: the largest |phi| distance of a sample from its pixel centre,
// the smallest cos(lat) and the latitude range of its samples (block per ring).
__global__ void __launch_bounds__(256) k_ring_phi(HpxParams h, RingRec *__restrict__ rings,
                                                  const uint64_t *__restrict__ keys, const double *__restrict__ l2,
                                                  const double *__restrict__ b2, const double *__restrict__ cb2) {
    __shared__ double s_d[8], s_c[8], s_lo[8], s_hi[8];
    const uint32_t lo = rings[blockIdx.x].lut_lo, hi = rings[blockIdx.x].lut_hi;
    double dmax = 0.0, cmin = 1.0, bl = 1e300, bh = -1e300;
    for (uint32_t j = lo + threadIdx.x; j < hi; j += blockDim.x) {
        double z, phi, sth;
        bool have;
        pix2loc(h, keys[j], z, phi, sth, have);
        dmax = fmax(dmax, fabs(remainder(l2[j] - phi, 2.0 * kPi)));
        cmin = fmin(cmin, cb2[j]);
        bl = fmin(bl, b2[j]);
        bh = fmax(bh, b2[j]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
        cmin = fmin(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
        bl = fmin(bl, __shfl_xor_sync(0xffffffffu, bl, o));
        bh = fmax(bh, __shfl_xor_sync(0xffffffffu, bh, o));
    }
    if ((threadIdx.x & 31) == 0) {
        s_d[threadIdx.x >> 5] = dmax;
        s_c[threadIdx.x >> 5] = cmin;
        s_lo[threadIdx.x >> 5] = bl;
        s_hi[threadIdx.x >> 5] = bh;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            dmax = fmax(dmax, s_d[w]);
            cmin = fmin(cmin, s_c[w]);
            bl = fmin(bl, s_lo[w]);
            bh = fmax(bh, s_hi[w]);
        }
        rings[blockIdx.x].dphi = dmax;
        rings[blockIdx.x].cbmin = cmin;
        rings[blockIdx.x].bmin = hi > lo ? bl : 0.0;
        rings[blockIdx.x].bmax = hi > lo ? bh : 0.0;
    }
}

// Per-ring pixel tables: entry q of ring k is the first sorted sample of the
// ring whose pixel is >= startpix + pmin + q (one block per ring).
__global__ void __launch_bounds__(256) k_ring_ptab(const RingRec *__restrict__ rings, const uint64_t *__restrict__ keys,
                                                   uint32_t *__restrict__ ptab) {
    const RingRec R = rings[blockIdx.x];
    const uint64_t p0 = R.startpix + R.pmin;
    for (uint32_t q = threadIdx.x; q < R.span; q += blockDim.x)
        ptab[R.tbl + q] = lower_bound_u64(keys, R.lut_lo, R.lut_hi, p0 + q);
}

// Also the largest |w| of the per-sample weights (when given) into *wbits as
// the bits of a non-negative double, whose order as integers is the order of
// the values; NaN sorts above infinity.
__global__ void k_permute_geometry(uint64_t n, const uint32_t *__restrict__ perm, const double *__restrict__ lon,
                                   const double *__restrict__ lat, const double *__restrict__ w,
                                   double *__restrict__ l2, double *__restrict__ b2, double *__restrict__ cb2,
                                   double *__restrict__ wout, double4 *__restrict__ half,
                                   unsigned long long *__restrict__ wbits) {
    uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    unsigned long long wb = 0;
    if (j < n) {
        uint32_t i = perm[j];
        double b = dmul(lat[i], kDeg2Rad);
        double l = dmul(lon[i], kDeg2Rad);
        l2[j] = l;
        b2[j] = b;
        cb2[j] = cos(b);
        const double wi = w ? w[i] : 1.0;
        wout[j] = wi;
        wb = (unsigned long long)__double_as_longlong(fabs(wi));
        double4 q;
        sincos(l * 0.5, &q.x, &q.y);
        sincos(b * 0.5, &q.z, &q.w);
        half[j] = q;
    }
    if (!w) return;
#pragma unroll
    for (int o = 16; o; o >>= 1) wb = max(wb, __shfl_xor_sync(0xffffffffu, wb, o));
    if ((threadIdx.x & 31) == 0 && wb) atomicMax(wbits, wb);
}

// out[j][0..cstride) = in[perm[j]][0..nchan), zero padded; one warp per row.
__global__ void k_permute_rows(uint64_t n, uint32_t nchan, uint32_t cstride, const uint32_t *__restrict__ perm,
                               const float *__restrict__ in, float *__restrict__ out) {
    uint64_t j = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (j >= n) return;
    const float *src = in + (uint64_t)perm[j] * nchan;
    float *dst = out + j * cstride;
    if ((nchan & 3) == 0 && ((uintptr_t)in & 15) == 0) {
        for (uint32_t c = lane * 4; c < nchan; c += 128)
            *reinterpret_cast<float4 *>(dst + c) = __ldg(reinterpret_cast<const float4 *>(src + c));
    } else {
        for (uint32_t c = lane; c < cstride; c += 32) dst[c] = c < nchan ? src[c] : 0.f;
    }
}

// out[j][c] = in[c][perm[j]]: 32x32 tiles through shared memory.
__global__ void k_permute_cols(uint64_t n, uint32_t nchan, uint32_t cstride, const uint32_t *__restrict__ perm,
                               const float *__restrict__ in, float *__restrict__ out) {
    __shared__ float tile[32][33];
    uint64_t j0 = (uint64_t)blockIdx.x * 32;
    uint32_t c0 = blockIdx.y * 32;
    int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int r = ty; r < 32; r += 8) {
        uint64_t j = j0 + tx;
        uint32_t c = c0 + r;
        tile[r][tx] = (j < n && c < nchan) ? in[(uint64_t)c * n + perm[j]] : 0.f;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        uint64_t j = j0 + r;
        uint32_t c = c0 + tx;
        if (j < n && c < cstride) out[j * cstride + c] = tile[tx][r];
    }
}

// inv[perm[j]] = j: the sorted position of each input sample.
__global__ void k_inverse_perm(uint64_t n, const uint32_t *__restrict__ perm, uint32_t *__restrict__ inv) {
    const uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (j < n) inv[perm[j]] = (uint32_t)j;
}

// One uploaded chunk of sample-major spectra (input rows [r0, r0 + rows))
// scattered to its sorted rows: one warp per row, zero padding to cstride.
__global__ void k_scatter_rows(uint64_t r0, uint64_t rows, uint32_t nchan, uint32_t cstride,
                               const uint32_t *__restrict__ inv, const float *__restrict__ in,
                               float *__restrict__ out) {
    const uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    const float *src = in + r * nchan;
    float *dst = out + (uint64_t)__ldg(inv + r0 + r) * cstride;
    if ((nchan & 3) == 0 && ((uintptr_t)in & 15) == 0) {
        for (uint32_t c = lane * 4; c < nchan; c += 128)
            *reinterpret_cast<float4 *>(dst + c) = __ldg(reinterpret_cast<const float4 *>(src + c));
    } else {
        for (uint32_t c = lane; c < cstride; c += 32) dst[c] = c < nchan ? src[c] : 0.f;
    }
}

// One uploaded chunk of channel-major spectra (planes [c0, c1) of n samples)
// scattered to the sorted sample-major rows: 32 samples x 32 channels per
// block through shared memory; the last chunk also writes the zero padding
// channels up to cstride.
__global__ void k_scatter_cols(uint64_t n, uint32_t c0, uint32_t c1, uint32_t cend, uint32_t cstride,
                               const uint32_t *__restrict__ inv, const float *__restrict__ in,
                               float *__restrict__ out) {
    __shared__ float tile[32][33];
    const uint64_t j0 = (uint64_t)blockIdx.x * 32;
    const uint32_t cb = c0 + blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int r = ty; r < 32; r += 8) {
        const uint64_t j = j0 + tx;
        const uint32_t c = cb + r;
        tile[r][tx] = (j < n && c < c1) ? in[(uint64_t)(c - c0) * n + j] : 0.f;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const uint64_t j = j0 + r;
        const uint32_t c = cb + tx;
        if (j < n && c < cend) out[(uint64_t)__ldg(inv + j) * cstride + c] = tile[tx][r];
    }
}

}  // namespace

cudaError_t build_field(hcg_context *ctx, hcg_field *f, const double *d_lon, const double *d_lat,
                        const double *d_w, std::string &why) {
    cudaStream_t s = ctx->stream;
    const uint64_t n = f->n;
    cudaError_t e;
    uint64_t *k0 = nullptr, *k1 = nullptr;
    uint32_t *v0 = nullptr, *v1 = nullptr, *hist = nullptr;
    KeyRange *range = nullptr;
    RingSpan *span = nullptr;
    unsigned long long *wbits = nullptr;
    uint32_t nblocks = (uint32_t)((n + kSortTile - 1) / kSortTile);
#define TRY(x)                         \
    do {                               \
        e = (x);                       \
        if (e != cudaSuccess) goto fail; \
    } while (0)
    TRY(dalloc(&k0, (n + 1) * sizeof(uint64_t), s, ctx->pool));
    TRY(dalloc(&k1, (n + 1) * sizeof(uint64_t), s, ctx->pool));
    TRY(dalloc(&v0, n * sizeof(uint32_t), s, ctx->pool));
    TRY(dalloc(&v1, n * sizeof(uint32_t), s, ctx->pool));
    TRY(dalloc(&hist, (size_t)256 * nblocks * sizeof(uint32_t), s, ctx->pool));
    TRY(dalloc(&range, sizeof(KeyRange) + sizeof(RingSpan), s, ctx->pool));
    span = reinterpret_cast<RingSpan *>(range + 1);
    TRY(cudaMemsetAsync(&ctx->d_stats->invalid_input, 0, sizeof(unsigned long long), s));
    k_init_range<<<1, 1, 0, s>>>(range);
    k_sample_keys<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(f->hpx, n, d_lon, d_lat, k0, v0, range, ctx->d_stats);
    TRY(cudaGetLastError());
    {
        KeyRange hr;
        unsigned long long invalid = 0;
        TRY(cudaMemcpyAsync(&hr, range, sizeof hr, cudaMemcpyDeviceToHost, s));
        TRY(cudaMemcpyAsync(&invalid, &ctx->d_stats->invalid_input, sizeof invalid, cudaMemcpyDeviceToHost, s));
        TRY(cudaStreamSynchronize(s));
        if (invalid) {
            why = "non-finite coordinates or |lat| > 90 in " + std::to_string(invalid) + " samples";
            e = cudaErrorInvalidValue;
            goto fail;
        }
        uint64_t span_bits = 64 - (hr.kmax == hr.kmin ? 64 : __builtin_clzll(hr.kmax - hr.kmin));
        int passes = (int)((span_bits + 7) / 8);
        for (int p = 0; p < passes; ++p) {
            int shift = 8 * p;
            k_rs_hist<<<nblocks, kSortThreads, 0, s>>>(k0, n, shift, hr.kmin, hist, nblocks);
            k_scan_u32_1block<<<1, 1024, 0, s>>>(hist, (uint64_t)256 * nblocks);
            k_rs_scatter<<<nblocks, kSortThreads, 0, s>>>(k0, v0, k1, v1, n, shift, hr.kmin, hist, nblocks);
            TRY(cudaGetLastError());
            std::swap(k0, k1);
            std::swap(v0, v1);
        }
    }
    k_ring_span<<<1, 1, 0, s>>>(f->hpx, n, k0, span);
    TRY(cudaGetLastError());
    {
        RingSpan hs;
        TRY(cudaMemcpyAsync(&hs, span, sizeof hs, cudaMemcpyDeviceToHost, s));
        TRY(cudaStreamSynchronize(s));
        f->firstring = hs.firstring;
        f->usedrings = hs.usedrings;
    }
    f->d_keys = k0;
    f->d_perm = v0;
    k0 = nullptr;
    v0 = nullptr;
    TRY(dalloc(&f->d_lut, (f->usedrings + 1) * sizeof(uint32_t), s, ctx->pool));
    TRY(dalloc(&f->d_rings, f->usedrings * sizeof(RingRec), s, ctx->pool));
    k_ring_lut<<<(unsigned)((f->usedrings + 1 + 255) / 256), 256, 0, s>>>(f->hpx, n, f->d_keys, f->firstring,
                                                                          f->usedrings, f->d_lut);
    k_ring_table<<<(unsigned)((f->usedrings + 255) / 256), 256, 0, s>>>(f->hpx, f->firstring, f->usedrings, f->d_lut,
                                                                        f->d_keys, f->d_rings, ctx->d_stats);
    TRY(cudaGetLastError());
    {
        // Pixel tables: one u32 per HEALPix pixel between the first and last
        // sample of each ring, when they fit in max(2^24, 4n) entries
        // (HCG_RING_TABLE_MAX overrides; 0 keeps the binary searches).
        uint64_t cap = std::max<uint64_t>(1ull << 24, 4 * n);
        if (const char *v = getenv("HCG_RING_TABLE_MAX")) cap = strtoull(v, nullptr, 10);
        std::vector<RingRec> hr(f->usedrings);
        TRY(cudaMemcpyAsync(hr.data(), f->d_rings, hr.size() * sizeof(RingRec), cudaMemcpyDeviceToHost, s));
        TRY(cudaStreamSynchronize(s));
        uint64_t total = 0;
        for (RingRec &R : hr) {
            R.tbl = total;
            total += R.span;
        }
        if (total > 0 && total <= cap && dalloc(&f->d_ptab, total * sizeof(uint32_t), s, ctx->pool) == cudaSuccess) {
            TRY(cudaMemcpyAsync(f->d_rings, hr.data(), hr.size() * sizeof(RingRec), cudaMemcpyHostToDevice, s));
            k_ring_ptab<<<(unsigned)f->usedrings, 256, 0, s>>>(f->d_rings, f->d_keys, f->d_ptab);
            TRY(cudaGetLastError());
            TRY(cudaStreamSynchronize(s));  // the host copy of the table must outlive the upload
        } else {
            cudaGetLastError();
            for (RingRec &R : hr) R.span = 0, R.tbl = 0;
            TRY(cudaMemcpyAsync(f->d_rings, hr.data(), hr.size() * sizeof(RingRec), cudaMemcpyHostToDevice, s));
            TRY(cudaStreamSynchronize(s));
        }
        f->ptab_entries = f->d_ptab ? total : 0;
    }
    TRY(dalloc(&f->d_l2, n * sizeof(double), s, ctx->pool));
    TRY(dalloc(&f->d_b2, n * sizeof(double), s, ctx->pool));
    TRY(dalloc(&f->d_cb2, n * sizeof(double), s, ctx->pool));
    TRY(dalloc(&f->d_half, n * sizeof(double4), s, ctx->pool));
    TRY(dalloc(&f->d_w, n * sizeof(double), s, ctx->pool));
    TRY(dalloc(&wbits, sizeof(unsigned long long), s, ctx->pool));
    TRY(dalloc(&f->d_inv, n * sizeof(uint32_t), s, ctx->pool));
    k_inverse_perm<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, f->d_perm, f->d_inv);
    TRY(cudaGetLastError());
    TRY(cudaMemsetAsync(wbits, 0, sizeof(unsigned long long), s));
    k_permute_geometry<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, f->d_perm, d_lon, d_lat, d_w, f->d_l2, f->d_b2,
                                                                   f->d_cb2, f->d_w, f->d_half, wbits);
    TRY(cudaGetLastError());
    k_ring_phi<<<(unsigned)f->usedrings, 256, 0, s>>>(f->hpx, f->d_rings, f->d_keys, f->d_l2, f->d_b2, f->d_cb2);
    TRY(cudaGetLastError());
    f->wmax = 1.0;
    if (d_w) {
        unsigned long long hb = 0;
        TRY(cudaMemcpyAsync(&hb, wbits, sizeof hb, cudaMemcpyDeviceToHost, s));
        TRY(cudaStreamSynchronize(s));
        memcpy(&f->wmax, &hb, sizeof hb);
    }
fail:
    if (wbits) cudaFreeAsync(wbits, s);
    if (k0) cudaFreeAsync(k0, s);
    if (k1) cudaFreeAsync(k1, s);
    if (v0) cudaFreeAsync(v0, s);
    if (v1) cudaFreeAsync(v1, s);
    if (hist) cudaFreeAsync(hist, s);
    if (range) cudaFreeAsync(range, s);
#undef TRY
    return e;
}

// Spectra from host memory, uploaded in chunks of kUploadChunk bytes through
// two staging buffers: the copy of chunk k + 1 (copy stream) overlaps the
// scatter of chunk k into sorted order (context stream). Copies wait for the
// work queued on the context stream before the call, and every later use of
// the spectra is ordered after the last scatter on the context stream.
cudaError_t upload_spectra(hcg_context *ctx, hcg_field *f, const float *h_in, uint32_t nchan, int layout) {
    cudaStream_t s = ctx->stream, cs = ctx->copy_stream;
    const uint32_t cstride = (nchan + 3) & ~3u;
    if (f->d_spec && f->cstride != cstride) {
        cudaFreeAsync(f->d_spec, s);
        f->d_spec = nullptr;
    }
    cudaError_t e = cudaSuccess;
    if (!f->d_spec) e = dalloc(&f->d_spec, f->n * cstride * sizeof(float), s, ctx->pool);
    if (e != cudaSuccess) return e;
    f->nchan = nchan;
    f->cstride = cstride;
    const uint64_t n = f->n;
    // chunk geometry: whole input rows (sample-major) or whole planes (channel-major)
    const uint64_t unit = layout == HCG_LAYOUT_SAMPLE_MAJOR ? (uint64_t)nchan * 4 : n * 4;
    const uint64_t units = layout == HCG_LAYOUT_SAMPLE_MAJOR ? n : nchan;
    const uint64_t per = std::max<uint64_t>(1, kUploadChunk / unit);
    float *stage[2];
    for (int b = 0; b < 2; ++b) {
        stage[b] = (float *)ctx->scratch.get(19 + b, std::min(per, units) * unit, s, e);
        if (e != cudaSuccess) return e;
    }
    if ((e = cudaEventRecord(ctx->evu[4], s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(cs, ctx->evu[4], 0)) != cudaSuccess) return e;
    uint64_t k = 0;
    for (uint64_t u0 = 0; u0 < units; u0 += per, ++k) {
        const uint64_t cnt = std::min(per, units - u0);
        const int b = (int)(k & 1);
        if (k >= 2 && (e = cudaStreamWaitEvent(cs, ctx->evu[2 + b], 0)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(stage[b], h_in + u0 * (unit / 4), cnt * unit, cudaMemcpyHostToDevice, cs)) !=
            cudaSuccess)
            return e;
        if ((e = cudaEventRecord(ctx->evu[b], cs)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, ctx->evu[b], 0)) != cudaSuccess) return e;
        if (layout == HCG_LAYOUT_SAMPLE_MAJOR) {
            const uint64_t threads = cnt * 32;
            k_scatter_rows<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(u0, cnt, nchan, cstride, f->d_inv,
                                                                             stage[b], f->d_spec);
        } else {
            const uint32_t c0 = (uint32_t)u0, c1 = (uint32_t)(u0 + cnt);
            const uint32_t cend = c1 == nchan ? cstride : c1;  // the last chunk writes the padding
            dim3 grid((unsigned)((n + 31) / 32), (cend - c0 + 31) / 32);
            k_scatter_cols<<<grid, dim3(32, 8), 0, s>>>(n, c0, c1, cend, cstride, f->d_inv, stage[b], f->d_spec);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = cudaEventRecord(ctx->evu[2 + b], s)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// `nb` channel planes (host floats [nb][n] at h_planes) into f's sorted
// spectra, in chunks of whole planes through the two staging buffers: copies
// on cs, scatters on us. A chunk's copy waits until the scatter that last read
// its staging buffer is done (ev_free), the scatter for its copy (ev_copied);
// `chunks` counts the chunks of every call that shares the staging buffers.
cudaError_t upload_plane_block(hcg_context *ctx, hcg_field *f, const float *h_planes, uint32_t nb, cudaStream_t cs,
                               cudaStream_t us, float *const stage[2], uint64_t stage_bytes,
                               cudaEvent_t ev_copied[2], cudaEvent_t ev_free[2], uint64_t &chunks) {
    const uint32_t cstride = (nb + 3) & ~3u;
    const uint64_t n = f->n;
    cudaError_t e = cudaSuccess;
    if (f->d_spec && f->cstride != cstride) {
        cudaFreeAsync(f->d_spec, us);
        f->d_spec = nullptr;
    }
    if (!f->d_spec && (e = dalloc(&f->d_spec, n * cstride * sizeof(float), us, ctx->pool)) != cudaSuccess) return e;
    f->nchan = nb;
    f->cstride = cstride;
    if (n == 0) return cudaSuccess;
    const uint64_t per = std::max<uint64_t>(1, stage_bytes / (n * 4));
    for (uint64_t u0 = 0; u0 < nb; u0 += per, ++chunks) {
        const uint64_t cnt = std::min<uint64_t>(per, nb - u0);
        const int b = (int)(chunks & 1);
        if (chunks >= 2 && (e = cudaStreamWaitEvent(cs, ev_free[b], 0)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(stage[b], h_planes + u0 * n, cnt * n * 4, cudaMemcpyHostToDevice, cs)) != cudaSuccess)
            return e;
        if ((e = cudaEventRecord(ev_copied[b], cs)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(us, ev_copied[b], 0)) != cudaSuccess) return e;
        const uint32_t c0 = (uint32_t)u0, c1 = (uint32_t)(u0 + cnt);
        const uint32_t cend = c1 == nb ? cstride : c1;  // the last chunk writes the padding
        dim3 grid((unsigned)((n + 31) / 32), (cend - c0 + 31) / 32);
        k_scatter_cols<<<grid, dim3(32, 8), 0, us>>>(n, c0, c1, cend, cstride, f->d_inv, stage[b], f->d_spec);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = cudaEventRecord(ev_free[b], us)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t permute_spectra(hcg_context *ctx, hcg_field *f, const float *d_in, uint32_t nchan, int layout) {
    cudaStream_t s = ctx->stream;
    uint32_t cstride = (nchan + 3) & ~3u;
    if (f->d_spec && f->cstride != cstride) {
        cudaFreeAsync(f->d_spec, s);
        f->d_spec = nullptr;
    }
    cudaError_t e = cudaSuccess;
    if (!f->d_spec) e = dalloc(&f->d_spec, f->n * cstride * sizeof(float), s, ctx->pool);
    if (e != cudaSuccess) return e;
    f->nchan = nchan;
    f->cstride = cstride;
    if (layout == HCG_LAYOUT_SAMPLE_MAJOR) {
        uint64_t threads = f->n * 32;
        k_permute_rows<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(f->n, nchan, cstride, f->d_perm, d_in,
                                                                         f->d_spec);
    } else {
        dim3 grid((unsigned)((f->n + 31) / 32), (cstride + 31) / 32);
        k_permute_cols<<<grid, dim3(32, 8), 0, s>>>(f->n, nchan, cstride, f->d_perm, d_in, f->d_spec);
    }
    return cudaGetLastError();
}

}  // namespace hcg
