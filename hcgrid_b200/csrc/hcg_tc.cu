// Tensor-core engine, host side and the single-job launch: the hi/lo split
// of a field's spectra and k_tile_tc, one CTA per (tile, channel block). The
// per-tile pipeline (tcgen05 MMAs fed by TMA) is in hcg_tc.cuh.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>
#include <string>

#include "hcg_internal.h"
#include "hcg_kernels.cuh"
#include "hcg_tc.cuh"

namespace hcg {
namespace {

template <class Cfg>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_tile_tc(const __grid_constant__ CUtensorMap tm, const __grid_constant__ CUtensorMap tm_out, int has_out, TcJob J,
              unsigned long long *timeouts, unsigned long long *macs) {
    __shared__ TcShared S;
    J.map = &tm;
    J.out_map = has_out ? &tm_out : nullptr;
    const uint64_t tile = J.T.t0 + blockIdx.x;
    tc_load_rings(S, J.T, tile);
    tc_setup<Cfg>(S);  // ends with a CTA barrier
    if (threadIdx.x == 0) sm100::prefetch_tensormap(&tm);
    uint32_t gk = 0;
    tc_item<Cfg>(S, J, tile, blockIdx.y, gk, 0, timeouts, macs);
    tc_teardown<Cfg>(S, gk, timeouts);
}

template <class Cfg>
__global__ void __launch_bounds__(kTcPersistThreads, 1)
    k_tile_tc_persist(const __grid_constant__ CUtensorMap tm, TcJob J, uint64_t nitems, uint64_t ntiles,
                      unsigned long long *timeouts, unsigned long long *macs) {
    __shared__ TcPShared S;
    J.map = &tm;
    J.out_map = nullptr;
    if (threadIdx.x == 0) sm100::prefetch_tensormap(&tm);
    tc_persist<Cfg>(S, J, nitems, ntiles, timeouts, macs);
}

template <class Cfg>
__global__ void __launch_bounds__(kTcDThreads, 1)
    k_tile_tc_weights(const __grid_constant__ CUtensorMap tm, TcJob J, uint64_t nitems, uint64_t ntiles,
                      unsigned long long *timeouts, unsigned long long *macs) {
    __shared__ TcDShared S;
    J.map = &tm;
    J.out_map = nullptr;
    if (threadIdx.x == 0) sm100::prefetch_tensormap(&tm);
    tc_persist_weights<Cfg>(S, J, nitems, ntiles, timeouts, macs);
}

// ------------------------------------------------------------ spectra split
// Per-channel largest magnitude and the count of non-finite values.
__global__ void k_split_amax(const float *__restrict__ spec, uint64_t n, uint32_t nchan, uint32_t cstride,
                             uint32_t rows_per_block, unsigned int *amax_bits,
                             unsigned long long *nonfinite) {
    const uint32_t ch = blockIdx.x * blockDim.x + threadIdx.x;
    if (ch >= nchan) return;
    const uint64_t r0 = (uint64_t)blockIdx.y * rows_per_block;
    const uint64_t r1 = r0 + rows_per_block < n ? r0 + rows_per_block : n;
    unsigned int m = 0;
    unsigned long long bad = 0;
    for (uint64_t r = r0; r < r1; ++r) {
        const float v = spec[r * cstride + ch];
        if (!isfinite(v)) {
            ++bad;
            continue;
        }
        m = max(m, __float_as_uint(fabsf(v)));
    }
    atomicMax(amax_bits + ch, m);
    if (bad) atomicAdd(nonfinite, bad);
}

// Channel scales: FP16 keeps |x| * scale in [2^13, 2^14); BF16 needs none.
__global__ void k_split_scales(const unsigned int *amax_bits, uint32_t nchan, uint32_t cpad, uint32_t fmt,
                               float wscale, float *scale, float *inv_scale) {
    const uint32_t ch = blockIdx.x * blockDim.x + threadIdx.x;
    if (ch >= cpad) return;
    float s = 1.f;
    if (fmt == 0 && ch < nchan) {
        const float a = __uint_as_float(amax_bits[ch]);
        if (a > 0.f) {
            int ex;
            frexpf(a, &ex);  // a = f * 2^ex, f in [0.5, 1)
            s = ldexpf(1.f, max(-126, min(127, 14 - ex)));
        }
    }
    scale[ch] = s;
    inv_scale[ch] = 1.f / (s * wscale);  // powers of two: exact
}

// hi/lo halves in one array, channel-blocked: element (row r, channel c) of
// half h at [h][c / 64][r][c % 64], so 8 consecutive rows of one 64-channel
// block are one contiguous kilobyte and one 4-D TMA box brings both halves.
// A thread takes 8 channels of a row (two 16-byte loads, one 16-byte store
// per half), a block kSplitRows rows.
constexpr uint32_t kSplitRows = 32;
__global__ void __launch_bounds__(256) k_split(const float *__restrict__ spec, uint64_t n, uint32_t nchan,
                                               uint32_t cstride, uint32_t cpad, uint32_t fmt,
                                               const float *__restrict__ scale, uint16_t *hi, uint16_t *lo) {
    const uint32_t opr = cpad / 8;  // channel octets per row
    const uint64_t r0 = (uint64_t)blockIdx.x * kSplitRows;
    const uint32_t nr = (uint32_t)(n - r0 < kSplitRows ? n - r0 : kSplitRows);
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint32_t k = threadIdx.x; k < nr * opr; k += blockDim.x) {
        const uint32_t rr = k / opr, c0 = 8 * (k - rr * opr);
        const uint64_t r = r0 + rr;
        const float *src = spec + r * cstride;
        // cstride is a multiple of 4: a float4 lies wholly inside the row or wholly past it
        const float4 a = c0 < cstride ? *reinterpret_cast<const float4 *>(src + c0) : zero;
        const float4 b = c0 + 4 < cstride ? *reinterpret_cast<const float4 *>(src + c0 + 4) : zero;
        const float4 s0 = *reinterpret_cast<const float4 *>(scale + c0);
        const float4 s1 = *reinterpret_cast<const float4 *>(scale + c0 + 4);
        const float v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        const float sc[8] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y, s1.z, s1.w};
        uint32_t h[4], l[4];
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
            uint16_t hh[2], ll[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                float x = c0 + j + u < nchan ? v[j + u] : 0.f;
                if (!isfinite(x)) x = 0.f;  // such fields are refused by the engine; keep the arrays finite
                x *= sc[j + u];
                hh[u] = tc_to16(x, fmt);
                ll[u] = tc_to16(x - tc_from16(hh[u], fmt), fmt);
            }
            h[j / 2] = (uint32_t)hh[0] | ((uint32_t)hh[1] << 16);
            l[j / 2] = (uint32_t)ll[0] | ((uint32_t)ll[1] << 16);
        }
        const uint64_t o = ((uint64_t)(c0 >> 6) * n + r) * 64 + (c0 & 63);  // lo = hi + (cpad / 64) n 64
        *reinterpret_cast<uint4 *>(hi + o) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4 *>(lo + o) = make_uint4(l[0], l[1], l[2], l[3]);
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        else
            cudaGetLastError();
    });
    return fn;
}

// [2][cpad / 64][rows][64] 16-bit array: boxes of 64 channels x 8 rows x nb
// channel blocks x 2 halves, 128-byte swizzle (each 64 x 8 slab is one
// MN-major atom)
bool make_map(CUtensorMap *m, const uint16_t *base, uint64_t rows, uint32_t cpad, uint32_t nb) {
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[4] = {64, rows, cpad / 64, 2};
    cuuint64_t strides[3] = {128, (cuuint64_t)rows * 128, (cuuint64_t)rows * 128 * (cpad / 64)};
    cuuint32_t box[4] = {64, 8, nb, 2};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT16, 4, (void *)base, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

void free_split(hcg_field *f, cudaStream_t s) {
    if (f->d_xhi) cudaFreeAsync(f->d_xhi, s);  // the lo half lives in the same allocation
    if (f->d_xinv) cudaFreeAsync(f->d_xinv, s);
    f->d_xhi = f->d_xlo = nullptr;
    f->d_xinv = nullptr;
    f->xcpad = 0;
    f->xfmt = 0;
    f->xnonfinite = 0;
}

// Power-of-two scale of the weight operand: BF16 holds any weight as it is;
// FP16 weights are scaled so that the field's weight bound stays below 2^15
// (2^15 for |w| <= 1, the kernels' own bound with unit sample weights).
static float tc_weight_scale(const hcg_field *f, bool bf16) {
    if (bf16 || !tc_weights_fit(f)) return 1.f;  // the engine refuses fields beyond 2^100
    int e = 0;
    if (f->wbound > 1.0) frexp(f->wbound, &e);  // wbound < 2^e
    return ldexpf(1.f, 15 - e);
}

cudaError_t split_spectra(hcg_context *ctx, hcg_field *f, int fmt_engine, std::string &why) {
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    const uint32_t fmt = fmt_engine == HCG_ENGINE_TC_BF16 ? 1u : 0u;
    const uint32_t cpad = (f->nchan + 63) / 64 * 64;
    const uint64_t n = f->n;
    uint16_t *hi = nullptr, *lo = nullptr;
    float *scale = nullptr, *inv = nullptr;
    unsigned int *amax = nullptr;
    unsigned long long *bad = nullptr;
    const size_t nb = (size_t)n * cpad * sizeof(uint16_t);
    if ((e = dalloc(&hi, nb ? 2 * nb : 16, s, ctx->pool)) != cudaSuccess ||
        (e = dalloc(&scale, cpad * sizeof(float), s, ctx->pool)) != cudaSuccess ||
        (e = dalloc(&inv, cpad * sizeof(float), s, ctx->pool)) != cudaSuccess ||
        (e = dalloc(&amax, cpad * sizeof(unsigned int) + sizeof(unsigned long long), s, ctx->pool)) != cudaSuccess) {
        why = "split spectra of " + std::to_string(2 * nb) + " bytes";
        if (hi) cudaFreeAsync(hi, s);
        if (scale) cudaFreeAsync(scale, s);
        if (inv) cudaFreeAsync(inv, s);
        return e;
    }
    lo = hi + (size_t)n * cpad;  // [2][cpad / 64][n][64]: the lo half follows the hi half
    bad = (unsigned long long *)(amax + cpad);  // cpad is a multiple of 64: 8-byte aligned
    cudaMemsetAsync(amax, 0, cpad * sizeof(unsigned int) + sizeof(unsigned long long), s);
    const float wscale = tc_weight_scale(f, fmt != 0);
    if (n > 0) {
        const uint32_t rpb = 4096;
        dim3 grid((f->nchan + 255) / 256, (unsigned)((n + rpb - 1) / rpb));
        k_split_amax<<<grid, 256, 0, s>>>(f->d_spec, n, f->nchan, f->cstride, rpb, amax, bad);
    }
    k_split_scales<<<(cpad + 255) / 256, 256, 0, s>>>(amax, f->nchan, cpad, fmt, wscale, scale, inv);
    if (n > 0)
        k_split<<<(unsigned)((n + kSplitRows - 1) / kSplitRows), 256, 0, s>>>(f->d_spec, n, f->nchan, f->cstride,
                                                                              cpad, fmt, scale, hi, lo);
    unsigned long long nonfinite = 0;
    cudaMemcpyAsync(&nonfinite, bad, sizeof(nonfinite), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(amax, s);
    cudaFreeAsync(scale, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess) {
        cudaFreeAsync(hi, s);
        cudaFreeAsync(inv, s);
        return e;
    }
    free_split(f, s);
    f->d_xhi = hi;
    f->d_xlo = lo;
    f->d_xinv = inv;
    f->xcpad = cpad;
    f->xfmt = fmt_engine;
    f->xnonfinite = nonfinite;
    return cudaSuccess;
}

// The cube as a 3-D tensor whose box is one item (tile x channel block):
// [y][x][channel] for sample-major cubes, [channel][y][x] for channel-major
// ones. false when a stride is not a multiple of 16 bytes (the kernel then
// stores directly).
bool tc_out_map(CUtensorMap *m, float *out, uint32_t ostride, uint32_t nx, uint32_t ny, uint32_t nchan,
                uint32_t nb) {
    auto fn = encode_fn();
    if (!fn || ((uintptr_t)out & 15)) return false;
    cuuint64_t dims[3];
    cuuint64_t strides[2];
    cuuint32_t box[3];
    if (ostride) {
        if (ostride != nchan || (nchan & 3)) return false;
        dims[0] = nchan; dims[1] = nx; dims[2] = ny;
        strides[0] = (cuuint64_t)nchan * 4; strides[1] = (cuuint64_t)nx * nchan * 4;
        box[0] = 64 * nb; box[1] = kTileX; box[2] = kTileY;
    } else {
        if (nx & 3) return false;
        dims[0] = nx; dims[1] = ny; dims[2] = nchan;
        strides[0] = (cuuint64_t)nx * 4; strides[1] = (cuuint64_t)nx * ny * 4;
        box[0] = kTileX; box[1] = kTileY; box[2] = 64 * nb;
    }
    cuuint32_t estr[3] = {1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)out, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

void tc_entry_format(const hcg_field *f, uint32_t &fmt, float &wscale) {
    fmt = f->xfmt == HCG_ENGINE_TC_BF16 ? 1u : 0u;
    wscale = tc_weight_scale(f, fmt != 0);
}

bool tc_prepare_job(const hcg_field *f, int nb_max, CUtensorMap *map, TcJob &J) {
    const uint32_t nblk64 = f->xcpad / 64;
    J.nb = nblk64 < (uint32_t)nb_max ? nblk64 : (uint32_t)nb_max;
    J.ncb = (nblk64 + J.nb - 1) / J.nb;
    if (!make_map(map, f->d_xhi, f->n, f->xcpad, J.nb)) return false;
    J.nchan = f->nchan;
    J.nrows = (uint32_t)f->n;
    J.fmt = f->xfmt == HCG_ENGINE_TC_BF16 ? 1u : 0u;
    J.wscale = tc_weight_scale(f, J.fmt != 0);
    J.inv_scale = f->d_xinv;
    return true;
}

cudaError_t tc_set_smem(const void *kernel, uint32_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

// Pipeline shape for a field: the autotuned choice of its channel class,
// else the widest item its channels fill.
void tc_pipeline(const hcg_context *ctx, const hcg_field *f, TcJob &J) {
    const int c = tc_class_of(f->xcpad);
    J.pf = (uint32_t)(ctx->tc_pf[c] >= 0 ? ctx->tc_pf[c] : kTcDefaultPrefetch);
    J.strip = (uint32_t)(ctx->tc_strip[c] >= 0 ? ctx->tc_strip[c] : kTcDefaultStrip);
}

int tc_pick(const hcg_context *ctx, const hcg_field *f) {
    const int t = ctx->tc_config[tc_class_of(f->xcpad)];
    if (t >= 0 && t < kTcConfigCount) return t;
    const uint32_t b = f->xcpad / 64;
    return b >= 4 ? 4 : (b >= 2 ? 1 : 2);
}

namespace {
template <class Cfg>
cudaError_t launch_tc_persist(hcg_context *ctx, const hcg_field *f, TcJob &J, const TileArgs &T, uint64_t ntiles,
                              std::string &why) {
    cudaStream_t s = ctx->stream;
    CUtensorMap tm;
    if (!tc_prepare_job(f, Cfg::kNb, &tm, J)) {
        why = "cuTensorMapEncodeTiled";
        return cudaErrorInvalidValue;
    }
    static bool attr_set = false;  // per instantiation
    if (!attr_set) {
        cudaError_t e = tc_set_smem((const void *)k_tile_tc_persist<Cfg>, Cfg::kSmem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
    J.T = T;
    const uint64_t nitems = ntiles * J.ncb;
    const unsigned grid = (unsigned)std::min<uint64_t>(nitems, (uint64_t)(nsm > 0 ? nsm : 148));
    if (grid == 0) return cudaSuccess;
    k_tile_tc_persist<Cfg><<<grid, kTcPersistThreads, Cfg::kSmem, s>>>(tm, J, nitems, ntiles,
                                                                      &ctx->d_stats->timeouts, &ctx->d_stats->tc_macs);
    return cudaGetLastError();
}

template <class Cfg>
cudaError_t launch_tc(hcg_context *ctx, const hcg_field *f, TcJob &J, const TileArgs &T, uint64_t ntiles,
                      std::string &why) {
    cudaStream_t s = ctx->stream;
    CUtensorMap tm, tm_out;
    if (!tc_prepare_job(f, Cfg::kNb, &tm, J)) {
        why = "cuTensorMapEncodeTiled";
        return cudaErrorInvalidValue;
    }
    const int has_out = tc_out_map(&tm_out, J.out, J.ostride, J.g.nx, J.g.ny, J.nchan, J.nb) ? 1 : 0;
    if (!has_out) memset(&tm_out, 0, sizeof tm_out);
    static bool attr_set = false;  // per instantiation
    if (!attr_set) {
        cudaError_t e = tc_set_smem((const void *)k_tile_tc<Cfg>, Cfg::kSmem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    for (uint64_t t0 = 0; t0 < ntiles; t0 += 0x7fffffffull) {
        J.T = T;
        J.T.t0 = T.t0 + t0;
        dim3 grid((unsigned)std::min<uint64_t>(ntiles - t0, 0x7fffffffull), J.ncb);
        k_tile_tc<Cfg><<<grid, kTcThreads, Cfg::kSmem, s>>>(tm, tm_out, has_out, J, &ctx->d_stats->timeouts,
                                                            &ctx->d_stats->tc_macs);
    }
    return cudaGetLastError();
}
}  // namespace

namespace {
template <class Cfg>
cudaError_t launch_tc_weights(hcg_context *ctx, const hcg_field *f, TcJob &J, const TileArgs &T, uint64_t ntiles,
                              std::string &why) {
    cudaStream_t s = ctx->stream;
    CUtensorMap tm;
    if (!tc_prepare_job(f, Cfg::kNb, &tm, J)) {
        why = "cuTensorMapEncodeTiled";
        return cudaErrorInvalidValue;
    }
    static bool attr_set = false;  // per instantiation
    if (!attr_set) {
        cudaError_t e = tc_set_smem((const void *)k_tile_tc_weights<Cfg>, Cfg::kSmem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
    J.T = T;
    const uint64_t nitems = ntiles * J.ncb;
    const unsigned grid = (unsigned)std::min<uint64_t>(nitems, (uint64_t)(nsm > 0 ? nsm : 148));
    if (grid == 0) return cudaSuccess;
    k_tile_tc_weights<Cfg><<<grid, kTcDThreads, Cfg::kSmem, s>>>(tm, J, nitems, ntiles,
                                                                      &ctx->d_stats->timeouts, &ctx->d_stats->tc_macs);
    return cudaGetLastError();
}
}  // namespace

cudaError_t tc_weights(hcg_context *ctx, const hcg_field *f, const GridArgs &a, const GroupArgs &g,
                       const TileArgs &T, uint64_t ntiles, float *out, uint32_t ostride, float *wout,
                       std::string &why) {
    TcJob J{};
    J.a = a;
    J.g = g;
    J.out = out;
    J.ostride = ostride;
    J.wout = wout;
    tc_pipeline(ctx, f, J);
    const uint32_t b = f->xcpad / 64;
    if (b >= 4) return launch_tc_weights<TcCfgN4S2>(ctx, f, J, T, ntiles, why);
    if (b >= 2) return launch_tc_weights<TcCfgN2S3>(ctx, f, J, T, ntiles, why);
    return launch_tc_weights<TcCfgN1S4>(ctx, f, J, T, ntiles, why);
}

cudaError_t tc_accum(hcg_context *ctx, const hcg_field *f, const GroupArgs &g, const TileArgs &T, uint64_t ntiles,
                     const unsigned long long *off, const uint32_t *cnt, const uint32_t *e_slot, const float4 *e_w,
                     const double *wsum, float *out, uint32_t ostride, float *wout, unsigned long long umax,
                     std::string &why) {
    TcJob J{};
    J.g = g;
    J.off = off;
    J.cnt = cnt;
    J.e_slot = e_slot;
    J.e_w = e_w;
    J.wsum = wsum;
    J.out = out;
    J.ostride = ostride;
    J.wout = wout;
    tc_pipeline(ctx, f, J);
    int cfg = tc_pick(ctx, f);
    // tiles longer than one accumulation segment take the persistent kernel,
    // which accumulates in segments (the one-item kernel does not)
    if (cfg < 4 && umax > kTcOneSegmentSlots) cfg = cfg == 3 ? 5 : 4;
    switch (cfg) {
        case 0: return launch_tc<TcCfgN4S2>(ctx, f, J, T, ntiles, why);
        case 1: return launch_tc<TcCfgN2S3>(ctx, f, J, T, ntiles, why);
        case 2: return launch_tc<TcCfgN1S4>(ctx, f, J, T, ntiles, why);
        case 3: return launch_tc<TcCfgN4K32>(ctx, f, J, T, ntiles, why);
        case 4: return launch_tc_persist<TcCfgN4S2>(ctx, f, J, T, ntiles, why);
        default: return launch_tc_persist<TcCfgN4K32>(ctx, f, J, T, ntiles, why);
    }
}

}  // namespace hcg
