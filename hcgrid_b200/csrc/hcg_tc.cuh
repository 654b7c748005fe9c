// Tensor-core channel accumulation (tcgen05, sm_100a): the per-tile device
// code of the single-job kernels (hcg_tc.cu: one item per CTA, persistent,
// and persistent with in-kernel weights) and of the persistent batch kernel
// (hcg_batch.cu).
//
// For one 16x8-pixel tile the gridded cube is a dense product
//     cube[pixel][channel] = sum_slot W[pixel][slot] * X[slot][channel]
// where the slots are the tile's staged samples (the union of the ring
// windows of its pixels, one contiguous run of sorted samples per HEALPix
// ring, padded to a multiple of 8) and W holds the GAUSS1D weights of the
// pairs inside sphere_radius (FP64 distance and cutoff, FP32 Gaussian; zero
// elsewhere): the weights the FP32 engine sums. The product runs on the 5th-generation tensor cores as a
// compensated 16-bit split, W = Wh + Wl and X = Xh + Xl with
// hi = round(x), lo = round(x - hi):
//     W X ~= Wh Xh + Wh Xl + Wl Xh
// three kind::f16 MMAs per K step into one FP32 accumulator in tensor memory.
// Split formats: BF16 hi/lo (8 + 8 significant bits, per-term relative error
// <= 3 * 2^-16) or FP16 hi/lo (11 + 11 bits) with power-of-two scales per
// channel and for the weights that keep both halves in FP16's normal range
// (per-term error ~3 * 2^-22). Scales are powers of two: exact.
//
// One work item = one tile x up to 256 channels (nb 64-channel blocks).
// Warp roles in the one-item 192-thread CTA (the persistent kernels below
// add epilogue warps and, with in-kernel weights, more builders):
//   warp 0    producer: per K chunk (64 or 32 slots), the spectra: runs of 8
//             sorted samples, each one 4-D TMA box (64 channels x 8 rows x nb
//             channel blocks x hi/lo, 128-byte swizzle: the MN-major B atoms);
//   warp 1    TMEM allocation and MMA issue (one thread);
//   warps 2-5 zero their operand rows and write the weights of the chunk's
//             entries into the K-major operand (swizzled), then run the
//             epilogue: tcgen05.ld
//             of the accumulator, multiplication by the inverse channel
//             scales and by 1 / (FP64 weight sum) into a shared-memory tile
//             laid out as the cube's box, written by one TMA bulk tensor
//             store (direct stores where the cube's strides do not allow
//             TMA).
// The pipeline shapes (channels per item, chunk size, stages) are the
// TcCfg instances below. Pipeline counters run on across the items a CTA
// processes. Every wait is bounded
// (1 s of global time): a wait that runs out counts a timeout and sets the
// CTA's abort flag; the roles wind down, the producer waits (bounded) for its
// copies, TMEM is freed and the host reports HCG_ETIMEOUT.
//
// Padding slots of a ring run hold real neighbouring samples (or TMA zero
// fill past the last sample) with zero weight; a non-finite spectrum value
// would turn 0 * x into NaN across the tile, so fields with non-finite
// spectra are refused by the tensor-core engines (the FP32 engine grids them).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "hcg_kernels.cuh"
#include "hcg_sm100.cuh"

namespace hcg {

constexpr int kTcM = kTileX * kTileY;  // 128 pixels: the MMA's M
constexpr int kTcThreads = 192;
constexpr int kTcBuilders = 128;
constexpr uint64_t kTcWaitNs = 1000000000ull;
constexpr uint32_t kTcMaxN = 256;         // channels per item (the MMA's largest N)
static_assert(kTcM == 128, "a tile is one M=128 MMA");

// Pipeline shapes: NB 64-channel blocks per item (the MMA's N = 64 NB), K
// slots per chunk (64: 128-byte rows of the weight operand, 128-byte
// swizzle; 32: 64-byte rows, 64-byte swizzle) and ST stages, in 192 KB of
// operand buffers. More channels per item build the weight operand fewer
// times per channel; more (smaller) stages hide more copy latency.
template <int NB, int ST, int KC>
struct TcCfg {
    static constexpr int kNb = NB;
    static constexpr int kStages = ST;
    static constexpr int kK = KC;
    static constexpr uint32_t kAHalf = kTcM * KC * 2;          // weight operand hi (or lo)
    static constexpr uint32_t kARow = KC * 2;                  // bytes per operand row
    static constexpr uint32_t kAAtom = 8 * kARow;              // 8-row swizzle atom
    static constexpr uint32_t kALayout = KC == 64 ? 2u : 4u;   // descriptor layout: SWIZZLE_128B / _64B
    // the entries builders' MN-major weight operand: per 8-slot K group two
    // 1 KB atoms of 64 pixels x 8 slots (128-byte swizzle)
    static constexpr uint32_t kAMnGroup = 2048;
    static constexpr uint32_t kBGroup = 2 * NB * 1024;         // one 8-slot row group: hi blocks, lo blocks
    static constexpr uint32_t kBBytes = (KC / 8) * kBGroup;
    static constexpr uint32_t kStageBytes = 2 * kAHalf + kBBytes;
    static constexpr uint32_t kSmem = ST * kStageBytes + 1024;  // + alignment of the swizzle atoms
    static constexpr uint32_t kTmemCols = NB * 64 <= 64 ? 64 : (NB * 64 <= 128 ? 128 : 256);
    static_assert(KC == 64 || KC == 32, "chunks of 64 or 32 slots");
    static_assert(ST * kStageBytes <= 192 * 1024, "operand buffers fit shared memory");
};
using TcCfgN4S2 = TcCfg<4, 2, 64>;  // 256 channels per item, 64-slot chunks, 2 stages
using TcCfgN2S3 = TcCfg<2, 3, 64>;  // 128 channels, 64-slot chunks, 3 stages
using TcCfgN1S4 = TcCfg<1, 4, 64>;  // 64 channels, 64-slot chunks, 4 stages
using TcCfgN4K32 = TcCfg<4, 4, 32>;  // 256 channels, 32-slot chunks, 4 stages
// 4, 5: shapes 0 and 3 in the persistent kernel (one CTA per SM, epilogue
// overlapped with the next item)
static_assert(kTcConfigCount == 6, "hcg_tc_set_config numbers the shapes 0-3 above and 4-5 persistent");

// One job's tensor-core arguments.
struct TcJob {
    const CUtensorMap *map;  // [2][ncb64][n][64] 16-bit hi/lo arrays, boxes 64 x 8 x nb x 2
    GroupArgs g;
    TileArgs T;
    const unsigned long long *off;  // entry offset of each group (minus g.ebase)
    const uint32_t *cnt;
    const uint32_t *e_slot;
    const float4 *e_w;
    const double *wsum;
    uint32_t nb;        // 64-channel blocks per item (1..4)
    uint32_t ncb;       // items per tile (channel blocks of nb * 64)
    uint32_t nchan;
    uint32_t nrows;     // samples
    uint32_t fmt;       // 0: f16, 1: bf16
    float wscale;       // weight scale (power of two)
    const float *inv_scale;  // [cpad]: 1 / (channel scale * wscale)
    float *out;
    uint32_t ostride;   // 0: [channel][pixel]; else [pixel][ostride]
    float *wout;
    const CUtensorMap *out_map;  // 3-D map of the cube (null: direct stores); box = one item
    GridArgs a;                  // geometry of the direct-weight builders (tc_build_weights)
    uint32_t pf;                 // the producer prefetches chunk k + pf into L2 (pf <= stages: k + stages)
    uint32_t strip;              // persistent kernels' tile walk: strips of `strip` tile columns (0: rows)
};

// Tile of the q-th item of a persistent launch over whole tile rows (ntiles =
// rows x ntx): with strip > 0 the columns are taken in strips of `strip`
// tiles, each strip row by row, so the tiles in flight at once form a compact
// block whose neighbours share staged samples in L2; 0 walks whole rows.
__host__ __device__ __forceinline__ uint64_t tc_walk(uint64_t q, uint64_t ntiles, uint32_t ntx, uint32_t strip) {
    if (strip == 0 || strip >= ntx) return q;
    const uint64_t rows = ntiles / ntx;
    const uint64_t nfull = ntx / strip, full_items = nfull * rows * strip;
    if (q < full_items) {
        const uint64_t s = q / (rows * strip), r = q % (rows * strip);
        return (r / strip) * ntx + s * strip + r % strip;
    }
    const uint64_t rem = ntx - nfull * strip, r = q - full_items;
    return (r / rem) * ntx + nfull * strip + r % rem;
}

constexpr int kTcRing = 8;  // entries in flight per builder thread
constexpr int kTcMaxStages = 4;

struct TcShared {
    uint64_t full_a[kTcMaxStages], full_b[kTcMaxStages], empty[kTcMaxStages], acc_full;
    uint32_t tmem;
    volatile int abort;
    unsigned long long item;
    uint32_t ulo[kTileMaxRings], base[kTileMaxRings + 1];
    float inv_scale[kTcMaxN];              // the item's channels: 1 / (channel scale * weight scale)
    float4 ring_w[kTcRing * kTcBuilders];  // builders' entry rings, [position][thread]
    uint32_t ring_slot[kTcRing * kTcBuilders];
};

// hcg_tc.cu: the tensor maps and format fields of a field with split
// spectra (false: the maps could not be encoded); the shared-memory opt-in of
// a kernel built on tc_item.
bool tc_prepare_job(const hcg_field *f, int nb_max, CUtensorMap *map, TcJob &J);
bool tc_out_map(CUtensorMap *m, float *out, uint32_t ostride, uint32_t nx, uint32_t ny, uint32_t nchan, uint32_t nb);
cudaError_t tc_set_smem(const void *kernel, uint32_t bytes);
int tc_pick(const hcg_context *ctx, const hcg_field *f);
// the channel class's prefetch distance and tile walk into J
void tc_pipeline(const hcg_context *ctx, const hcg_field *f, TcJob &J);

namespace {

// byte offset of element (row m, column k) of a K-major 128-row x KC-column
// 16-bit operand in swizzled 8-row atoms (the 16-byte chunk index is XORed
// with address bits 7-9 for the 128-byte swizzle, 7-8 for the 64-byte one)
template <int KC>
__device__ __forceinline__ uint32_t tc_a_offset(uint32_t m, uint32_t k) {
    if (KC == 64) return (m >> 3) * 1024u + (m & 7u) * 128u + ((((k >> 3) ^ (m & 7u)) << 4) | ((k & 7u) << 1));
    return (m >> 3) * 512u + (m & 7u) * 64u + ((((k >> 3) ^ ((m >> 1) & 3u)) << 4) | ((k & 7u) << 1));
}

__device__ __forceinline__ uint8_t *tc_smem_base() {
    extern __shared__ uint8_t s_tc_raw[];
    return (uint8_t *)(((uintptr_t)s_tc_raw + 1023) & ~(uintptr_t)1023);
}

// Whole CTA: barriers and TMEM.
template <class Cfg>
__device__ __forceinline__ void tc_setup(TcShared &S) {
    using namespace sm100;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < Cfg::kStages; ++s) {
            mbar_init(&S.full_a[s], kTcBuilders);
            mbar_init(&S.full_b[s], 1);
            mbar_init(&S.empty[s], 1);
        }
        mbar_init(&S.acc_full, 1);
        S.abort = 0;
        mbar_fence_init();
    }
    if ((tid >> 5) == 1) {
        tmem_alloc(&S.tmem, Cfg::kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

template <class SH>
__device__ __forceinline__ void tc_give_up(SH &S, unsigned long long *timeouts) {
    atomicAdd(timeouts, 1ULL);
    S.abort = 1;
}

// Whole CTA, after its last item: the producer waits (bounded) for the copies
// of the last chunks of each stage, then TMEM is freed.
template <class Cfg>
__device__ __forceinline__ void tc_teardown(TcShared &S, uint32_t gk, unsigned long long *timeouts) {
    using namespace sm100;
    constexpr uint32_t ST = Cfg::kStages;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (uint32_t g = gk > ST ? gk - ST : 0; g < gk; ++g) {
            const uint32_t s = g % ST, ph = (g / ST) & 1;
            if (!mbar_wait(&S.full_b[s], ph, kTcWaitNs)) {
                tc_give_up(S, timeouts);
                break;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if ((tid >> 5) == 1) {
        tc_fence_after();
        tmem_dealloc(S.tmem, Cfg::kTmemCols);
    }
}

// Whole CTA: the tile's ring table into shared memory (caller syncs after).
__device__ __forceinline__ void tc_load_rings(TcShared &S, const TileArgs &T, uint64_t tile) {
    const int nrt = T.nr[tile];
    for (int j = threadIdx.x; j < nrt; j += kTcThreads) S.ulo[j] = T.ulo[tile * kTileMaxRings + j];
    for (int j = threadIdx.x; j <= nrt; j += kTcThreads) S.base[j] = T.base[tile * (kTileMaxRings + 1) + j];
}

// Operand buffers of one pipeline stage.
template <class Cfg>
struct TcStage {
    uint8_t *smem;
    __device__ __forceinline__ uint8_t *A_hi(uint32_t s) const { return smem + s * Cfg::kStageBytes; }
    __device__ __forceinline__ uint8_t *A_lo(uint32_t s) const { return smem + s * Cfg::kStageBytes + Cfg::kAHalf; }
    __device__ __forceinline__ uint8_t *B(uint32_t s) const { return smem + s * Cfg::kStageBytes + 2 * Cfg::kAHalf; }
};

// Producer (the whole warp 0), one item: per chunk one 4-D TMA box per run of
// 8 slots, issued by lanes 0..KC/8-1 in parallel; with J.pf > 0 lanes
// KC/8..2KC/8-1 also prefetch the boxes of chunk k + pf into L2. S.ulo /
// S.base hold the item's ring table (nrt rings); `gk` is the CTA's chunk count
// before the item.
template <class Cfg, class SH>
__device__ __forceinline__ void tc_produce(SH &S, const TcJob &J, uint32_t cblk, uint32_t U, uint32_t nchunks,
                                           uint32_t gk, int nrt, unsigned long long *timeouts) {
    using namespace sm100;
    constexpr uint32_t ST = Cfg::kStages, KC = Cfg::kK;
    constexpr int NB8 = (int)(KC / 8);
    const TcStage<Cfg> st{tc_smem_base()};
    const int lane = threadIdx.x & 31;
    const uint32_t bytes = NB8 * 2u * J.nb * 1024u;
    const uint32_t pf = J.pf > ST ? J.pf : ST;  // chunks ahead of the loads that go to L2 first
    const int nlanes = J.pf ? 2 * NB8 : NB8;     // pf 0: no prefetches
    // TMA row of slot0: the ring run j with base[j] <= slot0 < base[j + 1]
    auto row_of = [&](uint32_t slot0) -> int {
        if (slot0 >= U) return (int)J.nrows;  // past the last sample: zero fill
        int lo = 0, hi = nrt;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (S.base[mid] <= slot0) lo = mid; else hi = mid;
        }
        return (int)(S.ulo[lo] + (slot0 - S.base[lo]));
    };
    // the item's chunks [ST, pf) are prefetched at its start; chunk k + pf with chunk k
    for (uint32_t i = lane; J.pf && i < (pf - ST) * (uint32_t)NB8; i += 32) {
        const uint32_t c = ST + i / NB8;
        if (c < nchunks) tma_prefetch_4d(J.map, 0, row_of(c * KC + 8 * (i % NB8)), (int)(cblk * J.nb), 0);
    }
    for (uint32_t k = 0; k < nchunks; ++k) {
        const uint32_t g = gk + k, s = g % ST;
        int go = 1;
        if (lane == 0) {
            if (S.abort) {
                go = 0;
            } else if (g >= ST && !mbar_wait(&S.empty[s], ((g / ST) - 1) & 1, kTcWaitNs)) {
                tc_give_up(S, timeouts);
                go = 0;
            } else {
                mbar_arrive_expect_tx(&S.full_b[s], bytes);
            }
        }
        if (!__shfl_sync(0xffffffffu, go, 0)) break;
        const int b = lane % NB8;
        const uint32_t kk = lane < NB8 ? k : k + pf;
        if (lane < nlanes && kk < nchunks) {
            const int row = row_of(kk * KC + 8 * b);
            if (lane < NB8)
                tma_load_4d(st.B(s) + b * Cfg::kBGroup, J.map, &S.full_b[s], 0, row, (int)(cblk * J.nb), 0);
            else
                tma_prefetch_4d(J.map, 0, row, (int)(cblk * J.nb), 0);
        }
    }
}

// MMA issue (one thread), one item into the accumulator at `d_tmem`; every
// chunk's stage is released on its `empty` barrier when its MMAs complete.
// Returns false if a wait ran out.
template <class Cfg, class SH>
__device__ __forceinline__ bool tc_mma(SH &S, const TcJob &J, uint32_t nchunks, uint32_t gk, uint32_t d_tmem,
                                       unsigned long long *timeouts, unsigned long long *macs) {
    using namespace sm100;
    constexpr uint32_t ST = Cfg::kStages, KC = Cfg::kK;
    const TcStage<Cfg> st{tc_smem_base()};
    const uint32_t idesc = idesc_f16_mnmaj_a_mnmaj_b(J.fmt, kTcM, 64 * J.nb);
    uint32_t acc = 0;
    bool ok = true;
    for (uint32_t k = 0; k < nchunks && !S.abort; ++k) {
        const uint32_t g = gk + k, s = g % ST, ph = (g / ST) & 1;
        if (!mbar_wait(&S.full_a[s], ph, kTcWaitNs) || !mbar_wait(&S.full_b[s], ph, kTcWaitNs)) {
            tc_give_up(S, timeouts);
            ok = false;
            break;
        }
        tc_fence_after();
        const uint32_t ah = smem_u32(st.A_hi(s)), al = smem_u32(st.A_lo(s));
        const uint32_t bh = smem_u32(st.B(s)), bl = bh + J.nb * 1024;  // lo blocks follow the hi blocks
        // K step 0's descriptors; step kk adds its byte offset / 16 (two 8-slot
        // row groups per K step; 64-channel atoms 1 KB apart)
        const uint64_t adh = smem_desc(ah, 1024, Cfg::kAMnGroup, 2);  // MN-major A (tc_build)
        const uint64_t adl = smem_desc(al, 1024, Cfg::kAMnGroup, 2);
        const uint64_t bdh = smem_desc(bh, 1024, Cfg::kBGroup, 2);
        const uint64_t bdl = smem_desc(bl, 1024, Cfg::kBGroup, 2);
#pragma unroll
        for (int kk = 0; kk < (int)(KC / 16); ++kk) {
            const uint64_t ao = (uint64_t)(kk * 2 * Cfg::kAMnGroup / 16), bo = (uint64_t)(kk * 2 * Cfg::kBGroup / 16);
            mma_f16_ss(d_tmem, adh + ao, bdh + bo, idesc, acc);
            mma_f16_ss(d_tmem, adh + ao, bdl + bo, idesc, 1);
            mma_f16_ss(d_tmem, adl + ao, bdh + bo, idesc, 1);
            acc = 1;
        }
        mma_commit(&S.empty[s]);
    }
    if (acc) atomicAdd(macs, 3ull * kTcM * (64ull * J.nb) * (uint64_t)KC * nchunks);
    return ok;
}

// Accumulation segments of the persistent kernels: the tensor cores' FP32
// accumulation drops low bits of the products it adds (the sums come out low
// by up to ~2^-24 of the running sum per MMA), so long K loops drift. An
// item's chunks are accumulated in segments of kTcSegSlots staged slots (the
// last one also takes a remainder of up to half a segment), each in a fresh
// accumulator (the two TMEM halves in turn), and the epilogue adds the
// segments with round-to-nearest FP32 adds (in the cube buffer) before it
// normalises them.
constexpr uint32_t kTcSegSlots = 1024;
// The one-item kernels (k_tile_tc, the batch kernel) accumulate an item in one
// segment: they take tiles of at most this many staged slots (longer ones go to
// the persistent kernels).
constexpr uint32_t kTcOneSegmentSlots = 1536;

// segments of an item of `nchunks` chunks of KC slots
template <uint32_t KC>
__host__ __device__ constexpr uint32_t tc_segments(uint32_t nchunks) {
    constexpr uint32_t seg = kTcSegSlots / KC;  // chunks per segment
    return nchunks > seg + seg / 2 ? (nchunks + seg / 2 - 1) / seg : 1;
}

// MMA issue (one thread) of one item in segments; `gs` counts the CTA's
// segments (accumulator gs & 1, barriers acc_full / acc_empty by parity).
// AMN: the weight operand is MN-major (the entries builders, tc_build), else
// K-major (the direct builders, tc_build_weights).
template <class Cfg, bool AMN, class SH>
__device__ __forceinline__ void tc_mma_seg(SH &S, const TcJob &J, uint32_t nchunks, uint32_t gk, uint32_t &gs,
                                           unsigned long long *timeouts, unsigned long long *macs) {
    using namespace sm100;
    constexpr uint32_t ST = Cfg::kStages, KC = Cfg::kK;
    const TcStage<Cfg> st{tc_smem_base()};
    const uint32_t idesc =
        AMN ? idesc_f16_mnmaj_a_mnmaj_b(J.fmt, kTcM, 64 * J.nb) : idesc_f16_kmaj_a_mnmaj_b(J.fmt, kTcM, 64 * J.nb);
    const uint32_t nseg = tc_segments<KC>(nchunks);
    bool ok = true;
    uint32_t k = 0, issued = 0;
    for (uint32_t q = 0; q < nseg; ++q, ++gs) {
        const uint32_t a = gs & 1;
        if (ok && gs >= 2 && !mbar_wait(&S.acc_empty[a], ((gs >> 1) - 1) & 1, kTcWaitNs)) {
            tc_give_up(S, timeouts);
            ok = false;
        }
        tc_fence_after();
        const uint32_t d_tmem = S.tmem + a * 256u;
        const uint32_t kend = q + 1 == nseg ? nchunks : (q + 1) * (kTcSegSlots / KC);
        uint32_t acc = 0;
        for (; k < kend && ok && !S.abort; ++k) {
            const uint32_t g = gk + k, s = g % ST, ph = (g / ST) & 1;
            if (!mbar_wait(&S.full_a[s], ph, kTcWaitNs) || !mbar_wait(&S.full_b[s], ph, kTcWaitNs)) {
                tc_give_up(S, timeouts);
                ok = false;
                break;
            }
            tc_fence_after();
            // descriptors of K step 0; step kk adds its byte offset / 16 to the
            // address field (shared-memory addresses stay below 2^18: no carry)
            const uint32_t ah = smem_u32(st.A_hi(s)), al = smem_u32(st.A_lo(s));
            const uint32_t bh = smem_u32(st.B(s)), bl = bh + J.nb * 1024;  // lo blocks follow the hi blocks
            const uint64_t adh = AMN ? smem_desc(ah, 1024, Cfg::kAMnGroup, 2) : smem_desc(ah, 16, Cfg::kAAtom, Cfg::kALayout);
            const uint64_t adl = AMN ? smem_desc(al, 1024, Cfg::kAMnGroup, 2) : smem_desc(al, 16, Cfg::kAAtom, Cfg::kALayout);
            const uint64_t bdh = smem_desc(bh, 1024, Cfg::kBGroup, 2);
            const uint64_t bdl = smem_desc(bl, 1024, Cfg::kBGroup, 2);
#pragma unroll
            for (int kk = 0; kk < (int)(KC / 16); ++kk) {
                const uint64_t ao = (uint64_t)(AMN ? kk * 2 * Cfg::kAMnGroup / 16 : kk * 32 / 16);
                const uint64_t bo = (uint64_t)(kk * 2 * Cfg::kBGroup / 16);
                mma_f16_ss(d_tmem, adh + ao, bdh + bo, idesc, acc);
                mma_f16_ss(d_tmem, adh + ao, bdl + bo, idesc, 1);
                mma_f16_ss(d_tmem, adl + ao, bdh + bo, idesc, 1);
                acc = 1;
            }
            mma_commit(&S.empty[s]);
            ++issued;
        }
        if (acc)
            mma_commit(&S.acc_full[a]);  // fires once this segment's MMAs have completed
        else
            mbar_arrive(&S.acc_full[a]);
    }
    if (issued) atomicAdd(macs, 3ull * kTcM * (64ull * J.nb) * (uint64_t)KC * issued);
}

// Builders (kTcBuilders threads, index bt), one item: the chunk's entries
// into the MN-major weight operand (pixels contiguous in 128-byte swizzled
// atoms of 64 pixels x 8 slots). The weight pass stores each entry's weights
// already split into 16-bit hi/lo pairs (GroupArgs::pack), so a 2 x 2 group's
// entry is four 32-bit stores: hi and lo of its two horizontal pixel pairs.
// Warp w's eight groups are the tile's pixels 32w .. 32w + 31 (rows 2w and
// 2w + 1), so each warp zeroes exactly its own cells of the chunk before it
// scatters into them and no warp waits for another.
template <class Cfg, class SH>
__device__ __forceinline__ void tc_build(SH &S, const TcJob &J, uint64_t tile, uint32_t nchunks, uint32_t gk, int bt,
                                         unsigned long long *timeouts) {
    using namespace sm100;
    constexpr uint32_t ST = Cfg::kStages, KC = Cfg::kK;
    const TcStage<Cfg> st{tc_smem_base()};
    const TileArgs &T = J.T;
    const GroupArgs &G = J.g;
    const int gq = bt >> 2, sub = bt & 3, lane = bt & 31, w = bt >> 5;
    const uint32_t gxl = gq & 7, gyl = gq >> 3;  // gyl == w
    const uint32_t gxi = (uint32_t)(tile % T.ntx) * (kTileX / 2) + gxl;
    const uint32_t gyi = (uint32_t)(tile / T.ntx) * (kTileY / 2) + gyl;
    const uint64_t grp = (uint64_t)gyi * G.gx + gxi;
    uint64_t e = 0, e_end = 0;
    if (gxi < G.gx && grp < G.ngroups) {
        e = J.off[grp] - G.ebase;
        e_end = e + J.cnt[grp];
    }
    e += sub;
    // This thread takes every 4th entry of its group. Its next eight entries
    // sit in a private ring in shared memory filled by cp.async: the copy of
    // an entry is issued eight entries before it is read, and reading the ring
    // at a per-thread position needs neither register moves nor divergent
    // branches.
    uint32_t *rs = S.ring_slot + bt;  // [kTcRing][kTcBuilders]
    float4 *rw = S.ring_w + bt;
    auto issue = [&](int i) {
        if (e < e_end) {
            cp_async4(rs + i * kTcBuilders, J.e_slot + e);
            cp_async16(rw + i * kTcBuilders, J.e_w + e, true);
        } else {
            rs[i * kTcBuilders] = 0xffffffffu;
        }
        cp_async_commit();
        e += 4;
    };
#pragma unroll
    for (int i = 0; i < kTcRing; ++i) issue(i);
    int head = 0;
    // byte offset of (pixel m, chunk slot col): atom (col / 8, m / 64) of 1 KB,
    // row col % 8 of 128 bytes, 16-byte chunk (m % 64) / 8 XORed with that row
    auto a_off = [](uint32_t m, uint32_t col) -> uint32_t {
        const uint32_t r = col & 7u;
        return ((col >> 3) * 2u + (m >> 6)) * 1024u + r * 128u + ((((m & 63u) >> 3) ^ r) << 4) + ((m & 7u) << 1);
    };
    const uint32_t m0 = 2 * gyl * kTileX + 2 * gxl, m1 = m0 + kTileX;  // the group's pixel pairs (x, x + 1)
    for (uint32_t k = 0; k < nchunks; ++k) {
        const uint32_t g = gk + k, s = g % ST;
        // warp-uniform exits: the zeroing below ends with __syncwarp
        if (__any_sync(0xffffffffu, S.abort)) break;
        const bool free = g < ST || mbar_wait(&S.empty[s], ((g / ST) - 1) & 1, kTcWaitNs);
        if (__any_sync(0xffffffffu, !free)) {
            if (!free) tc_give_up(S, timeouts);
            break;
        }
        uint8_t *ah = st.A_hi(s), *al = st.A_lo(s);
        {
            // this warp's cells: pixels 32w .. 32w + 31 of every slot row, four
            // 16-byte chunks of an atom row (hi and lo)
            constexpr uint32_t kPieces = 4 * KC;
            for (uint32_t p = (uint32_t)lane; p < kPieces; p += 32) {
                const uint32_t r = p >> 2, c = 4u * (uint32_t)(w & 1) + (p & 3u);
                const uint32_t o = ((r >> 3) * 2u + (uint32_t)(w >> 1)) * 1024u + (r & 7u) * 128u + ((c ^ (r & 7u)) << 4);
                *reinterpret_cast<uint4 *>(ah + o) = make_uint4(0, 0, 0, 0);
                *reinterpret_cast<uint4 *>(al + o) = make_uint4(0, 0, 0, 0);
            }
            __syncwarp();
        }
        const uint32_t cs = k * KC, ce = cs + KC;
        for (;;) {
            cp_async_wait<kTcRing - 1>();  // the ring's oldest copy has landed
            const uint32_t slot = rs[head * kTcBuilders];
            if (slot >= ce) break;
            const float4 wq = rw[head * kTcBuilders];  // {hi(p0, p1), lo(p0, p1), hi(p2, p3), lo(p2, p3)}
            const uint32_t col = slot - cs;
            const uint32_t o0 = a_off(m0, col), o1 = a_off(m1, col);
            *reinterpret_cast<uint32_t *>(ah + o0) = __float_as_uint(wq.x);
            *reinterpret_cast<uint32_t *>(al + o0) = __float_as_uint(wq.y);
            *reinterpret_cast<uint32_t *>(ah + o1) = __float_as_uint(wq.z);
            *reinterpret_cast<uint32_t *>(al + o1) = __float_as_uint(wq.w);
            issue(head);
            head = (head + 1) & (kTcRing - 1);
        }
        fence_proxy_async_smem();
        mbar_arrive(&S.full_a[s]);
    }
    cp_async_wait<0>();  // no copy into the ring outlives the item
}

// Whole CTA: one item. `gk` counts the K chunks this CTA has run (all items),
// `itn` its items; both advance identically in every thread.
template <class Cfg>
__device__ __forceinline__ void tc_item(TcShared &S, const TcJob &J, uint64_t tile, uint32_t cblk, uint32_t &gk,
                                        uint32_t itn, unsigned long long *timeouts,
                                        unsigned long long *macs) {
    using namespace sm100;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const TileArgs &T = J.T;
    const uint32_t U = T.U[tile];
    const uint32_t nchunks = (U + Cfg::kK - 1) / Cfg::kK;
    const uint32_t taddr = S.tmem;
    if (warp == 0) {
        tc_produce<Cfg>(S, J, cblk, U, nchunks, gk, T.nr[tile], timeouts);
    } else if (warp == 1) {
        if (lane == 0) {
            tc_mma<Cfg>(S, J, nchunks, gk, taddr, timeouts, macs);
            if (nchunks == 0)
                mbar_arrive(&S.acc_full);
            else
                mma_commit(&S.acc_full);  // also after a timeout: every MMA issued has completed once it fires
        }
    } else {
        const GroupArgs &G = J.g;
        const int bt = tid - 64;
        tc_build<Cfg>(S, J, tile, nchunks, gk, bt, timeouts);
        // -------------------------------------------------------- epilogue
        const uint32_t c_item = cblk * J.nb * 64;  // first channel of the item
        const uint32_t ncols = 64 * J.nb;
        for (uint32_t c = bt; c < ncols; c += kTcBuilders)
            S.inv_scale[c] = c_item + c < J.nchan ? J.inv_scale[c_item + c] : 0.f;
        const bool ok = mbar_wait(&S.acc_full, itn & 1, kTcWaitNs);
        if (!ok) tc_give_up(S, timeouts);
        tc_fence_after();
        // inv_scale staged; the store decision is the same in every builder
        const bool store = !named_barrier_or(2, kTcBuilders, !ok || S.abort);
        const uint32_t q4 = warp & 3;  // TMEM lane quarter this warp may access
        const uint32_t m = q4 * 32 + lane;
        const uint32_t tx0 = (uint32_t)(tile % T.ntx) * kTileX, ty0 = (uint32_t)(tile / T.ntx) * kTileY;
        const uint32_t xx = tx0 + (m & (kTileX - 1));
        const uint32_t yy = ty0 + m / kTileX;
        const bool valid = xx < G.nx && yy < G.ny;
        const uint64_t P = (uint64_t)G.nx * G.ny;
        const uint64_t p = (uint64_t)yy * G.nx + xx;
        const double ws = valid ? J.wsum[p] : 0.0;
        const float inv = (float)(1.0 / ws);
        if (valid && cblk == 0 && J.wout) J.wout[p] = (float)ws;
        // the item's operand buffers are idle now: the staging tile of the cube
        float *stage = (float *)tc_smem_base();
        for (uint32_t cb = 0; cb < 2 * J.nb; ++cb) {
            uint32_t r[32];
            if (nchunks > 0) {
                tmem_ld_32x32b_x32(taddr + ((q4 * 32u) << 16) + cb * 32u, r);
                tmem_wait_ld();
            } else {
#pragma unroll
                for (int i = 0; i < 32; ++i) r[i] = 0u;
            }
            float v[32];
#pragma unroll
            for (int i = 0; i < 32; ++i) v[i] = (__uint_as_float(r[i]) * S.inv_scale[cb * 32 + i]) * inv;
            if (!store) continue;
            if (J.out_map) {
                if (J.ostride) {
                    // box [y][x][channel]: this pixel's 32 values, 16-byte pieces in a
                    // lane-rotated order (fewer bank conflicts)
                    float4 *row = (float4 *)(stage + (size_t)m * ncols + cb * 32);
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const int k = (u + lane) & 7;  // 16-byte bank group of this lane's piece
                        float4 q = make_float4(v[0], v[1], v[2], v[3]);
#pragma unroll
                        for (int kk = 1; kk < 8; ++kk)  // lane-dependent index into registers: selects
                            if (kk == k) q = make_float4(v[4 * kk], v[4 * kk + 1], v[4 * kk + 2], v[4 * kk + 3]);
                        row[k] = q;
                    }
                } else {
                    // box [channel][y][x]
#pragma unroll
                    for (int i = 0; i < 32; ++i) stage[(size_t)(cb * 32 + i) * kTcM + m] = v[i];
                }
            } else if (valid) {
                const uint32_t c0 = c_item + cb * 32;
                if (J.ostride == 0) {
#pragma unroll
                    for (int i = 0; i < 32; ++i)
                        if (c0 + i < J.nchan) J.out[(uint64_t)(c0 + i) * P + p] = v[i];
                } else {
                    float *dst = J.out + p * J.ostride;
#pragma unroll
                    for (int i = 0; i < 32; ++i)
                        if (c0 + i < J.nchan) dst[c0 + i] = v[i];
                }
            }
        }
        if (store && J.out_map) {
            fence_proxy_async_smem();
            named_barrier(2, kTcBuilders);  // the staging tile is complete
            if (bt == 0) {
                if (J.ostride)
                    tma_store_3d(J.out_map, stage, (int)c_item, (int)tx0, (int)ty0);
                else
                    tma_store_3d(J.out_map, stage, (int)tx0, (int)ty0, (int)c_item);
                bulk_commit_group();
                bulk_wait_group_read0();  // the staging tile may be overwritten after this
            }
        }
        tc_fence_before();
    }
    gk += nchunks;
}

// ---------------------------------------------------------------- persistent
// One CTA per SM over a static sequence of items (item it = blockIdx.x +
// i * gridDim.x; a tile's channel blocks are consecutive items, so they run on
// neighbouring SMs together and read the tile's entries from HBM once). Each
// role walks the sequence on its own, coupled to the others only through
// mbarriers: the producer runs ahead into the next item while the MMAs of the
// current one run, and four epilogue warps (6-9) drain item i's accumulator
// while the MMAs of item i+1 fill the other one (two TMEM accumulators of 256
// columns).
constexpr int kTcPersistThreads = 320;

struct TcPShared {
    uint64_t full_a[kTcMaxStages], full_b[kTcMaxStages], empty[kTcMaxStages];
    uint64_t acc_full[2], acc_empty[2];
    uint32_t tmem;
    volatile int abort;
    uint32_t ulo[kTileMaxRings], base[kTileMaxRings + 1];  // the producer's current item
    float inv_scale[2][kTcMaxN];                           // the epilogue's items (by parity)
    float4 ring_w[kTcRing * kTcBuilders];
    uint32_t ring_slot[kTcRing * kTcBuilders];
};

// Epilogue warps (128 threads, index eb), one item from accumulator `a`:
// normalise and store straight from registers (16-byte stores along channels
// for [pixel][channel] cubes; along pixels for [channel][pixel] cubes).
template <uint32_t KC, class SH, bool WSMEM = false>
__device__ __forceinline__ void tc_epilogue_direct(SH &S, const TcJob &J, uint64_t tile, uint32_t cblk,
                                                   uint32_t nchunks, uint32_t il, uint32_t &gse, int eb,
                                                   unsigned long long *timeouts) {
    using namespace sm100;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t ia = il & 1;  // the item's scale buffer
    const TileArgs &T = J.T;
    const GroupArgs &G = J.g;
    const uint32_t c_item = cblk * J.nb * 64;
    const uint32_t ncols = 64 * J.nb;
    for (uint32_t c = eb; c < ncols; c += kTcBuilders)
        S.inv_scale[ia][c] = c_item + c < J.nchan ? J.inv_scale[c_item + c] : 0.f;
    const uint32_t q4 = warp & 3;  // TMEM lane quarter this warp may access
    const uint32_t m = q4 * 32 + lane;
    const uint32_t xx = (uint32_t)(tile % T.ntx) * kTileX + (m & (kTileX - 1));
    const uint32_t yy = (uint32_t)(tile / T.ntx) * kTileY + m / kTileX;
    const bool valid = xx < G.nx && yy < G.ny;
    const uint64_t P = (uint64_t)G.nx * G.ny;
    const uint64_t p = (uint64_t)yy * G.nx + xx;
    const float *sc = S.inv_scale[ia];
    const uint32_t nseg = tc_segments<KC>(nchunks);
    bool store = false;
    float inv = 0.f;
    for (uint32_t q = 0; q < nseg; ++q, ++gse) {
        const uint32_t a = gse & 1;
        const bool ok = mbar_wait(&S.acc_full[a], (gse >> 1) & 1, kTcWaitNs);
        if (!ok) tc_give_up(S, timeouts);
        tc_fence_after();
        if (q == 0) store = !named_barrier_or(3, kTcBuilders, !ok || S.abort);  // scales staged, same decision
        // Segments before the last are added up unnormalised; the last one
        // brings the weight sum (the builders' sums are complete once every
        // chunk has been accumulated) and the sum is normalised.
        const bool last = q + 1 == nseg;
        if (last) {
            double ws = 0.0;
            if constexpr (WSMEM) {
                // the builders' FP64 weight sums of this item (shared memory, by item parity)
                if (!mbar_wait(&S.ws_full[ia], (il >> 1) & 1, kTcWaitNs)) tc_give_up(S, timeouts);
                ws = (S.wsum[ia][0][m] + S.wsum[ia][1][m]) + S.wsum[ia][2][m];
                mbar_arrive(&S.ws_empty[ia]);
            } else {
                ws = valid ? J.wsum[p] : 0.0;
            }
            inv = (float)(1.0 / ws);
            if (store && valid && cblk == 0 && J.wout) J.wout[p] = (float)ws;
        }
        for (uint32_t cb = 0; cb < 2 * J.nb; ++cb) {
            uint32_t r[32];
            if (nchunks > 0) {
                tmem_ld_32x32b_x32(S.tmem + a * 256u + ((q4 * 32u) << 16) + cb * 32u, r);
                tmem_wait_ld();
            } else {
#pragma unroll
                for (int i = 0; i < 32; ++i) r[i] = 0u;
            }
            if (!store || !valid) continue;
            const uint32_t c0 = c_item + cb * 32;
            const float f = last ? inv : 1.f;
            float v[32];
#pragma unroll
            for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]) * sc[cb * 32 + i];
            if (J.ostride == 0) {
#pragma unroll
                for (int i = 0; i < 32; ++i)
                    if (c0 + i < J.nchan) {
                        float *d = J.out + (uint64_t)(c0 + i) * P + p;
                        *d = (q ? *d + v[i] : v[i]) * f;
                    }
            } else {
                float *dst = J.out + p * J.ostride + c0;
                if ((J.ostride & 7) == 0 && c0 + 32 <= J.nchan && (((uintptr_t)J.out) & 31) == 0) {
                    // 32-byte accesses: each store fills whole sectors of the pixel's row
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        float o[8];
#pragma unroll
                        for (int u = 0; u < 8; ++u) o[u] = v[8 * i + u];
                        if (q) {
                            float b[8];
                            ld_global_v8(dst + 8 * i, b);
#pragma unroll
                            for (int u = 0; u < 8; ++u) o[u] += b[u];
                        }
#pragma unroll
                        for (int u = 0; u < 8; ++u) o[u] *= f;
                        st_global_v8(dst + 8 * i, o);
                    }
                } else if ((J.ostride & 3) == 0 && c0 + 32 <= J.nchan && (((uintptr_t)J.out) & 15) == 0) {
                    float4 *d4 = reinterpret_cast<float4 *>(dst);
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        float4 o = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                        if (q) {
                            const float4 b = d4[i];
                            o.x += b.x;
                            o.y += b.y;
                            o.z += b.z;
                            o.w += b.w;
                        }
                        o.x *= f;
                        o.y *= f;
                        o.z *= f;
                        o.w *= f;
                        d4[i] = o;
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 32; ++i)
                        if (c0 + i < J.nchan) dst[i] = (q ? dst[i] + v[i] : v[i]) * f;
                }
            }
        }
        tc_fence_before();
        mbar_arrive(&S.acc_empty[a]);  // the accumulator may be overwritten
    }
}

template <class Cfg>
__device__ __forceinline__ void tc_persist(TcPShared &S, const TcJob &J, uint64_t nitems, uint64_t ntiles,
                                           unsigned long long *timeouts, unsigned long long *macs) {
    using namespace sm100;
    constexpr uint32_t ST = Cfg::kStages, KC = Cfg::kK;
    static_assert(Cfg::kTmemCols <= 256, "two accumulators fit the 512 TMEM columns");
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (uint32_t s = 0; s < ST; ++s) {
            mbar_init(&S.full_a[s], kTcBuilders);
            mbar_init(&S.full_b[s], 1);
            mbar_init(&S.empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&S.acc_full[a], 1);
            mbar_init(&S.acc_empty[a], kTcBuilders);
        }
        S.abort = 0;
        mbar_fence_init();
    }
    if (warp == 1) {
        tmem_alloc(&S.tmem, 512);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    uint32_t gk = 0, il = 0, gs = 0, gse = 0;  // chunks, items, MMA and epilogue segments
    for (uint64_t it = blockIdx.x; it < nitems; it += gridDim.x, ++il) {
        const uint64_t tile = J.T.t0 + tc_walk(it / J.ncb, ntiles, J.T.ntx, J.strip);
        const uint32_t cblk = (uint32_t)(it % J.ncb);
        const uint32_t U = J.T.U[tile];
        const uint32_t nchunks = (U + KC - 1) / KC;
        if (warp == 0) {
            // the item's ring table, loaded by the whole producer warp
            __syncwarp();
            const int nrt = J.T.nr[tile];
            for (int j = lane; j < nrt; j += 32) S.ulo[j] = J.T.ulo[tile * kTileMaxRings + j];
            for (int j = lane; j <= nrt; j += 32) S.base[j] = J.T.base[tile * (kTileMaxRings + 1) + j];
            __syncwarp();
            tc_produce<Cfg>(S, J, cblk, U, nchunks, gk, nrt, timeouts);
        } else if (warp == 1) {
            if (lane == 0) tc_mma_seg<Cfg, true>(S, J, nchunks, gk, gs, timeouts, macs);
        } else if (warp < 6) {
            tc_build<Cfg>(S, J, tile, nchunks, gk, tid - 64, timeouts);
        } else {
            tc_epilogue_direct<KC>(S, J, tile, cblk, nchunks, il, gse, tid - 192, timeouts);
        }
        gk += nchunks;
    }
    // the copies of the last chunks land before the shared memory is given back
    if (tid == 0) {
        for (uint32_t g = gk > ST ? gk - ST : 0; g < gk; ++g) {
            const uint32_t s = g % ST, ph = (g / ST) & 1;
            if (!mbar_wait(&S.full_b[s], ph, kTcWaitNs)) {
                tc_give_up(S, timeouts);
                break;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(S.tmem, 512);
    }
}

// ----------------------------------------------------------- direct weights
// Dense tiles (most staged samples lie within the radius of most of the
// tile's pixels, e.g. beams many pixels wide): the builders evaluate the
// weights of the chunk's slots for their own pixel from the samples'
// geometry, so no entries are written or read and no FP64 weight pass runs
// before. Twelve builder warps (latency hiding for the FP64 chains): thread
// bt owns operand row m = bt % 128 (pixel (m % 16, m / 16) of the tile) and
// the 8-slot pieces p = bt / 128 (mod 3) of each 64-slot chunk. Per chunk
// the first 64 builders load the chunk's sample geometry into shared memory
// (cp.async, one chunk ahead); then, for each slot whose sample lies in its
// pixel's window of the slot's ring (ring_window_mc, the windows the tile pass
// unioned), a builder evaluates the FP64 distance, cutoff and FP32 Gaussian
// (pair_weight_s's arithmetic), accumulates the FP64 weight sum and writes its
// hi/lo pieces of the K-major operand row (16-byte stores). The epilogue adds
// the three partial weight sums of a row from shared memory.
constexpr int kTcGeo = 64;          // slots per chunk of the direct builders
constexpr int kTcGeoBufs = 2;       // geometry buffers: loads run one chunk ahead
constexpr int kTcDRow = 3;          // direct builders per operand row
constexpr int kTcDBuilders = kTcDRow * kTcM;
constexpr int kTcDThreads = 64 + kTcDBuilders + kTcBuilders;  // producer, MMA, builders, epilogue

struct TcDShared {
    uint64_t full_a[kTcMaxStages], full_b[kTcMaxStages], empty[kTcMaxStages];
    uint64_t acc_full[2], acc_empty[2], ws_full[2], ws_empty[2];
    uint32_t tmem;
    volatile int abort;
    uint32_t ulo[kTileMaxRings], base[kTileMaxRings + 1];    // the producer's current item
    uint32_t bulo[kTileMaxRings], bbase[kTileMaxRings + 1];  // the builders' current item
    float inv_scale[2][kTcMaxN];
    double wsum[2][kTcDRow][kTcM];  // by item parity: the builders' partial sums of each row
    double4 g_half[kTcGeoBufs][kTcGeo];  // sample geometry of the chunks in flight
    double g_cb[kTcGeoBufs][kTcGeo], g_w[kTcGeoBufs][kTcGeo];
};

template <class Cfg>
__device__ __forceinline__ void tc_build_weights(TcDShared &S, const TcJob &J, uint64_t tile, uint32_t cblk,
                                                 uint32_t U, uint32_t nchunks, uint32_t gk, uint32_t il, int bt,
                                                 unsigned long long *timeouts) {
    using namespace sm100;
    constexpr uint32_t ST = Cfg::kStages, KC = Cfg::kK;
    static_assert(KC == kTcGeo, "direct builders take 64-slot chunks");
    const TcStage<Cfg> st{tc_smem_base()};
    const TileArgs &T = J.T;
    const GridArgs &a = J.a;
    const uint32_t a2 = il & 1;
    // the builders' copy of the tile's ring table (after every builder is done with the last one)
    named_barrier(4, kTcDBuilders);
    const int nrt = T.nr[tile];
    for (int j = bt; j < nrt; j += kTcDBuilders) S.bulo[j] = T.ulo[tile * kTileMaxRings + j];
    for (int j = bt; j <= nrt; j += kTcDBuilders) S.bbase[j] = T.base[tile * (kTileMaxRings + 1) + j];
    named_barrier(4, kTcDBuilders);
    // this thread's pixel and pieces; its 2x2 group and place there (the tile pass's kept windows)
    const uint32_t m = (uint32_t)bt & (kTcM - 1), qb = (uint32_t)bt / kTcM;
    const uint32_t wgq = (m >> 5) * (kTileX / 2) + ((m & (kTileX - 1)) >> 1);
    const uint32_t wq = (((m >> 4) & 1) << 1) | (m & 1);
    const uint32_t xx = (uint32_t)(tile % T.ntx) * kTileX + (m & (kTileX - 1));
    const uint32_t yy = (uint32_t)(tile / T.ntx) * kTileY + m / kTileX;
    const bool valid = xx < J.g.nx && yy < J.g.ny;
    PixPrep P{};
    if (valid) P = a.prep[(uint64_t)yy * J.g.nx + xx];
    const PixHalf ph = pix_half(P);
    const int r0 = T.r0[tile];
    const uint32_t nrows = J.nrows;
    // kernel-parameter scalars held in registers for the slot loop
    const double hlo = a.hlo, hhi = a.hhi, p0 = a.p0, cb1 = P.cb1;
    const bool series = a.series != 0;
    const float x2scale = a.x2scale;
    const float wscale = J.wscale;
    const uint32_t fmt = J.fmt;
    // geometry of chunk kk into buffer kk % kTcGeoBufs (threads 0..63, one slot each)
    auto load = [&](uint32_t kk) {
        if (bt < kTcGeo && kk < nchunks) {
            const uint32_t slot = kk * KC + bt;
            uint32_t idx = nrows - 1;
            if (slot < U) {
                int lo = 0, hi = nrt;
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (S.bbase[mid] <= slot) lo = mid; else hi = mid;
                }
                idx = min(S.bulo[lo] + (slot - S.bbase[lo]), nrows - 1);
            }
            const uint32_t b = kk % kTcGeoBufs;
            cp_async16(&S.g_half[b][bt], a.half + idx, true);
            cp_async16(reinterpret_cast<uint8_t *>(&S.g_half[b][bt]) + 16,
                       reinterpret_cast<const uint8_t *>(a.half + idx) + 16, true);
            cp_async8(&S.g_cb[b][bt], a.cb2 + idx);
            cp_async8(&S.g_w[b][bt], a.w + idx);
        }
        cp_async_commit();
    };
    load(0);
    // ring cursor: compacted ring c of the current slot, its span index j and this pixel's window there
    int c = -1, j = -1;
    uint32_t cbase = 0, cnext = 0, culo = 0, wlo = 0, whi = 0;
    double wsum = 0.0;
    uint32_t within = 0;
    bool failed = false;
    for (uint32_t k = 0; k < nchunks; ++k) {
        const uint32_t g = gk + k, s = g % ST;
        named_barrier(4, kTcDBuilders);  // every builder is done with chunk k - 1's geometry
        load(k + 1);
        cp_async_wait<1>();  // this thread's copies of chunk k have landed
        bool bad = S.abort;
        if (!bad && g >= ST && !mbar_wait(&S.empty[s], ((g / ST) - 1) & 1, kTcWaitNs)) {
            tc_give_up(S, timeouts);
            bad = true;
        }
        if (named_barrier_or(4, kTcDBuilders, bad)) {  // chunk k's geometry visible; the same exit in every builder
            failed = true;
            break;
        }
        const uint32_t b = k % kTcGeoBufs;
        uint8_t *ah = st.A_hi(s), *al = st.A_lo(s);
        for (uint32_t s8 = qb; s8 < KC / 8; s8 += kTcDRow) {
            // ring runs take multiples of 8 slots: one ring per 8-slot piece
            const uint32_t slot0 = k * KC + s8 * 8;
            if (slot0 < U && (slot0 >= cnext || c < 0)) {
                // next occupied ring (the same in the builders of a piece) and this pixel's window there
                while (c + 1 < nrt && S.bbase[c + 1] <= slot0) ++c;
                cbase = S.bbase[c];
                cnext = S.bbase[c + 1];
                culo = S.bulo[c];
                do {
                    ++j;
                } while (j < kTileMaxSpan && T.ring_idx[tile * kTileMaxSpan + j] != (uint16_t)c);
                wlo = whi = 0;
                const int kr = r0 + j;
                if (T.win && j < kWinSpan) {
                    // the window the tile pass kept for this pixel and ring (lo > hi: none)
                    const uint32_t *w = reinterpret_cast<const uint32_t *>(
                        T.win + ((tile * kWinSpan + (uint64_t)j) * kTileGroups + wgq) * 2);
                    const uint32_t lo = __ldg(w + 2 * wq), hi = __ldg(w + 2 * wq + 1);
                    if (lo <= hi) {
                        wlo = lo;
                        whi = hi;
                    }
                } else if (P.nr > 0 && kr >= P.ur && kr < P.ur + P.nr) {
                    uint32_t lo, hi, rl;
                    if (ring_window_mc(a, a.rings[kr], P, lo, hi, rl)) {
                        wlo = lo;
                        whi = hi;
                    }
                }
            }
            // The piece's pair tests in two halves of 4 slots as straight-line
            // code (independent FP64 chains the scheduler can interleave):
            // haversines, then the weights of the pairs below the threshold
            // band, the same arithmetic as pair_weight_s; pairs inside the band
            // take pair_weight_s itself.
            uint32_t hv[4], lv[4];
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                double hh[4];
                bool inw[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const uint32_t q = s8 * 8 + half * 4 + e;
                    const uint32_t idx = culo + (slot0 + half * 4 + e - cbase);
                    inw[e] = slot0 + half * 4 + e < U && idx >= wlo && idx < whi;
                    const double4 gq = S.g_half[b][q];
                    const double sb = ph.sb * gq.w - ph.cb * gq.z;  // sin((b1 - b2) / 2)
                    const double sl = ph.sl * gq.y - ph.cl * gq.x;  // sin((l1 - l2) / 2)
                    hh[e] = sb * sb + cb1 * S.g_cb[b][q] * (sl * sl);
                }
                float wv[4];
                bool band = false;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const double h = hh[e];
                    // the Gaussian of an accepted pair, as pair_weight_s evaluates it
                    float ex;
                    if (series) {
                        ex = gauss_series_f32(h, x2scale);
                    } else {
                        const double d = 2.0 * asin(sqrt(h)) * kRad2Deg;
                        ex = gauss_f32(d * d * p0);
                    }
                    const bool acc = inw[e] && h < hlo;
                    band |= inw[e] && h >= hlo && h <= hhi;
                    const double wt = acc ? S.g_w[b][s8 * 8 + half * 4 + e] * (double)ex : 0.0;
                    wv[e] = 0.f;
                    if (wt != 0.0) {
                        wsum += wt;
                        ++within;
                        wv[e] = (float)wt;
                    }
                }
                if (band) {
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        if (!(inw[e] && hh[e] >= hlo && hh[e] <= hhi)) continue;
                        const uint32_t q = s8 * 8 + half * 4 + e;
                        const double wt =
                            pair_weight_s<true, false>(a, P, ph, S.g_half[b][q], S.g_cb[b][q], S.g_w[b][q],
                                                       culo + (slot0 + half * 4 + e - cbase));
                        if (wt != 0.0) {
                            wsum += wt;
                            ++within;
                            wv[e] = (float)wt;
                        }
                    }
                }
#pragma unroll
                for (int e = 0; e < 4; e += 2)
                    tc_split2(wv[e] * wscale, wv[e + 1] * wscale, fmt, hv[half * 2 + e / 2], lv[half * 2 + e / 2]);
            }
            const uint32_t o = tc_a_offset<KC>(m, s8 * 8);
            *reinterpret_cast<uint4 *>(ah + o) = make_uint4(hv[0], hv[1], hv[2], hv[3]);
            *reinterpret_cast<uint4 *>(al + o) = make_uint4(lv[0], lv[1], lv[2], lv[3]);
        }
        fence_proxy_async_smem();
        mbar_arrive(&S.full_a[s]);
    }
    cp_async_wait<0>();  // no geometry copy outlives the item
    // the pixel's FP64 weight sum for the epilogue (after it has read the sum two items back)
    if (!failed && il >= 2 && !mbar_wait(&S.ws_empty[a2], ((il >> 1) - 1) & 1, kTcWaitNs)) tc_give_up(S, timeouts);
    S.wsum[a2][qb][m] = valid ? wsum : 0.0;
    mbar_arrive(&S.ws_full[a2]);
    // the accepted pairs (candidates and skipped rings are counted by the tile pass)
    const unsigned long long wsum_pairs = warp_sum_u64(within);
    if (cblk == 0 && (bt & 31) == 0 && wsum_pairs) atomicAdd(&a.stats->pairs_within, wsum_pairs);
}

// Persistent direct-weight kernel body: roles as in tc_persist, the builders
// being tc_build_weights and the epilogue reading their weight sums.
template <class Cfg>
__device__ __forceinline__ void tc_persist_weights(TcDShared &S, const TcJob &J, uint64_t nitems, uint64_t ntiles,
                                                   unsigned long long *timeouts, unsigned long long *macs) {
    using namespace sm100;
    constexpr uint32_t ST = Cfg::kStages, KC = Cfg::kK;
    static_assert(Cfg::kTmemCols <= 256, "two accumulators fit the 512 TMEM columns");
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (uint32_t s = 0; s < ST; ++s) {
            mbar_init(&S.full_a[s], kTcDBuilders);
            mbar_init(&S.full_b[s], 1);
            mbar_init(&S.empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&S.acc_full[a], 1);
            mbar_init(&S.acc_empty[a], kTcBuilders);
            mbar_init(&S.ws_full[a], kTcDBuilders);
            mbar_init(&S.ws_empty[a], kTcBuilders);
        }
        S.abort = 0;
        mbar_fence_init();
    }
    if (warp == 1) {
        tmem_alloc(&S.tmem, 512);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    uint32_t gk = 0, il = 0, gs = 0, gse = 0;  // chunks, items, MMA and epilogue segments
    for (uint64_t it = blockIdx.x; it < nitems; it += gridDim.x, ++il) {
        const uint64_t tile = J.T.t0 + tc_walk(it / J.ncb, ntiles, J.T.ntx, J.strip);
        const uint32_t cblk = (uint32_t)(it % J.ncb);
        const uint32_t U = J.T.U[tile];
        const uint32_t nchunks = (U + KC - 1) / KC;
        if (warp == 0) {
            __syncwarp();
            const int nrt = J.T.nr[tile];
            for (int j = lane; j < nrt; j += 32) S.ulo[j] = J.T.ulo[tile * kTileMaxRings + j];
            for (int j = lane; j <= nrt; j += 32) S.base[j] = J.T.base[tile * (kTileMaxRings + 1) + j];
            __syncwarp();
            tc_produce<Cfg>(S, J, cblk, U, nchunks, gk, nrt, timeouts);
        } else if (warp == 1) {
            if (lane == 0) tc_mma_seg<Cfg, false>(S, J, nchunks, gk, gs, timeouts, macs);
        } else if (tid < 64 + kTcDBuilders) {
            tc_build_weights<Cfg>(S, J, tile, cblk, U, nchunks, gk, il, tid - 64, timeouts);
        } else {
            tc_epilogue_direct<KC, TcDShared, true>(S, J, tile, cblk, nchunks, il, gse, tid - (64 + kTcDBuilders),
                                                timeouts);
        }
        gk += nchunks;
    }
    if (tid == 0) {
        for (uint32_t g = gk > ST ? gk - ST : 0; g < gk; ++g) {
            const uint32_t s = g % ST, ph = (g / ST) & 1;
            if (!mbar_wait(&S.full_b[s], ph, kTcWaitNs)) {
                tc_give_up(S, timeouts);
                break;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(S.tmem, 512);
    }
}

}  // namespace
}  // namespace hcg
