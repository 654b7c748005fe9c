// Batched gridding: many independent jobs (field, target, cube) in one pass.
//
// Every phase is one persistent launch over the work of all jobs: a fixed
// number of CTAs per SM pull work items (pixels, 2x2 groups, tiles, tile x
// channel-slice pairs) from a device-side queue (an atomic head per phase)
// and look the item's job up in a device job table. Launch shapes do not
// depend on the batch, and all per-batch state (job table, queue heads,
// totals, scratch pointers) lives in device memory, so the phases are
// captured once into two CUDA graphs and replayed for every batch:
//   geometry: pixel setup, tile ring tables and candidate counts, offsets,
//             per-job entry totals;
//   sums:     FP64 weights -> entries, channel sums (FP32 or tensor cores),
//             single-channel pixels.
// Between the two the host reads the entry totals, sizes the shared entry
// pool for them and routes to the single-job path (hcg_grid, which runs in
// budget-sized passes) the jobs whose entries do not fit the context's entry
// budget and those whose tiles span more rings than the tile table holds;
// routed jobs are skipped by the second graph.
//
// Items run the same device functions as the single-job launches
// (hcg_kernels.cuh), so each job's cube is identical to hcg_grid's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "hcg_internal.h"
#include "hcg_kernels.cuh"
#include "hcg_tc.cuh"

namespace hcg {
namespace {

struct JobDesc {
    GridArgs a;       // per-job geometry (prep -> batch prep array + pixel base)
    GroupArgs g;      // map shape; off/cnt/cap below are already offset to this job
    TileArgs T;       // tile table slice of this job
    const double *X, *Y;
    uint64_t firstring, usedrings;
    double disc;
    const float *spec;
    uint32_t nchan, cstride, nslices, ostride;  // ostride 0: [channel][pixel]
    float *out, *wout;
    uint32_t *cap, *cnt;
    unsigned long long *off;
    double *wsum;
    PixPrep *prep;
    // first item of this job in each phase's item space
    unsigned long long pix_base, grp_base, tile_base, acc_base, c1_base;
    unsigned long long tc_base;  // in the item space of the job's tensor-core shape
    uint32_t tc_shape;           // kb_tc pipeline shape (kKbNb)
    TcJob tc;  // tensor-core engine arguments (jobs whose field holds split spectra)
    uint32_t skip;  // routed to the single-job path: no entries, no sums here
};

enum { Q_TILE = 0, Q_COUNT, Q_GEOM, Q_ACC, Q_C1, Q_TC, Q_N = Q_TC + kKbShapes };

struct BatchHdr {
    uint32_t njobs;
    unsigned long long tot_pix, tot_grp, tot_tile, tot_acc, tot_c1;
    unsigned long long tot_tc[kKbShapes];  // items of each tensor-core shape
    const uint32_t *tc_list;               // jobs of shape k: tc_list[tc_off[k] .. tc_off[k + 1])
    uint32_t tc_off[kKbShapes + 1];
    unsigned long long head[Q_N];
    unsigned long long entry_cap;      // entries the pool holds
    unsigned long long entries_needed; // total entries of the batch (set by the scan)
    unsigned long long pool_overflow;  // groups skipped for lack of pool space
    uint32_t *e_idx;
    float4 *e_w;
    unsigned long long *off_all;       // [tot_grp + 1]
    uint32_t *cap_all;
    unsigned long long *scan_part;     // [kBatchScanParts + 1]
};

constexpr int kPersistPerSM = 8;

// Job owning item `it` of a phase: last job whose base is <= it.
template <typename F>
__device__ __forceinline__ int find_job(const JobDesc *__restrict__ jobs, uint32_t njobs, unsigned long long it,
                                        F base_of) {
    int lo = 0, hi = (int)njobs;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (base_of(jobs[mid]) <= it) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(256) kb_prep(const BatchHdr *__restrict__ H, const JobDesc *__restrict__ jobs,
                                               DevStats *stats) {
    for (unsigned long long it = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; it < H->tot_pix;
         it += (unsigned long long)gridDim.x * blockDim.x) {
        int j = find_job(jobs, H->njobs, it, [](const JobDesc &d) { return d.pix_base; });
        const JobDesc &J = jobs[j];
        prep_item(J.a.h, J.firstring, J.usedrings, J.disc, J.X, J.Y, J.prep, stats, it - J.pix_base);
    }
}

__device__ __forceinline__ unsigned long long block_fetch(BatchHdr *H, int q) {
    __shared__ unsigned long long s_item;
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(&H->head[q], 1ULL);
    __syncthreads();
    return s_item;
}

__device__ __forceinline__ unsigned long long warp_fetch(BatchHdr *H, int q) {
    unsigned long long v = 0;
    if ((threadIdx.x & 31) == 0) v = atomicAdd(&H->head[q], 1ULL);
    return __shfl_sync(0xffffffffu, v, 0);
}

__global__ void __launch_bounds__(256) kb_tile_rings(BatchHdr *H, const JobDesc *__restrict__ jobs) {
    for (;;) {
        unsigned long long it = block_fetch(H, Q_TILE);
        if (it >= H->tot_tile) return;
        int j = find_job(jobs, H->njobs, it, [](const JobDesc &d) { return d.tile_base; });
        const JobDesc &J = jobs[j];
        tile_rings_item(J.a, J.g, J.T, it - J.tile_base);
    }
}

template <bool COUNT>
__global__ void __launch_bounds__(256, 3) kb_group(BatchHdr *H, const JobDesc *__restrict__ jobs) {
    __shared__ PixPrep s_prep[8][4];
    __shared__ PixHalf s_half[8][4];
    const int warp = threadIdx.x >> 5;
    for (;;) {
        unsigned long long it = warp_fetch(H, COUNT ? Q_COUNT : Q_GEOM);
        if (it >= H->tot_grp) return;
        int j = find_job(jobs, H->njobs, it, [](const JobDesc &d) { return d.grp_base; });
        const JobDesc &J = jobs[j];
        uint64_t grp = it - J.grp_base;
        if (!COUNT) {
            if (J.skip) continue;
            // the pool must hold this group's entries; otherwise skip and report
            // (no entries recorded: the pass is replayed once the pool has grown)
            unsigned long long end = J.off[grp] + J.cap[grp];
            if (end > H->entry_cap) {
                if ((threadIdx.x & 31) == 0) {
                    J.cnt[grp] = 0;
                    atomicAdd(&H->pool_overflow, 1ULL);
                }
                continue;
            }
        }
        group_item<COUNT>(J.a, J.g, J.cap, J.off, H->e_idx, H->e_w, J.cnt, J.wsum, J.T, grp, s_prep[warp],
                          s_half[warp]);
    }
}

// Exclusive scan of all jobs' group capacities: three fixed-shape passes
// over kBatchScanParts parts (graph-captured; the count is read on the device).
constexpr uint32_t kBatchScanParts = 296;
__global__ void __launch_bounds__(kScanThreads) kb_scan_sums(BatchHdr *H) {
    scan_sums_item(H->cap_all, H->tot_grp, kBatchScanParts, H->scan_part, blockIdx.x);
}
__global__ void __launch_bounds__(kScanThreads) kb_scan_psum(BatchHdr *H) {
    scan_psum_item(H->scan_part, kBatchScanParts);
    if (threadIdx.x == 0) H->entries_needed = H->scan_part[kBatchScanParts];
}
__global__ void __launch_bounds__(kScanThreads) kb_scan_apply(BatchHdr *H) {
    scan_apply_item(H->cap_all, H->tot_grp, kBatchScanParts, H->scan_part, H->off_all, blockIdx.x);
}

// Entries of each job: the difference of the offsets at its group range ends.
__global__ void __launch_bounds__(256) kb_job_entries(const BatchHdr *__restrict__ H,
                                                      const JobDesc *__restrict__ jobs,
                                                      unsigned long long *__restrict__ jent) {
    for (uint32_t j = threadIdx.x; j < H->njobs; j += blockDim.x)
        jent[j] = H->off_all[jobs[j].grp_base + jobs[j].g.ngroups] - H->off_all[jobs[j].grp_base];
}

__global__ void __launch_bounds__(kBatchTileThreads) kb_accum(BatchHdr *H, const JobDesc *__restrict__ jobs,
                                                             unsigned long long *timeouts) {
    if (H->pool_overflow) return;  // entries incomplete: this pass is replayed after the pool grows
    for (;;) {
        unsigned long long it = block_fetch(H, Q_ACC);
        if (it >= H->tot_acc) return;
        int j = find_job(jobs, H->njobs, it, [](const JobDesc &d) { return d.acc_base; });
        const JobDesc &J = jobs[j];
        if (J.skip) continue;
        unsigned long long local = it - J.acc_base;
        uint64_t tile = local / J.nslices;
        uint32_t c0 = (uint32_t)(local % J.nslices) * kBatchSlice;
        tile_accum_item<kBatchAccumBufs, kBatchAccumRows, kBatchAccumCpt, kBatchSlice>(
            J.g, J.T, J.off, J.cnt, H->e_idx, H->e_w, J.wsum, J.spec, J.nchan, J.cstride, J.out, J.ostride, J.wout,
            tile, c0, timeouts);
    }
}

// Tensor-core channel sums: one CTA per SM takes (job, channel block, tile)
// items from the queue of its pipeline shape SH (the jobs whose channel
// class the context assigns that shape); barrier phases and TMEM persist
// across items. One launch per shape, in sequence; a shape without items
// returns at once.
template <int SH>
struct KbShape;
template <> struct KbShape<0> { using Cfg = TcCfgN4K32; };
template <> struct KbShape<1> { using Cfg = TcCfgN4S2; };
template <> struct KbShape<2> { using Cfg = TcCfgN2S3; };
template <> struct KbShape<3> { using Cfg = TcCfgN1S4; };
static_assert(kKbShapes == 4, "one KbShape per batch tensor-core shape");

template <int SH>
__global__ void __launch_bounds__(kTcThreads, 1)
    kb_tc(BatchHdr *H, const JobDesc *__restrict__ jobs, unsigned long long *timeouts,
          unsigned long long *macs) {
    using KbTcCfg = typename KbShape<SH>::Cfg;
    static_assert(KbTcCfg::kNb == kKbNb[SH], "shape table and configurations agree");
    __shared__ TcShared S;
    // entries incomplete (this pass is replayed after the pool grows), or no items of this shape
    if (H->pool_overflow || H->tot_tc[SH] == 0) return;
    tc_setup<KbTcCfg>(S);
    uint32_t gk = 0, itn = 0;
    const uint32_t *list = H->tc_list + H->tc_off[SH];
    const int nlist = (int)(H->tc_off[SH + 1] - H->tc_off[SH]);
    for (;;) {
        if (threadIdx.x == 0) S.item = S.abort ? ~0ULL : atomicAdd(&H->head[Q_TC + SH], 1ULL);
        __syncthreads();
        const unsigned long long it = S.item;
        if (it >= H->tot_tc[SH]) break;
        int lo = 0, hi = nlist;  // the shape's last job whose base is <= it
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (jobs[list[mid]].tc_base <= it) lo = mid; else hi = mid;
        }
        const int j = (int)list[lo];
        if (jobs[j].skip) {
            __syncthreads();  // every thread has read S.item
            continue;
        }
        const TcJob &J = jobs[j].tc;
        const unsigned long long local = it - jobs[j].tc_base;
        const uint64_t ntiles = (uint64_t)J.T.ntx * J.T.nty;
        const uint64_t tile = local % ntiles;  // tiles fastest: neighbours share staged samples in L2
        tc_load_rings(S, J.T, tile);
        __syncthreads();
        tc_item<KbTcCfg>(S, J, tile, (uint32_t)(local / ntiles), gk, itn, timeouts, macs);
        ++itn;
        __syncthreads();  // every role is done with the item's ring table and accumulator
    }
    tc_teardown<KbTcCfg>(S, gk, timeouts);
}

__global__ void __launch_bounds__(256) kb_1chan(BatchHdr *H, const JobDesc *__restrict__ jobs) {
    for (;;) {
        unsigned long long it = warp_fetch(H, Q_C1);
        if (it >= H->tot_c1) return;
        int j = find_job(jobs, H->njobs, it, [](const JobDesc &d) { return d.c1_base; });
        const JobDesc &J = jobs[j];
        grid1_item<false>(J.a, J.spec, J.cstride, J.out, J.wout, it - J.c1_base);  // GAUSS1D jobs only
    }
}

}  // namespace

static bool batch_uses_tc(const hcg_field *f) { return auto_engine(f) != HCG_ENGINE_FP32; }

// HCG_BATCH_TRACE=1 prints one line per batch pass on stderr (sizes, entry
// pool, fallbacks, device time).
bool batch_trace() {
    static const bool on = [] {
        const char *v = getenv("HCG_BATCH_TRACE");
        return v && *v && *v != '0';
    }();
    return on;
}

// Batch state kept by a context: device header + job table, scratch and the
// captured graph.
struct BatchState {
    BatchHdr *d_hdr = nullptr;
    BatchHdr *h_hdr = nullptr;  // pinned
    JobDesc *d_jobs = nullptr;
    JobDesc *h_jobs = nullptr;  // pinned
    uint32_t job_cap = 0;
    cudaGraphExec_t exec_geom = nullptr, exec_sums = nullptr;
    int nsm = 0;
    void *scratch[11] = {};
    size_t scratch_size[11] = {};
    CUtensorMap *d_maps = nullptr, *h_maps = nullptr;  // two per job: spectra (hi and lo halves), cube
    unsigned long long *d_jovf = nullptr, *h_jovf = nullptr;  // per job: tiles beyond the ring table
    unsigned long long *d_jent = nullptr, *h_jent = nullptr;  // per job: entries
    unsigned long long *d_jusum = nullptr, *h_jusum = nullptr;  // per job: staged slots of its tiles (sum, largest)
    uint32_t *d_tclist = nullptr, *h_tclist = nullptr;          // tensor-core jobs grouped by shape
    uint32_t map_cap = 0;
    unsigned long long entry_cap = 0;
    cudaMemPool_t pool = nullptr;  // the context's memory pool
};

static cudaError_t grow(BatchState &B, int slot, size_t bytes, cudaStream_t s, void **out) {
    if (B.scratch_size[slot] < bytes) {
        if (B.scratch[slot]) cudaFreeAsync(B.scratch[slot], s);
        size_t want = bytes + bytes / 4 + 256;
        cudaError_t e = dalloc(&B.scratch[slot], want, s, B.pool);
        if (e != cudaSuccess) {
            B.scratch[slot] = nullptr;
            B.scratch_size[slot] = 0;
            return e;
        }
        B.scratch_size[slot] = want;
    }
    *out = B.scratch[slot];
    return cudaSuccess;
}

static cudaError_t capture(hcg_context *ctx, BatchState &B) {
    cudaStream_t s = ctx->stream;
    const int smem = kBatchAccumBufs * kBatchAccumRows * kBatchSlice * (int)sizeof(float);
    cudaError_t e = cudaFuncSetAttribute(kb_accum, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    if ((e = tc_set_smem((const void *)kb_tc<0>, KbShape<0>::Cfg::kSmem)) != cudaSuccess ||
        (e = tc_set_smem((const void *)kb_tc<1>, KbShape<1>::Cfg::kSmem)) != cudaSuccess ||
        (e = tc_set_smem((const void *)kb_tc<2>, KbShape<2>::Cfg::kSmem)) != cudaSuccess ||
        (e = tc_set_smem((const void *)kb_tc<3>, KbShape<3>::Cfg::kSmem)) != cudaSuccess)
        return e;
    const int n = B.nsm;
    for (int part = 0; part < 2; ++part) {
        cudaGraph_t graph;
        if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return e;
        cudaMemsetAsync(&B.d_hdr->head[0], 0, sizeof(B.d_hdr->head), s);
        cudaMemsetAsync(&B.d_hdr->pool_overflow, 0, sizeof(unsigned long long), s);
        if (part == 0) {
            kb_prep<<<n * kPersistPerSM, 256, 0, s>>>(B.d_hdr, B.d_jobs, ctx->d_stats);
            kb_tile_rings<<<n * 4, 256, 0, s>>>(B.d_hdr, B.d_jobs);
            kb_group<true><<<n * kPersistPerSM, 256, 0, s>>>(B.d_hdr, B.d_jobs);
            kb_scan_sums<<<kBatchScanParts, kScanThreads, 0, s>>>(B.d_hdr);
            kb_scan_psum<<<1, kScanThreads, 0, s>>>(B.d_hdr);
            kb_scan_apply<<<kBatchScanParts, kScanThreads, 0, s>>>(B.d_hdr);
            kb_job_entries<<<1, 256, 0, s>>>(B.d_hdr, B.d_jobs, B.d_jent);
        } else {
            kb_group<false><<<n * kPersistPerSM, 256, 0, s>>>(B.d_hdr, B.d_jobs);
            kb_accum<<<n, kBatchTileThreads, smem, s>>>(B.d_hdr, B.d_jobs, &ctx->d_stats->timeouts);
            unsigned long long *to = &ctx->d_stats->timeouts, *macs = &ctx->d_stats->tc_macs;
            kb_tc<0><<<n, kTcThreads, KbShape<0>::Cfg::kSmem, s>>>(B.d_hdr, B.d_jobs, to, macs);
            kb_tc<1><<<n, kTcThreads, KbShape<1>::Cfg::kSmem, s>>>(B.d_hdr, B.d_jobs, to, macs);
            kb_tc<2><<<n, kTcThreads, KbShape<2>::Cfg::kSmem, s>>>(B.d_hdr, B.d_jobs, to, macs);
            kb_tc<3><<<n, kTcThreads, KbShape<3>::Cfg::kSmem, s>>>(B.d_hdr, B.d_jobs, to, macs);
            kb_1chan<<<n * kPersistPerSM, 256, 0, s>>>(B.d_hdr, B.d_jobs);
        }
        cudaError_t ce = cudaStreamEndCapture(s, &graph);
        if (ce != cudaSuccess) return ce;
        e = cudaGraphInstantiate(part == 0 ? &B.exec_geom : &B.exec_sums, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t batch_release(hcg_context *ctx) {
    BatchState *B = (BatchState *)ctx->batch;
    if (!B) return cudaSuccess;
    if (B->exec_geom) cudaGraphExecDestroy(B->exec_geom);
    if (B->exec_sums) cudaGraphExecDestroy(B->exec_sums);
    for (auto &p : B->scratch)
        if (p) cudaFreeAsync(p, ctx->stream);
    if (B->d_hdr) cudaFreeAsync(B->d_hdr, ctx->stream);
    if (B->d_jobs) cudaFreeAsync(B->d_jobs, ctx->stream);
    if (B->d_maps) cudaFreeAsync(B->d_maps, ctx->stream);
    if (B->h_maps) cudaFreeHost(B->h_maps);
    if (B->d_jovf) cudaFreeAsync(B->d_jovf, ctx->stream);
    if (B->h_jovf) cudaFreeHost(B->h_jovf);
    if (B->d_jent) cudaFreeAsync(B->d_jent, ctx->stream);
    if (B->h_jent) cudaFreeHost(B->h_jent);
    if (B->d_jusum) cudaFreeAsync(B->d_jusum, ctx->stream);
    if (B->h_jusum) cudaFreeHost(B->h_jusum);
    if (B->d_tclist) cudaFreeAsync(B->d_tclist, ctx->stream);
    if (B->h_tclist) cudaFreeHost(B->h_tclist);
    if (B->h_hdr) cudaFreeHost(B->h_hdr);
    if (B->h_jobs) cudaFreeHost(B->h_jobs);
    delete B;
    ctx->batch = nullptr;
    return cudaSuccess;
}

// Grid `njobs` jobs with device output buffers in one graph replay.
// `fallback[j]` is set for jobs that must be re-run through hcg_grid.
cudaError_t grid_batch(hcg_context *ctx, uint32_t njobs, const hcg_job *jobs, std::vector<char> &fallback,
                       std::string &why) {
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    if (!ctx->batch) {
        BatchState *B = new BatchState();
        B->pool = ctx->pool;
        cudaDeviceGetAttribute(&B->nsm, cudaDevAttrMultiProcessorCount, ctx->device);
        if ((e = dalloc(&B->d_hdr, sizeof(BatchHdr), s, ctx->pool)) != cudaSuccess ||
            (e = cudaMallocHost(&B->h_hdr, sizeof(BatchHdr))) != cudaSuccess) {
            if (B->d_hdr) cudaFreeAsync(B->d_hdr, s);
            if (B->h_hdr) cudaFreeHost(B->h_hdr);
            delete B;
            return e;
        }
        ctx->batch = B;
    }
    BatchState &B = *(BatchState *)ctx->batch;
    if (njobs > B.job_cap) {
        if (B.d_jobs) cudaFreeAsync(B.d_jobs, s);
        if (B.h_jobs) cudaFreeHost(B.h_jobs);
        if (B.d_jovf) cudaFreeAsync(B.d_jovf, s);
        if (B.h_jovf) cudaFreeHost(B.h_jovf);
        if (B.d_jent) cudaFreeAsync(B.d_jent, s);
        if (B.h_jent) cudaFreeHost(B.h_jent);
        if (B.d_jusum) cudaFreeAsync(B.d_jusum, s);
        if (B.h_jusum) cudaFreeHost(B.h_jusum);
        if (B.d_tclist) cudaFreeAsync(B.d_tclist, s);
        if (B.h_tclist) cudaFreeHost(B.h_tclist);
        // the captured graphs hold the job table's and the entry totals'
        // addresses as launch arguments: capture again with the new ones (no
        // replay is in flight: every batch ends with a stream synchronize)
        if (B.exec_geom) cudaGraphExecDestroy(B.exec_geom);
        if (B.exec_sums) cudaGraphExecDestroy(B.exec_sums);
        B.exec_geom = B.exec_sums = nullptr;
        B.job_cap = std::max<uint32_t>(njobs, 64);
        if ((e = dalloc(&B.d_jobs, B.job_cap * sizeof(JobDesc), s, ctx->pool)) != cudaSuccess) return e;
        if ((e = cudaMallocHost(&B.h_jobs, B.job_cap * sizeof(JobDesc))) != cudaSuccess) return e;
        if ((e = dalloc(&B.d_jovf, B.job_cap * sizeof(unsigned long long), s, ctx->pool)) != cudaSuccess) return e;
        if ((e = cudaMallocHost(&B.h_jovf, B.job_cap * sizeof(unsigned long long))) != cudaSuccess) return e;
        if ((e = dalloc(&B.d_jent, B.job_cap * sizeof(unsigned long long), s, ctx->pool)) != cudaSuccess) return e;
        if ((e = cudaMallocHost(&B.h_jent, B.job_cap * sizeof(unsigned long long))) != cudaSuccess) return e;
        if ((e = dalloc(&B.d_jusum, 2 * B.job_cap * sizeof(unsigned long long), s, ctx->pool)) != cudaSuccess) return e;
        if ((e = cudaMallocHost(&B.h_jusum, 2 * B.job_cap * sizeof(unsigned long long))) != cudaSuccess) return e;
        if ((e = dalloc(&B.d_tclist, B.job_cap * sizeof(uint32_t), s, ctx->pool)) != cudaSuccess) return e;
        if ((e = cudaMallocHost(&B.h_tclist, B.job_cap * sizeof(uint32_t))) != cudaSuccess) return e;
    }
    if (2 * njobs > B.map_cap) {
        if (B.d_maps) cudaFreeAsync(B.d_maps, s);
        if (B.h_maps) cudaFreeHost(B.h_maps);
        B.map_cap = std::max<uint32_t>(2 * njobs, 128);
        if ((e = dalloc(&B.d_maps, B.map_cap * sizeof(CUtensorMap), s, ctx->pool)) != cudaSuccess) return e;
        if ((e = cudaMallocHost(&B.h_maps, B.map_cap * sizeof(CUtensorMap))) != cudaSuccess) return e;
    }
    // item spaces and scratch sizes
    unsigned long long pix = 0, grp = 0, tile = 0, acc = 0, c1 = 0, tcn = 0;
    unsigned long long tcs[kKbShapes] = {};  // tensor-core items per shape
    std::vector<JobDesc> J(njobs);
    for (uint32_t i = 0; i < njobs; ++i) {
        const hcg_field *f = jobs[i].field;
        const hcg_target *t = jobs[i].target;
        JobDesc &d = J[i];
        memset(&d, 0, sizeof d);
        uint64_t P = (uint64_t)t->nx * t->ny;
        d.g.nx = t->nx;
        d.g.ny = t->ny;
        d.g.gx = (t->nx + 1) / 2;
        d.g.ngroups = (f->nchan > 1) ? (uint64_t)d.g.gx * ((t->ny + 1) / 2) : 0;
        d.g.g0 = 0;
        d.g.g1 = d.g.ngroups;
        d.g.ebase = 0;
        d.T.ntx = (t->nx + kTileX - 1) / kTileX;
        d.T.nty = (t->ny + kTileY - 1) / kTileY;
        uint64_t ntiles = (f->nchan > 1) ? (uint64_t)d.T.ntx * d.T.nty : 0;
        const bool tc = batch_uses_tc(f);
        d.nslices = tc ? 0 : (f->cstride + kBatchSlice - 1) / kBatchSlice;
        if (tc) {
            d.T.pad = 8;  // ring runs as boxes of 8 samples
            d.tc_shape = (uint32_t)kb_shape_of(ctx, f);
            if (!tc_prepare_job(f, (int)kKbNb[d.tc_shape], &B.h_maps[2 * i], d.tc)) {
                why = "cuTensorMapEncodeTiled";
                return cudaErrorInvalidValue;
            }
            d.g.pack = 1;  // the tensor-core builders take packed hi/lo weights
            d.g.fmt = d.tc.fmt;
            d.g.wscale = d.tc.wscale;
        }
        d.pix_base = pix;
        d.grp_base = grp;
        d.tile_base = tile;
        d.acc_base = acc;
        d.c1_base = c1;
        d.tc_base = tcs[d.tc_shape];
        pix += P;
        grp += d.g.ngroups;
        tile += ntiles;
        acc += ntiles * d.nslices;
        if (tc) {
            tcs[d.tc_shape] += ntiles * d.tc.ncb;
            tcn += ntiles * d.tc.ncb;
        }
        if (f->nchan == 1) c1 += P;
    }
    // tensor-core jobs grouped by shape, in job order within a shape (their
    // bases rise along the list)
    uint32_t tc_off[kKbShapes + 1] = {};
    {
        uint32_t k = 0;
        for (int sh = 0; sh < kKbShapes; ++sh) {
            tc_off[sh] = k;
            for (uint32_t i = 0; i < njobs; ++i)
                if (J[i].tc.nb && J[i].tc_shape == (uint32_t)sh) B.h_tclist[k++] = i;
        }
        tc_off[kKbShapes] = k;
    }
    void *p_prep, *p_wsum, *p_cap, *p_cnt, *p_off, *p_tiles, *p_ridx, *p_scan;
    const size_t tile_words = 3 + kTileMaxRings + kTileMaxRings + 1;  // r0, nr, U, ulo[], base[]
    if ((e = grow(B, 0, (pix + 1) * sizeof(PixPrep), s, &p_prep)) != cudaSuccess ||
        (e = grow(B, 1, (pix + 1) * sizeof(double), s, &p_wsum)) != cudaSuccess ||
        (e = grow(B, 2, (grp + 1) * sizeof(uint32_t), s, &p_cap)) != cudaSuccess ||
        (e = grow(B, 3, (grp + 1) * sizeof(uint32_t), s, &p_cnt)) != cudaSuccess ||
        (e = grow(B, 4, (grp + 2) * sizeof(unsigned long long), s, &p_off)) != cudaSuccess ||
        (e = grow(B, 5, (tile + 1) * tile_words * sizeof(uint32_t), s, &p_tiles)) != cudaSuccess ||
        (e = grow(B, 8, (tile + 1) * kTileMaxSpan * sizeof(uint16_t), s, &p_ridx)) != cudaSuccess ||
        (e = grow(B, 9, (kBatchScanParts + 1) * sizeof(unsigned long long), s, &p_scan)) != cudaSuccess)
        return e;
    // Per-group windows kept by the tile pass for the weight pass: up to
    // 4 GiB of them, given to the jobs in order while they fit.
    const size_t win_tile = (size_t)kWinSpan * kTileGroups * 2 * sizeof(uint4);
    const size_t wbytes = std::min<size_t>((size_t)(tile + 1) * win_tile, 4ull << 30);
    void *p_win = nullptr;
    if (grow(B, 10, wbytes, s, &p_win) != cudaSuccess) {
        cudaGetLastError();
        p_win = nullptr;
    }
    const unsigned long long win_tiles = p_win ? wbytes / win_tile : 0;
    if (B.entry_cap == 0) B.entry_cap = 1ULL << 20;
    void *p_eidx = nullptr, *p_ew = nullptr;
    auto pool = [&](unsigned long long cap) -> cudaError_t {
        cudaError_t pe;
        if ((pe = grow(B, 6, (cap + 1) * sizeof(uint32_t), s, &p_eidx)) != cudaSuccess ||
            (pe = grow(B, 7, (cap + 1) * sizeof(float4), s, &p_ew)) != cudaSuccess) {
            why = "entry pool of " + std::to_string(cap) + " entries";
            return pe;
        }
        B.entry_cap = cap;
        return cudaSuccess;
    };
    if ((e = pool(B.entry_cap)) != cudaSuccess) return e;
    int *t_r0 = (int *)p_tiles;
    int *t_nr = t_r0 + (tile + 1);
    uint32_t *t_U = (uint32_t *)(t_nr + (tile + 1));
    uint32_t *t_ulo = t_U + (tile + 1);
    uint32_t *t_base = t_ulo + (tile + 1) * kTileMaxRings;
    // job table and header, with the current entry pool
    auto fill = [&]() {
        for (uint32_t i = 0; i < njobs; ++i) {
            const hcg_field *f = jobs[i].field;
            const hcg_target *t = jobs[i].target;
            JobDesc &d = J[i];
            d.prep = (PixPrep *)p_prep + d.pix_base;
            d.wsum = (double *)p_wsum + d.pix_base;
            d.cap = (uint32_t *)p_cap + d.grp_base;
            d.cnt = (uint32_t *)p_cnt + d.grp_base;
            d.off = (unsigned long long *)p_off + d.grp_base;
            d.a = grid_args(f, d.prep, ctx->d_stats);
            d.T.t0 = 0;
            d.T.r0 = t_r0 + d.tile_base;
            d.T.nr = t_nr + d.tile_base;
            d.T.U = t_U + d.tile_base;
            d.T.ulo = t_ulo + d.tile_base * kTileMaxRings;
            d.T.base = t_base + d.tile_base * (kTileMaxRings + 1);
            d.T.ring_idx = (uint16_t *)p_ridx + d.tile_base * kTileMaxSpan;
            d.T.cap = d.cap;  // the tile pass counts each group's candidates
            const uint64_t ntiles = (f->nchan > 1) ? (uint64_t)d.T.ntx * d.T.nty : 0;
            d.T.win = (p_win && d.tile_base + ntiles <= win_tiles)
                          ? (uint4 *)p_win + d.tile_base * kWinSpan * kTileGroups * 2
                          : nullptr;
            d.T.overflow = B.d_jovf + i;
            d.T.ustat = B.d_jusum + 2 * i;
            d.X = t->d_x;
            d.Y = t->d_y;
            d.firstring = f->firstring;
            d.usedrings = f->usedrings;
            d.disc = f->disc_size;
            d.spec = f->d_spec;
            d.nchan = f->nchan;
            d.cstride = f->cstride;
            d.ostride = jobs[i].layout == HCG_LAYOUT_CHANNEL_MAJOR ? 0 : f->nchan;
            d.out = jobs[i].cube;
            d.wout = jobs[i].weights;
            if (d.tc.nb) {
                TcJob &c = d.tc;
                c.map = B.d_maps + 2 * i;
                c.out_map = tc_out_map(&B.h_maps[2 * i + 1], d.out, d.ostride, d.g.nx, d.g.ny, c.nchan, c.nb)
                                ? B.d_maps + 2 * i + 1
                                : nullptr;
                c.g = d.g;
                c.T = d.T;
                c.off = d.off;
                c.cnt = d.cnt;
                c.e_slot = (const uint32_t *)p_eidx;
                c.e_w = (const float4 *)p_ew;
                c.wsum = d.wsum;
                c.out = d.out;
                c.ostride = d.ostride;
                c.wout = d.wout;
            }
        }
        memcpy(B.h_jobs, J.data(), njobs * sizeof(JobDesc));
        BatchHdr &h = *B.h_hdr;
        memset(&h, 0, sizeof h);
        h.njobs = njobs;
        h.tot_pix = pix;
        h.tot_grp = grp;
        h.tot_tile = tile;
        h.tot_acc = acc;
        h.tot_c1 = c1;
        for (int sh = 0; sh < kKbShapes; ++sh) h.tot_tc[sh] = tcs[sh];
        h.tc_list = B.d_tclist;
        for (int sh = 0; sh <= kKbShapes; ++sh) h.tc_off[sh] = tc_off[sh];
        h.entry_cap = B.entry_cap;
        h.e_idx = (uint32_t *)p_eidx;
        h.e_w = (float4 *)p_ew;
        h.off_all = (unsigned long long *)p_off;
        h.cap_all = (uint32_t *)p_cap;
        h.scan_part = (unsigned long long *)p_scan;
    };
    fill();
    if ((e = cudaMemcpyAsync(B.d_jobs, B.h_jobs, njobs * sizeof(JobDesc), cudaMemcpyHostToDevice, s)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(B.d_hdr, B.h_hdr, sizeof(BatchHdr), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(&ctx->d_stats->overflow, 0, 3 * sizeof(unsigned long long), s)) != cudaSuccess ||
        (e = cudaMemsetAsync(B.d_jovf, 0, njobs * sizeof(unsigned long long), s)) != cudaSuccess ||
        (e = cudaMemsetAsync(B.d_jusum, 0, 2 * njobs * sizeof(unsigned long long), s)) != cudaSuccess)
        return e;
    if (tcn && ((e = cudaMemcpyAsync(B.d_maps, B.h_maps, 2 * njobs * sizeof(CUtensorMap), cudaMemcpyHostToDevice,
                                     s)) != cudaSuccess ||
                (e = cudaMemcpyAsync(B.d_tclist, B.h_tclist, tc_off[kKbShapes] * sizeof(uint32_t),
                                     cudaMemcpyHostToDevice, s)) != cudaSuccess))
        return e;
    if (!B.exec_geom && (e = capture(ctx, B)) != cudaSuccess) return e;
    // geometry graph, then the entry totals of every job
    cudaEventRecord(ctx->ev0, s);
    if ((e = cudaGraphLaunch(B.exec_geom, s)) != cudaSuccess) return e;
    cudaEventRecord(ctx->evp[0], s);
    if ((e = cudaMemcpyAsync(B.h_jent, B.d_jent, njobs * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(B.h_jovf, B.d_jovf, njobs * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(B.h_jusum, B.d_jusum, 2 * njobs * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             s)) != cudaSuccess)
        return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    // Routing: jobs whose tiles overflowed the ring table, tensor-core jobs
    // with dense tiles (the single-job kernel evaluates their weights itself)
    // or with tiles longer than one accumulation segment (the single-job
    // kernels accumulate in segments), then the jobs with the most entries
    // until the rest fit the context's entry budget.
    fallback.assign(njobs, 0);
    unsigned long long total = 0;
    uint32_t nrouted = 0;
    for (uint32_t i = 0; i < njobs; ++i) {
        if ((B.h_jovf[i] && jobs[i].field->nchan > 1) ||
            (J[i].tc.nb &&
             (tc_use_weights(ctx, jobs[i].field, B.h_jusum[2 * i], B.h_jent[i], (unsigned long long)J[i].T.ntx * J[i].T.nty) ||
              B.h_jusum[2 * i + 1] > kTcOneSegmentSlots))) {
            fallback[i] = 1;
            ++nrouted;
        } else {
            total += B.h_jent[i];
        }
    }
    const unsigned long long max_pool = ctx->entry_budget / (sizeof(uint32_t) + sizeof(float4));
    auto with_slack = [](unsigned long long x) { return x + (x >> 4) + 1024; };
    if (with_slack(total) > max_pool) {
        std::vector<uint32_t> order;
        for (uint32_t i = 0; i < njobs; ++i)
            if (!fallback[i]) order.push_back(i);
        std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return B.h_jent[a] > B.h_jent[b]; });
        for (uint32_t k = 0; k < order.size() && with_slack(total) > max_pool; ++k) {
            fallback[order[k]] = 1;
            total -= B.h_jent[order[k]];
            ++nrouted;
        }
    }
    if (with_slack(total) > B.entry_cap && (e = pool(with_slack(total))) != cudaSuccess) return e;
    for (uint32_t i = 0; i < njobs; ++i) J[i].skip = fallback[i];
    fill();
    if (nrouted) {
        // routed jobs hold no entries: their offsets are taken out of the scan
        for (uint32_t i = 0; i < njobs; ++i)
            if (fallback[i] && J[i].g.ngroups &&
                (e = cudaMemsetAsync(J[i].cap, 0, J[i].g.ngroups * sizeof(uint32_t), s)) != cudaSuccess)
                return e;
    }
    if ((e = cudaMemcpyAsync(B.d_jobs, B.h_jobs, njobs * sizeof(JobDesc), cudaMemcpyHostToDevice, s)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(B.d_hdr, B.h_hdr, sizeof(BatchHdr), cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return e;
    if (nrouted) {
        kb_scan_sums<<<kBatchScanParts, kScanThreads, 0, s>>>(B.d_hdr);
        kb_scan_psum<<<1, kScanThreads, 0, s>>>(B.d_hdr);
        kb_scan_apply<<<kBatchScanParts, kScanThreads, 0, s>>>(B.d_hdr);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    cudaEventRecord(ctx->evp[1], s);
    cudaEventRecord(ctx->evp[2], s);
    if ((e = cudaGraphLaunch(B.exec_sums, s)) != cudaSuccess) return e;
    cudaEventRecord(ctx->ev1, s);
    if ((e = cudaMemcpyAsync(B.h_hdr, B.d_hdr, sizeof(BatchHdr), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return e;
    unsigned long long timeouts = 0;
    if ((e = cudaMemcpyAsync(&timeouts, &ctx->d_stats->timeouts, sizeof timeouts, cudaMemcpyDeviceToHost, s)) !=
        cudaSuccess)
        return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    if (batch_trace()) {
        float mg = 0.f, ms = 0.f;
        cudaEventElapsedTime(&mg, ctx->ev0, ctx->evp[0]);
        cudaEventElapsedTime(&ms, ctx->evp[2], ctx->ev1);
        fprintf(stderr,
                "[hcg batch] jobs %u pixels %llu tiles %llu (windows kept for %llu) tc-items %llu entries %llu "
                "pool %llu routed %u geometry %.3f ms sums %.3f ms\n",
                njobs, pix, tile, win_tiles, tcn, total, B.entry_cap, nrouted, mg, ms);
    }
    if (timeouts) {
        why = std::to_string(timeouts) + " device pipeline waits ran out";
        return cudaErrorTimeout;
    }
    if (B.h_hdr->pool_overflow) {  // the pool was sized from the same counts: not expected
        why = "entry pool smaller than the counted entries";
        return cudaErrorMemoryAllocation;
    }
    return cudaSuccess;
}

}  // namespace hcg
