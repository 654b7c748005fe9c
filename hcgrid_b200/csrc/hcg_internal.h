// Internal types of the B200 gridder (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "hcg_math.cuh"
#include "hcgrid_c.h"

namespace hcg {

// Counters the kernels bump (read back by hcg_get_stats).
struct DevStats {
    unsigned long long pairs_candidate;
    unsigned long long pairs_within;
    unsigned long long ring_skips;
    unsigned long long hard_roundings;
    unsigned long long invalid_input;
    unsigned long long overflow;
    unsigned long long timeouts;  // bounded device waits that ran out (tensor-core engine)
    unsigned long long tc_macs;   // tensor-core multiply-adds issued (tensor-core engine)
    unsigned long long ustat[2];  // staged slots of all tiles and of the largest (tile pass)
};

// One HEALPix ring that holds samples, with the ring half of loc2pix
// precomputed (healpix.cu:126-165 splits into a ring part and a phi part).
struct RingRec {
    uint64_t startpix;
    uint64_t npr;
    double t2;       // equatorial: nside*z*0.75; polar: the `tmp` factor
    uint32_t lut_lo; // first sorted sample of the ring (start_int)
    uint32_t lut_hi; // first sample of the next ring (end_int)
    int eq;          // |z| <= 2/3
    int zpos;        // z > 0
    // Pixel table of the ring (span > 0): entry q at tbl + q is the first
    // sorted sample whose pixel is >= startpix + pmin + q, for the pixels
    // pmin .. pmin + span - 1 between the ring's first and last sample.
    uint32_t pmin;
    uint32_t span;
    uint64_t tbl;
    // Chord windows of the multi-channel path: phi of the first pixel centre,
    // the largest |phi| distance of a sample of the ring from its pixel
    // centre, the smallest cos(lat) and the latitude range (radians) of the
    // ring's samples.
    double phi0;
    double dphi;
    double cbmin;
    double bmin, bmax;
};

// One target pixel: its coordinates and the phi half of loc2pix for the two
// window edges phi -/+ disc_size (gridding.cu:306-351).
struct PixPrep {
    double l1, b1, cb1;    // radians, cos(b1)
    double tt[2];          // fmodulo((phi -/+ disc) / (pi/2), 4)
    double t1[2];          // nside * (0.5 + tt)
    double tp[2];          // tt - trunc(tt)
    int ur;                // first ring, relative to firstring
    int nr;                // number of rings (0: pixel sees no samples)
    int polar;             // whole-ring windows (theta <= 20 or >= 160 deg)
    int pad;
};

// Stream-ordered allocation from a context's memory pool. The pool keeps
// freed memory mapped (release threshold: never), so the multi-GB buffers of
// one call are reused by the next instead of being unmapped at every
// synchronize and mapped again; the pool is released with the context.
inline cudaError_t dalloc(void **p, size_t bytes, cudaStream_t s, cudaMemPool_t pool) {
    return pool ? cudaMallocFromPoolAsync(p, bytes, pool, s) : cudaMallocAsync(p, bytes, s);
}
template <class T>
inline cudaError_t dalloc(T **p, size_t bytes, cudaStream_t s, cudaMemPool_t pool) {
    return dalloc(reinterpret_cast<void **>(p), bytes, s, pool);
}

// Grow-only device scratch buffers, stream-ordered.
struct Scratch {
    cudaMemPool_t pool = nullptr;
    std::vector<void *> ptr;
    std::vector<size_t> size;
    void *get(int slot, size_t bytes, cudaStream_t s, cudaError_t &err);
    void release(cudaStream_t s);
};

}  // namespace hcg

struct hcg_context {
    std::atomic<int> refs{1};  // the context itself + each field and target made on it
    bool closed = false;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaMemPool_t pool = nullptr;        // the context's device memory (dalloc)
    cudaStream_t copy_stream = nullptr;  // host uploads overlapped with the context stream's kernels
    std::mutex mu;
    std::string err;
    // _prepare_grid_kernel state (gmap.cpp:64-99)
    bool prepared = false;
    uint32_t kernel_type = 0;
    double kparams[3] = {0, 0, 0};
    double sphere_radius = 0, disc_size = 0;
    bool bearing = false;
    bool taper_fix = false;  // HCG_TAPER_FIX
    double last_r = -1, last_res = -1;
    hcg::HpxParams hpx = {};
    hcg::DevStats *d_stats = nullptr;
    hcg::Scratch scratch;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t evp[4] = {nullptr, nullptr, nullptr, nullptr};  // phase boundaries inside hcg_grid
    cudaEvent_t evu[5] = {};  // chunked uploads: chunk copied (2), chunk scattered (2), call start
    float last_ms = 0.f;
    unsigned long long entry_budget = 4ULL << 30;  // bytes of (sample, weights) entries per launch run
    int tc_config[8] = {-1, -1, -1, -1, -1, -1, -1, -1};  // tensor-core pipeline shape per channel class (-1: default)
    int tc_pf[8] = {-1, -1, -1, -1, -1, -1, -1, -1};      // prefetch distance (chunks) per class (-1: default)
    int tc_strip[8] = {-1, -1, -1, -1, -1, -1, -1, -1};   // persistent tile walk per class (-1: default)
    int tc_weights = 0;  // tensor-core weight operands: 0 automatic, 1 from entries, 2 evaluated in the kernel
    int tune_layout = HCG_LAYOUT_SAMPLE_MAJOR;  // cube layout the single-job autotuner times
    int kb_shape[8] = {-1, -1, -1, -1, -1, -1, -1, -1};  // batch tensor-core shape per channel class (-1: default)
    uint32_t factor = 1;  // coarsening factor (hcg_set_coarsening_factor)
    void *batch = nullptr;                          // batch engine state (hcg_batch.cu)
};

struct hcg_field {
    hcg_context *ctx = nullptr;
    uint64_t n = 0;
    hcg::HpxParams hpx = {};
    double sphere_radius = 0, kparam0 = 0, disc_size = 0;  // kernel setup the field was built with
    double kparams[3] = {0, 0, 0};
    uint32_t kernel_type = 0;
    bool taper_fix = false;
    double wmax = 1.0;    // max |per-sample weight| (inf or NaN when one is not finite)
    double wbound = 1.0;  // bound of |weight| of an accepted pair: wmax * the kernel's bound
    uint64_t firstring = 0, usedrings = 0;
    uint64_t *d_keys = nullptr;   // n + 1, sorted, sentinel npix
    uint32_t *d_perm = nullptr;   // sorted position -> input index
    uint32_t *d_inv = nullptr;    // input index -> sorted position
    double *d_l2 = nullptr;       // radians, sorted
    double *d_b2 = nullptr;
    double *d_cb2 = nullptr;      // cos(b2)
    double *d_w = nullptr;        // per-sample input weight, sorted
    double4 *d_half = nullptr;    // sorted: sin(l/2), cos(l/2), sin(b/2), cos(b/2) of each sample
    uint32_t *d_lut = nullptr;    // usedrings + 1
    uint32_t *d_ptab = nullptr;   // per-ring pixel tables (RingRec::tbl), or none when too large
    uint64_t ptab_entries = 0;
    hcg::RingRec *d_rings = nullptr;
    float *d_spec = nullptr;      // [n][cstride], sorted
    uint32_t nchan = 0, cstride = 0;
    // 16-bit hi/lo split of the sorted spectra for the tensor-core engine
    uint16_t *d_xhi = nullptr, *d_xlo = nullptr;  // [n][xcpad]
    float *d_xinv = nullptr;      // [xcpad]: 1 / (channel scale * weight scale)
    uint32_t xcpad = 0;           // nchan rounded up to 64
    int xfmt = 0;                 // HCG_ENGINE_TC_BF16 / HCG_ENGINE_TC_F16, 0: no split
    unsigned long long xnonfinite = 0;  // non-finite spectrum values seen by the split
    int *geom_refs = nullptr;     // fields sharing the arrays above except d_spec (hcg_field_share)
};

struct hcg_target {
    hcg_context *ctx = nullptr;
    uint32_t nx = 0, ny = 0;
    double *d_x = nullptr, *d_y = nullptr;  // degrees
};

// Launchers (hcg_field.cu, hcg_grid.cu). All return cudaGetLastError().
namespace hcg {
constexpr int kTcClasses = 8;
constexpr int kTcConfigCount = 6;  // tensor-core pipeline shapes (hcg_tc_set_config)
constexpr int kTcDefaultPrefetch = 0;  // chunks the producer prefetches into L2 ahead of its loads (0: none)
constexpr int kTcDefaultStrip = 8;     // tile columns per strip of the persistent tile walk
constexpr uint64_t kBatchMaxPixels = 1ull << 20;  // larger targets skip hcg_grid_batch's batch pass
// Pipeline shapes of the batch engine's tensor-core kernel (kb_tc), chosen
// per channel class (hcg_batch_set_shape, hcg_autotune_batch): 64-channel
// blocks per item (the MMA's N / 64), K slots per chunk and stages.
//   0: 256 channels x 32 slots x 4 stages   1: 256 x 64 x 2
//   2: 128 x 64 x 3                         3: 64 x 64 x 4
constexpr int kKbShapes = 4;
constexpr uint32_t kKbNb[kKbShapes] = {4, 4, 2, 1};
constexpr int kKbDefaultShape = 0;
// channel class of a split field: 64-channel blocks 1, 2, 3-4, 5-8, ... -> 0, 1, 2, 3, ...
inline int tc_class_of(uint32_t cpad) {
    const uint32_t b = cpad / 64;
    int c = 0;
    while ((1u << c) < b && c < kTcClasses - 1) ++c;
    return c;
}
// HCG_ENGINE_AUTO: the tensor-core engine of the field's split spectra
// (multi-channel fields with finite spectra), else the FP32 engine.
// The tensor-core weight operand holds |w| * (power-of-two weight scale)
// below 2^15 (FP16 range); weights above 2^100 or not finite stay on FP32.
inline bool tc_weights_fit(const hcg_field *f) { return f->wbound <= 0x1p100; }
// The FP32 engine keeps weights as FP32 entries and sums w x in FP32: a
// multi-channel field whose weight bound passes 2^100 (the reference's taper
// with a narrow taper width) is refused, which leaves 2^28 for the sample
// count times |x| below FP32's range; single-channel fields sum in FP64.
inline bool fp32_weights_fit(const hcg_field *f) { return f->nchan <= 1 || !(f->wbound > 0x1p100); }
// the batch engine's tensor-core shape for a split field's channel class
inline int kb_shape_of(const hcg_context *ctx, const hcg_field *f) {
    const int c = ctx->kb_shape[tc_class_of(f->xcpad)];
    return c >= 0 && c < kKbShapes ? c : kKbDefaultShape;
}
inline int auto_engine(const hcg_field *f) {
    return (f->xfmt && f->nchan > 1 && f->xnonfinite == 0 && tc_weights_fit(f)) ? f->xfmt : HCG_ENGINE_FP32;
}
// Tensor-core weight operand: evaluated in the kernel (HCG_TC_WEIGHTS_DIRECT)
// or written as entries by the FP64 weight pass. Automatic mode evaluates in
// the kernel for dense tiles: at least 1024 staged samples per tile on average
// (beams many pixels wide over dense sampling), where the kernel's 128 x U pair
// tests are at most 2.5x the weight pass's (usum: staged slots of all `ntiles`
// tiles; cap_total: union candidates of all 2x2 groups, each for up to 4
// pixels). Measured on B200, the entries are faster below that.
// Only GAUSS1D weights are evaluated in the kernel.
inline bool tc_use_weights(const hcg_context *ctx, const hcg_field *f, unsigned long long usum,
                           unsigned long long cap_total, unsigned long long ntiles) {
    if (f->kernel_type != HCG_GAUSS1D || ctx->tc_weights == HCG_TC_WEIGHTS_ENTRIES) return false;
    if (ctx->tc_weights == HCG_TC_WEIGHTS_DIRECT) return true;
    return usum >= 1024ull * ntiles && 128.0 * (double)usum <= 2.5 * 4.0 * (double)cap_total;
}
cudaError_t build_field(hcg_context *ctx, hcg_field *f, const double *d_lon, const double *d_lat,
                        const double *d_w, std::string &why);
cudaError_t permute_spectra(hcg_context *ctx, hcg_field *f, const float *d_in, uint32_t nchan, int layout);
// Spectra from host memory in chunks, each scattered into sorted order while
// the next is copied (needs ctx->copy_stream).
constexpr uint64_t kUploadChunk = 256ull << 20;
constexpr uint32_t kPlaneBlock = 64;  // hcg_grid_planes' default block of channels
cudaError_t upload_spectra(hcg_context *ctx, hcg_field *f, const float *h_in, uint32_t nchan, int layout);
// Channel planes [nb][n] from host memory into a field's sorted spectra
// (hcg_grid_planes): copies on cs, scatters on us, staging buffers shared
// across calls through ev_copied / ev_free and the running chunk count.
cudaError_t upload_plane_block(hcg_context *ctx, hcg_field *f, const float *h_planes, uint32_t nb, cudaStream_t cs,
                               cudaStream_t us, float *const stage[2], uint64_t stage_bytes,
                               cudaEvent_t ev_copied[2], cudaEvent_t ev_free[2], uint64_t &chunks);
// Coarsening (hcg_set_coarsening_factor): each pixel takes the window fields
// of the first pixel of its run of `factor` along its row.
cudaError_t coarsen_prep(PixPrep *prep, uint32_t nx, uint64_t npix, uint32_t factor, cudaStream_t s);
cudaError_t grid_field(hcg_context *ctx, const hcg_field *f, const hcg_target *t, float *d_cube, int layout,
                       float *d_wts, int engine, std::string &why);
// hcg_tc.cu: hi/lo split of a field's spectra; tensor-core accumulation
cudaError_t split_spectra(hcg_context *ctx, hcg_field *f, int fmt_engine, std::string &why);
void free_split(hcg_field *f, cudaStream_t s);
int sin_target_coords(const char *header, size_t len, uint32_t &nx, uint32_t &ny, std::vector<double> &x,
                      std::vector<double> &y, std::string &why);
cudaError_t grid_batch(hcg_context *ctx, uint32_t njobs, const hcg_job *jobs, std::vector<char> &fallback,
                       std::string &why);
cudaError_t batch_release(hcg_context *ctx);
bool batch_trace();
uint64_t job_pixels(const hcg_job &job);         // the target's pixel count
bool job_fills_gpu(const hcg_job &job, int nsm);  // the server's large jobs (run alone)
int device_sms(int device);                       // streaming multiprocessors of a device (0: unknown)
hcg_status grid_job(hcg_context *ctx, const hcg_job &job);  // one server job, device buffers, automatic engine
struct SinWcs;
int parse_sin_header(const char *header, size_t len, uint32_t &nx, uint32_t &ny, SinWcs &w, std::string &why);
cudaError_t sin_coords_device(const SinWcs &w, uint32_t nx, uint32_t ny, double *d_x, double *d_y, cudaStream_t s);
}  // namespace hcg
