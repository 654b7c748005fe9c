/*
 * hcgrid_b200 -- C ABI of the B200 convolution gridder.
 *
 * A drop-in for the gridding path of HCGrid / HCGrid+: HEALPix pre-sort,
 * two-level ring lookup table, GAUSS1D gather gridding and weight
 * normalisation. Plain pointers and sizes only; every call returns an
 * hcg_status (no exit()), and a context is safe to use from one host thread
 * at a time (calls on one context are serialised by an internal lock).
 *
 * Reference interfaces each entry point replaces (paths inside the HCGrid
 * project):
 *   hcg_prepare_grid_kernel  _prepare_grid_kernel       HCGrid/gmap.h:121, gmap.cpp:64-99
 *   hcg_field_create         init_input_with_cpu/thrust  HCGrid/gridding.h:53-60, gridding.cu:70-216
 *                            (+ data_alloc/data_h2d of the sample arrays, gridding.cu:406-445)
 *   hcg_field_set_spectra    read_input_map data / HCGrid+ pre_order_data
 *                                                        HCGrid/gmap.cpp:102-148, HCGrid+/gridding-omp.cu:146-157
 *   hcg_target_create        set_WCS output (h_xwcs/h_ywcs) HCGrid/gmap.cpp:183-250
 *   hcg_target_from_header   read_output_map + set_WCS   HCGrid/gmap.cpp:151-250
 *   hcg_grid                 hcgrid<<<>>> + data_d2h + normalisation
 *                                                        HCGrid/gridding.cu:277-403, 448-452; gmap.cpp:306-312
 *   hcg_field_sorted         h_hpx_idx / h_start_ring (for parity checks)
 *                                                        HCGrid/gmap.h:78-81
 */
#ifndef HCGRID_C_H
#define HCGRID_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    HCG_OK = 0,
    HCG_EINVAL = 1,       /* bad argument (sizes, NaN or |lat| > 90 coordinates, unknown kernel) */
    HCG_ENOMEM = 2,       /* device or host allocation failed */
    HCG_ETIMEOUT = 3,     /* a bounded device wait ran out */
    HCG_EDEVICE = 4,      /* CUDA error */
    HCG_EIO = 5,          /* file read/write failed */
    HCG_EUNSUPPORTED = 6, /* feature not available in this build (e.g. HDF5 without libhdf5) */
    HCG_ESTATE = 7        /* call out of order (e.g. grid before prepare) */
} hcg_status;

/* Kernel types (HCGrid/constants.h:66-69) and their weights at distance d
 * (degrees) inside sphere_radius (HCGrid/gridding.cu:237-257):
 *   GAUSS1D      params (sigma): exp(-d^2 p0), p0 = 0.5 / sigma^2;
 *   GAUSS2D      params (sigma_maj, sigma_min, PA), PA in radians:
 *                exp(-(d / (smaj smin))^2 / 2 * (smaj^2 sin^2(bear - PA) +
 *                smin^2 cos^2(bear - PA))), bear the great-circle bearing of
 *                the sample seen from the pixel (helpers.cu:133-137);
 *   TAPERED_SINC params (sigma, a, b): arg = pi d / sigma,
 *                sinc(arg / b) * exp(+(arg / a)^2), the reference's taper
 *                (exp(pow(-(arg/a), 2)), gridding.cu:255);
 *   HCG_TAPERED_SINC | HCG_TAPER_FIX: the same with exp(-(arg / a)^2).
 * GAUSS1D's weights come from its FP32 exponential on the multi-channel
 * engines; the other kernels are evaluated in FP64. */
#define HCG_GAUSS1D 1
#define HCG_GAUSS2D 2
#define HCG_TAPERED_SINC 3
#define HCG_TAPER_FIX 0x100u

/* Where a buffer lives. */
#define HCG_MEM_HOST 0
#define HCG_MEM_DEVICE 1

/* Spectra / cube layouts. SAMPLE_MAJOR: values[sample][channel] (cube
 * [pixel][channel]); CHANNEL_MAJOR: values[channel][sample] (cube
 * [channel][pixel], the FITS NAXIS3-slowest order and HCGrid+'s per-channel
 * planes). */
#define HCG_LAYOUT_SAMPLE_MAJOR 0
#define HCG_LAYOUT_CHANNEL_MAJOR 1

/* Gridding engines. */
#define HCG_ENGINE_AUTO 0
#define HCG_ENGINE_FP32 1 /* FP64 geometry, FP32 CUDA-core channel accumulation */
/* FP64 geometry and weights, channel sums on the tensor cores (tcgen05) as a
 * compensated 16-bit split W X ~= Wh Xh + Wh Xl + Wl Xh with FP32
 * accumulation. Needs hcg_field_split_spectra with the same engine first;
 * single-channel fields always use the FP32 single-channel kernel. */
#define HCG_ENGINE_TC_BF16 2 /* BF16 hi/lo: per-term relative error <= 3 * 2^-16 */
#define HCG_ENGINE_TC_F16 3  /* FP16 hi/lo with power-of-two channel scales: ~3 * 2^-22 */

typedef struct hcg_context hcg_context;
typedef struct hcg_field hcg_field;
typedef struct hcg_target hcg_target;

typedef struct {
    uint64_t nside, npix, firstring, usedrings;
    double resolution; /* radians */
    double disc_size;  /* radians: sphere_radius + resolution */
    double kernel_param0; /* GAUSS1D: 0.5 / sigma^2 (sigma in degrees) */
    double sphere_radius; /* degrees */
} hcg_info;

typedef struct {
    uint64_t pairs_candidate; /* (pixel, sample) pairs inside the ring windows */
    uint64_t pairs_within;    /* of those, distance < sphere_radius */
    uint64_t ring_skips;      /* rings the reference would loop on forever (lpix/rpix outside ring) */
    uint64_t hard_roundings;  /* cos/sin roundings the double-double test could not decide */
    double ms_total;          /* device time of the last hcg_grid call */
    double ms_phase[4];       /* of which: pixel setup, candidate count + scan, FP64 weights, channel sums */
    uint64_t tc_macs;         /* tensor-core multiply-adds issued (3 per compensated product; 0 on the FP32 engine) */
} hcg_stats;

const char *hcg_status_string(hcg_status s);

/* Context on CUDA device `device`; `stream` (cudaStream_t, may be NULL for a
 * private stream) orders all work of the context. */
hcg_status hcg_context_create(int device, void *stream, hcg_context **out);
hcg_status hcg_context_destroy(hcg_context *ctx);
const char *hcg_last_error(const hcg_context *ctx);

/* _prepare_grid_kernel: GAUSS1D params[0] = sigma (deg) is replaced in place
 * by 0.5/sigma^2, as the reference does (GAUSS2D and TAPERED_SINC take their
 * three parameters as given); nside follows from hpx_max_res
 * (deg); HEALPix is rebuilt only if sphere_radius or hpx_max_res moved by
 * more than 3e-5 since the previous call on this context. */
hcg_status hcg_prepare_grid_kernel(hcg_context *ctx, uint32_t kernel_type, double *kernel_params,
                                   double sphere_radius, double hpx_max_res);
hcg_status hcg_get_info(const hcg_context *ctx, const hcg_field *field, hcg_info *out);

/* Samples: lon/lat in degrees (float64), optional per-sample weights
 * (float64, NULL = 1 as in the reference). Computes HEALPix keys, the stable
 * on-device radix sort, the permuted geometry and the ring lookup table. */
hcg_status hcg_field_create(hcg_context *ctx, uint64_t n, const double *lon, const double *lat,
                            const double *weights, int mem, hcg_field **out);
/* Attach spectra (float32) in either layout; permuted into sorted order on
 * the device and kept resident. */
hcg_status hcg_field_set_spectra(hcg_field *field, uint32_t nchan, const float *values, int layout, int mem);

/* Store the field's spectra a second time as 16-bit hi/lo pairs (per-channel
 * power-of-two scale for HCG_ENGINE_TC_F16) for the tensor-core engine
 * `engine`. keep_fp32 = 0 frees the FP32 copy (the FP32 engine is then not
 * available for this field until hcg_field_set_spectra). Non-finite values
 * are counted: such fields are refused by the tensor-core engines
 * (HCG_EINVAL). hcg_field_set_spectra drops the split. No reference
 * counterpart (the reference grids FP64 on CUDA cores). */
hcg_status hcg_field_split_spectra(hcg_field *field, int engine, int keep_fp32);

/* Tensor-core pipeline shapes (the autotuner's search space), per CTA work
 * item of one 16x8-pixel tile:
 *   0: 256 channels per item, 64-sample chunks, 2 pipeline stages
 *   1: 128 channels per item, 64-sample chunks, 3 stages
 *   2:  64 channels per item, 64-sample chunks, 4 stages
 *   3: 256 channels per item, 32-sample chunks, 4 stages
 *   4: shape 0 in a persistent kernel (one CTA per SM; the epilogue of a
 *      tile overlaps the next tile's MMAs)
 *   5: shape 3 in the persistent kernel
 * Channel classes: 64-channel blocks 1, 2, 3-4, 5-8, 9-16, ... -> 0, 1, 2, 3, 4, ...
 * hcg_tc_set_config sets the shape of one class (-1: every class); config -1
 * restores the default (the widest item the channels fill).
 * hcg_autotune grids (field, target) with each shape `reps` times (device
 * scratch output), keeps the fastest for the field's channel class and
 * returns it and the best time of each shape (ms[6], may be NULL). The field
 * must hold split spectra. No reference counterpart. */
hcg_status hcg_tc_set_config(hcg_context *ctx, int channel_class, int config);

/* How the tensor-core engines build the weight operand of a tile:
 *   HCG_TC_WEIGHTS_AUTO    (0): per call, from the tile pass's counts: evaluated in
 *                              the kernel for dense tiles (at least 1024 staged
 *                              samples per tile, dense evaluation at most 2.5x the
 *                              weight pass's pairs), else entries;
 *   HCG_TC_WEIGHTS_ENTRIES (1): an FP64 weight pass writes entries (pixel-group,
 *                              sample, 4 weights) that the kernel scatters;
 *   HCG_TC_WEIGHTS_DIRECT  (2): the kernel's builder warps evaluate the FP64
 *                              distance, cutoff and Gaussian of every staged
 *                              sample for every pixel of the tile (GAUSS1D
 *                              fields; the other kernels always use entries).
 * The accepted pairs and weights are the same; the FP64 weight sums can differ
 * in the last bits (summation order). No reference counterpart. */
#define HCG_TC_WEIGHTS_AUTO 0
#define HCG_TC_WEIGHTS_ENTRIES 1
#define HCG_TC_WEIGHTS_DIRECT 2
hcg_status hcg_tc_set_weights(hcg_context *ctx, int mode);
hcg_status hcg_autotune(hcg_context *ctx, const hcg_field *field, const hcg_target *target, int reps, int *best,
                        float *ms);

/* Pipeline depth and tile walk of the tensor-core engine, per channel class
 * (-1: every class; a value of -1 restores the default):
 *   prefetch  chunks of staged spectra the producer also requests into L2
 *             ahead of its shared-memory loads (0: none; values up to the
 *             shape's stages mean the stages themselves); a prefetch
 *             instruction holds the producer warp as long as a load, so it
 *             pays only where the loads' latency is exposed; default 0;
 *   strip     the persistent kernels take the tiles of a launch in strips of
 *             `strip` tile columns, row by row inside a strip, so that the
 *             tiles in flight together form a compact block whose neighbours
 *             share staged samples in L2 (0: whole tile rows); default 8.
 * No reference counterpart. */
hcg_status hcg_tc_set_pipeline(hcg_context *ctx, int channel_class, int prefetch, int strip);

/* Cube layout the single-job autotuners (hcg_autotune, hcg_autotune_ex) grid
 * in while they time the pipeline choices (default HCG_LAYOUT_SAMPLE_MAJOR):
 * the epilogue's stores differ between layouts, so tune in the layout the
 * application grids in. No reference counterpart. */
hcg_status hcg_autotune_layout(hcg_context *ctx, int layout);

/* The autotuner's full search (hcg_autotune is its shape part): the
 * pipeline shape (ms_shape, defaults elsewhere), then with that shape the
 * prefetch distance over kTunePrefetch, then the strip width over
 * kTuneStrip; each setting is timed `reps` times after a warm-up run and
 * scored by its best run. The choices are kept for the field's channel class
 * and returned; spread = (slowest - fastest) / fastest over the chosen
 * setting's repeats. */
#define HCG_TUNE_PREFETCH {0, 2, 4, 6, 8}
#define HCG_TUNE_STRIP {0, 4, 8, 16, 32}
typedef struct {
    int shape, prefetch, strip;
    float ms_shape[6];
    float ms_prefetch[5];
    float ms_strip[5];
    float ms_best, spread;
} hcg_tuning;
hcg_status hcg_autotune_ex(hcg_context *ctx, const hcg_field *field, const hcg_target *target, int reps,
                           hcg_tuning *out);
/* Sorted keys (n+1 with the npix sentinel), permutation (n) and ring LUT
 * (usedrings+1); any pointer may be NULL. Host memory. */
hcg_status hcg_field_sorted(const hcg_field *field, uint64_t *keys, uint32_t *perm, uint32_t *lut);

/* Dec-band sharding (no reference counterpart). For the target rows
 * [y0, y1): the sorted positions [*s0, *s1) (positions in hcg_field_sorted's
 * order; perm maps them to input samples) such that a field made of those
 * samples alone, in that order, grids the rows as this field does: the
 * complete rings their pixels visit (HCGrid/gridding.cu:306-323) and one
 * sample in front, whose ring takes the place of the first used ring that
 * the reference never grids (gridding.cu:326,363-367). *s0 == *s1 when the
 * rows see no samples (their pixels are empty: NaN, weight 0). */
hcg_status hcg_field_band_samples(hcg_context *ctx, const hcg_field *field, const hcg_target *target,
                                  uint32_t y0, uint32_t y1, uint64_t *s0, uint64_t *s1);
hcg_status hcg_field_destroy(hcg_field *field);
/* A second handle on the same resident geometry (sorted samples, LUT, ring
 * table) without spectra: new spectra on known sample positions skip the
 * sort. The geometry is freed with the last handle. */
hcg_status hcg_field_share(const hcg_field *field, hcg_field **out);

/* Target pixel centres in degrees, indexed yy*nx + xx. */
hcg_status hcg_target_create(hcg_context *ctx, uint32_t nx, uint32_t ny, const double *xwcs, const double *ywcs,
                             int mem, hcg_target **out);
/* Target from a FITS header (80-char cards): RA---SIN / DEC--SIN with
 * CRPIX/CDELT/CRVAL (and LONPOLE); pixel (xx+1, yy+1) as set_WCS does. */
hcg_status hcg_target_from_header(hcg_context *ctx, const char *header, size_t len, hcg_target **out);
hcg_status hcg_target_coords(const hcg_target *t, uint32_t *nx, uint32_t *ny, double *xwcs, double *ywcs);
/* The same SIN pixel centres on the host, without a device: first call with
 * xwcs = ywcs = NULL for nx, ny; then with arrays of nx*ny doubles. */
hcg_status hcg_header_coords(const char *header, size_t len, uint32_t *nx, uint32_t *ny, double *xwcs,
                             double *ywcs);
hcg_status hcg_target_destroy(hcg_target *t);

/* Grid the field's spectra onto the target and normalise: cube = sum(w x) /
 * sum(w) (NaN where no sample contributes, as the reference's 0/0), float32;
 * weights_out (optional, float32 [npix]) = sum(w). mem says where cube and
 * weights_out live. */
hcg_status hcg_grid(hcg_context *ctx, const hcg_field *field, const hcg_target *target, float *cube, int layout,
                    float *weights_out, int mem, int engine);
/* Host spectra in, host cube out, as one pipelined call: `planes` holds the
 * spectra as channel planes in input sample order, [nchan][n] floats (the
 * reference's h_data[channel][sample]); `geometry` is a field of the same n
 * samples from hcg_field_create (its own spectra, if any, are not used).
 * The channels go through in blocks of `block` (a multiple of 64; 0: 64):
 * while block b is split and gridded, block b + 1 is uploaded and block b - 1
 * downloaded, the two copies on their own streams in the two directions of
 * the bus. cube: [nchan][npix] (HCG_LAYOUT_CHANNEL_MAJOR) or [npix][nchan];
 * weights_out optional, [npix]. planes, cube and weights_out are host memory,
 * page-locked for the copies to overlap. engine: HCG_ENGINE_FP32 or a
 * tensor-core engine (each block is split for it; AUTO: FP16 hi/lo). The
 * FP32 engine's cube equals hcg_grid's bit for bit; the tensor cores run
 * the pipeline shape of each block's channel count, which agrees with
 * hcg_grid's to the FP32 accumulation's rounding; a block of one channel
 * takes the single-channel FP64 path, as a one-channel field does. The
 * statistics (hcg_get_stats) are the last block's. Counterpart: the
 * reference's per-channel streams, each uploading its channel, gridding it
 * and downloading its plane (HCGrid+/gridding-omp.cu:616-626). */
hcg_status hcg_grid_planes(hcg_context *ctx, const hcg_field *geometry, const hcg_target *target,
                           const float *planes, uint32_t nchan, float *cube, int layout, float *weights_out,
                           int engine, uint32_t block);
hcg_status hcg_get_stats(hcg_context *ctx, hcg_stats *out);

/* One job of a batch: a field (with spectra), a target and DEVICE output
 * buffers (cube in `layout`, weights optional). */
typedef struct {
    const hcg_field *field;
    const hcg_target *target;
    float *cube;
    float *weights;
    int layout;
} hcg_job;

/* Grid many independent jobs in one pass: each phase is one persistent
 * launch over all jobs' work items fed by a device-side queue, and the pass
 * is a CUDA graph replayed per batch. Jobs may differ in sample count, map
 * size, channel count and kernel (each field grids with the kernel setup it
 * was created under; the batch pass takes GAUSS1D jobs, GAUSS2D and
 * TAPERED_SINC jobs run after it one at a time, as do jobs whose targets
 * have 2^20 pixels or more: those fill the GPU by themselves). Returns when
 * all cubes are written; each cube equals what hcg_grid writes for that
 * job. */
hcg_status hcg_grid_batch(hcg_context *ctx, uint32_t njobs, const hcg_job *jobs);

/* Pipeline shape of the batch pass's tensor-core kernel, per channel class
 * (the tensor-core classes of hcg_tc_set_pipeline; -1: every class; shape -1
 * restores the default 0). Every shape takes 16 x 8-pixel tiles (128 pixels
 * per item, the MMA's M); they differ in channels per item (the MMA's N),
 * sample slots per pipeline chunk and pipeline depth:
 *   0: 256 channels x 32 slots x 4 stages   1: 256 x 64 x 2
 *   2: 128 x 64 x 3                         3: 64 x 64 x 4
 * The cubes do not depend on the shape. No reference counterpart (HCGrid
 * grids one job per call). */
#define HCG_BATCH_SHAPES 4
hcg_status hcg_batch_set_shape(hcg_context *ctx, int channel_class, int shape);

/* Autotuner of the batch pass: the jobs the batch pass would take on the
 * tensor cores are grouped by channel class; for each class present, every
 * shape runs the class's jobs as one hcg_grid_batch (one warm-up, then
 * `reps` timed runs, host clock around the call), the fastest best-of-reps
 * is kept for the class (hcg_batch_set_shape) and reported in out[0..*nout)
 * (at most max_out entries); spread = (slowest - fastest) / fastest of the
 * chosen shape's runs. The jobs' cubes are written along the way. */
typedef struct {
    int channel_class;
    int shape;
    uint32_t jobs;
    float ms[HCG_BATCH_SHAPES];
    float spread;
} hcg_batch_tuning;
hcg_status hcg_autotune_batch(hcg_context *ctx, uint32_t njobs, const hcg_job *jobs, int reps, uint32_t max_out,
                              hcg_batch_tuning *out, uint32_t *nout);

/* Serving loop with continuous batching. `lanes` contexts on `device` (the
 * first is ctx) each replay their own batch graph on their own stream, so a
 * batch admitted while another runs overlaps with it on the GPU. Jobs are
 * admitted in arrival order while the sum of their footprints (bytes,
 * caller's estimate of output + scratch) stays within hbm_budget_bytes, at
 * most max_batch per batch. Fields and targets must be ready (their upload
 * finished: hcg_synchronize on their context) before submission; outputs
 * are device buffers. hcg_server_wait returns the job's status and its
 * latency (submit -> cube written) and queueing time in seconds. */
typedef struct hcg_server hcg_server;
hcg_status hcg_server_create(hcg_context *ctx, int device, uint32_t lanes, uint64_t hbm_budget_bytes,
                             uint32_t max_batch, hcg_server **out);
hcg_status hcg_server_submit(hcg_server *server, const hcg_job *job, uint64_t footprint_bytes, uint64_t *ticket);
hcg_status hcg_server_wait(hcg_server *server, uint64_t ticket, double *latency_s, double *queue_s);
hcg_status hcg_server_drain(hcg_server *server);
hcg_status hcg_server_stats(hcg_server *server, double *p50_s, double *p99_s, uint64_t *jobs, uint32_t *batches);
hcg_status hcg_server_destroy(hcg_server *server);
/* Upper bound (bytes) of the per-call candidate entry buffer of the
 * multi-channel engine; larger jobs are processed in runs of tile rows
 * (default 4 GiB). */
hcg_status hcg_set_entry_budget(hcg_context *ctx, uint64_t bytes);

/* HCGrid's coarsening factor (h_GMaps.factor, HCGrid/gridding.cu:284-308):
 * the pixels of each target row are taken in runs of `factor` (1-3) from
 * x = 0; every pixel of a run takes the ring range, the HEALPix pixel
 * windows of each ring and the polar rule from the disc of the run's first
 * pixel, and keeps its own distance, cutoff and weight. 1 (the default):
 * every pixel its own disc. Applies to hcg_grid and hcg_grid_noalloc on
 * this context; hcg_grid_batch on a context with factor > 1 grids each job
 * on its own. */
hcg_status hcg_set_coarsening_factor(hcg_context *ctx, uint32_t factor);

/* Device memory: every buffer of a context (fields, targets, scratch) comes
 * from the context's own stream-ordered pool, which keeps freed memory
 * mapped so that the next field or call reuses it without new mappings (no
 * reference counterpart; the reference cudaMallocs and frees per run). This
 * returns what the pool keeps beyond the buffers in use to the driver. */
hcg_status hcg_context_trim(hcg_context *ctx);

/* Wait for all work queued on the context's stream. */
hcg_status hcg_synchronize(hcg_context *ctx);

/* hcg_grid for single-channel fields without any allocation. No counterpart
 * in the reference. For callers that cannot allocate device memory at the
 * time they grid: a real-time pipeline (a telescope backend gridding each
 * scan as it lands) that reserves all its device memory when it starts, so
 * that an observation never meets an allocation failure or the device-wide
 * stall of cudaMalloc/cudaFree; or a host application whose own allocator
 * already holds the GPU's memory and lends the library only the inputs and
 * outputs. Its per-pixel scratch is a fixed array inside the library of
 * 131072 pixels (12 MiB, held on every GPU that loads the library until the
 * process exits): larger targets are rejected with HCG_EINVAL. cube and
 * weights_out (optional) are device buffers of nx*ny floats on the
 * context's device, and field and target must belong to a context on that
 * device (HCG_EINVAL otherwise, before anything is launched). The first
 * call on a device looks up the array's device address; make it before any
 * stream capture. Calls share the array, so calls whose work overlaps on the
 * GPU race: issue them one after another. Asynchronous on the context's
 * stream, like hcg_grid with device buffers. */
hcg_status hcg_grid_noalloc(hcg_context *ctx, const hcg_field *field, const hcg_target *target, float *cube,
                            float *weights_out);

/* FITS boundary, host only, in the reference's formats (HCGrid/gmap.cpp):
 *   hcg_fits_read_samples   read_input_map (gmap.cpp:102-148): values from the
 *                           primary image (N = NAXIS1*NAXIS2 samples, NAXIS3
 *                           channels, written [nchan][n]), lon/lat (deg) from
 *                           the second HDU. Call with NULL arrays for n, nchan.
 *   hcg_fits_read_header    read_output_map (gmap.cpp:151-180): the primary
 *                           header as 80-char cards ending with END.
 *   hcg_fits_write_cube     write_output_map (gmap.cpp:253-323): the cube
 *                           [nchan][ny][nx] (BITPIX -32 or -64) with the
 *                           target's cards, plus a WEIGHTS image extension when
 *                           weights is not NULL.
 *   hcg_fits_write_samples  write_ordered_map (gmap.cpp:326-379): samples in
 *                           the given (sorted) order, same layout as the input. */
hcg_status hcg_fits_read_samples(const char *path, uint64_t *n, uint32_t *nchan, double *lon, double *lat,
                                 float *values);
hcg_status hcg_fits_read_header(const char *path, char *header, size_t cap, size_t *len);
hcg_status hcg_fits_write_cube(const char *path, const char *target_header, size_t len, uint32_t nx, uint32_t ny,
                               uint32_t nchan, const float *cube, const float *weights, int bitpix);
hcg_status hcg_fits_write_samples(const char *path, uint64_t n, uint32_t nchan, const double *lon,
                                  const double *lat, const float *values);

#ifdef __cplusplus
}
#endif
#endif
