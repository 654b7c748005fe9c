/*
 * CPU restatement of HCGrid's gridding path (test infrastructure only).
 *
 * This is the checker for the CUDA path: tests, the smoke check and the
 * bench's CPU-baseline leg call it; the product never does. Each function
 * names the reference file:line it restates. Parity of this restatement is
 * pinned against the reference's own code compiled for the host
 * (oracle/_ref, built by oracle/Makefile) and against the committed golden
 * vectors in tests/golden/.
 */
#ifndef HCG_ORACLE_H
#define HCG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_Y 1073741824ULL /* constants.h:57, returned for invalid theta */
#define ORC_GAUSS1D 1
#define ORC_GAUSS2D 2
#define ORC_TAPERED_SINC 3
/* OR'd into the kernel type: TAPERED_SINC with the taper exp(-(arg/p1)^2)
 * instead of the reference's exp(+(arg/p1)^2) (gridding.cu:255). */
#define ORC_TAPER_FIX 0x100u

typedef struct {
    uint64_t nside, order, nrings, npface, ncap, npix;
    double fact1, fact2, resolution, omega;
} orc_healpix;

typedef struct {
    orc_healpix hpx;
    uint32_t kernel_type;
    double params[3];      /* after the in-place transform of _prepare_grid_kernel */
    double sphere_radius;  /* degrees */
    double disc_size;      /* radians */
    int bearing_needed;
    int taper_fix;         /* ORC_TAPER_FIX was given */
} orc_gmaps;

typedef struct {
    long long pairs_visited;  /* candidate (pixel, sample) pairs the ring windows produced */
    long long pairs_within;   /* pairs with distance < sphere_radius */
    long long a3_events;      /* rings skipped because lpix/rpix fell outside the ring */
} orc_stats;

/* helpers.cu */
uint64_t orc_ilog2(uint64_t arg);
uint64_t orc_isqrt(uint64_t arg);
double orc_fmodulo(double v1, double v2);
uint64_t orc_set_optimal_nside(double target_res);
uint64_t orc_nside_to_order(uint64_t nside);

/* healpix.cu */
void orc_healpix_init(orc_healpix *h, uint64_t nside);
void orc_ring_info(const orc_healpix *h, uint64_t ring, uint64_t *startpix, uint64_t *npr, int *shifted);
uint64_t orc_pix2ring(const orc_healpix *h, uint64_t pix);
uint64_t orc_loc2pix(const orc_healpix *h, double z, double phi, double sth, int have_sth);
uint64_t orc_ang2pix(const orc_healpix *h, double theta, double phi);
void orc_pix2loc(const orc_healpix *h, uint64_t pix, double *z, double *phi, double *sth, int *have_sth);
void orc_pix2ang(const orc_healpix *h, uint64_t pix, double *theta, double *phi);

/* gmap.cpp:64-99 (params is transformed in place for GAUSS1D) */
int orc_prepare_grid_kernel(orc_gmaps *g, uint32_t kernel_type, double *params, double sphere_radius,
                            double hpx_max_res);

/* gridding.cu:70-136 with order_arg = PARALLEL_STABLE_SORT */
void orc_sample_keys(const orc_healpix *h, long n, const double *lons, const double *lats, uint64_t *keys);
void orc_stable_sort(long n, const uint64_t *keys, uint64_t *sorted_keys, uint32_t *perm);
long orc_ring_lut(const orc_healpix *h, long n, const uint64_t *sorted_keys, uint64_t *firstring,
                  uint64_t *usedrings, uint32_t *lut, long lut_cap);

/* gridding.cu:277-403 kernel semantics, FP64, for C channels (HCGrid+ runs
 * the same body once per channel). data is [n][nchan] in sorted order;
 * cube_out is [npix][nchan]; wts_out is [npix]. Unnormalised, as the
 * kernel leaves them. Pixels are indexed yy*nx+xx (rectangular maps are
 * handled properly; for square maps this is the reference's indexing).
 * mode 0 = compat (reference selection, quirks A1-A5 reproduced, A3 counted
 * and skipped), mode 1 = exact disc (every sample with d < sphere_radius). */
void orc_grid(const orc_gmaps *g, long n, const uint64_t *sorted_keys, const uint32_t *lut, uint64_t firstring,
              uint64_t usedrings, const double *lons, const double *lats, const double *weights, const double *data,
              long nchan, long npix_map, const double *xwcs, const double *ywcs, int mode, double *cube_out,
              double *wts_out, orc_stats *stats);
/* orc_grid, and when wabs_out is not NULL also sum |weight| per pixel (the
 * conditioning of the normalisation for kernels with negative lobes). */
void orc_grid_ex(const orc_gmaps *g, long n, const uint64_t *sorted_keys, const uint32_t *lut, uint64_t firstring,
                 uint64_t usedrings, const double *lons, const double *lats, const double *weights,
                 const double *data, long nchan, long npix_map, const double *xwcs, const double *ywcs, int mode,
                 double *cube_out, double *wts_out, double *wabs_out, orc_stats *stats);

/* gmap.cpp:306-312: datacube / weights (0/0 gives NaN). */
void orc_normalize(long npix_map, long nchan, const double *cube, const double *wts, double *out);

/* Per-pixel ring range and per-ring sample windows exactly as the kernel
 * forms them (gridding.cu:306-367); used to pin the device window logic.
 * For pixel p returns uring, dring and, for each ring in between, the
 * [lo, hi) index interval of candidate samples (hi == lo when skipped). */
long orc_pixel_windows(const orc_gmaps *g, long n, const uint64_t *sorted_keys, const uint32_t *lut,
                       uint64_t firstring, uint64_t usedrings, double xwcs, double ywcs, uint64_t *uring,
                       uint64_t *dring, uint32_t *lo, uint32_t *hi, long cap, long *a3);

/* Bulk forms used by the tests. */
void orc_ang2pix_many(const orc_healpix *h, long n, const double *theta, const double *phi, uint64_t *out);
void orc_pix2ring_many(const orc_healpix *h, long n, const uint64_t *pix, uint64_t *out);
void orc_pix2ang_many(const orc_healpix *h, long n, const uint64_t *pix, double *theta, double *phi);
void orc_ring_info_many(const orc_healpix *h, long n, const uint64_t *ring, uint64_t *startpix, uint64_t *npr);

#ifdef __cplusplus
}
#endif
#endif
