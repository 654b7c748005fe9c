/*
 * Entry points around the reference's own HCGrid code, built for the host.
 *
 * TEST INFRASTRUCTURE ONLY. oracle/Makefile compiles this file together with
 * the reference's HCGrid/healpix.cu, helpers.cu, gmap.cpp and gridding.cu
 * (taken from the read-only reference tree at build time, never copied into
 * the repository) against the emulation headers in oracle/shim/. Every
 * function below only sets the reference's globals and calls the
 * reference's functions; none of the algorithm is restated here.
 *
 *   ref_prepare_grid_kernel  -> _prepare_grid_kernel   (HCGrid/gmap.cpp:64-99)
 *   ref_ang2pix etc.         -> h_ang2pix, h_pix2ring,  (HCGrid/healpix.cu)
 *                               h_get_ring_info_small, h_pix2ang, h_loc2pix
 *   ref_presort              -> init_input_with_cpu / init_input_with_thrust
 *                               (HCGrid/gridding.cu:70-216)
 *   ref_grid                 -> init_output, data_alloc, data_h2d, the body
 *                               of the `hcgrid` kernel, data_d2h
 *                               (HCGrid/gridding.cu:219-452, 277-403)
 *   ref_solve_gridding       -> solve_gridding (HCGrid/gridding.cu:484-556),
 *                               the reference's whole FITS-in/FITS-out path.
 */
#include <sys/time.h>
#include <stdint.h>
#include <string.h>
#include <vector>

#include "gridding.h"

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;

double hcg_emu_now_ms() {
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec * 1e3 + tv.tv_usec * 1e-3;
}

/* The reference kernel and device-side pointers defined in gridding.cu. */
extern double *d_lons, *d_lats, *d_data, *d_weights, *d_xwcs, *d_ywcs, *d_datacube, *d_weightscube;
extern uint64_t *d_hpx_idx;
extern uint32_t *d_start_ring;
extern texture<uint32_t> tex_start_ring;

extern "C" {

/* Healpix state as plain numbers: [nside, order, nrings, npface, ncap, npix,
 * firstring, usedrings] and [fact1, fact2, resolution, omega]. */
void ref_healpix_state(uint64_t *u, double *d) {
    u[0] = h_Healpix._nside; u[1] = h_Healpix._order; u[2] = h_Healpix._nrings; u[3] = h_Healpix._npface;
    u[4] = h_Healpix._ncap; u[5] = h_Healpix._npix; u[6] = h_Healpix.firstring; u[7] = h_Healpix.usedrings;
    d[0] = h_Healpix._fact1; d[1] = h_Healpix._fact2; d[2] = h_Healpix._resolution; d[3] = h_Healpix._omega;
}

void ref_healpix_init(uint64_t nside) { _Healpix_init(nside, RING); }

/* HCGrid.cpp:137-151 order of calls: _Healpix_init(1, RING) then
 * _prepare_grid_kernel. kernel_params is copied into a malloc'd array because
 * the reference keeps (and later frees) the pointer it is given. */
void ref_prepare_grid_kernel(uint32_t kernel_type, const double *params3, double sphere_radius, double hpx_max_res,
                             double *params_out, double *disc_size, double *sphere_radius_out) {
    double *kp = (double *)malloc(3 * sizeof(double));
    memcpy(kp, params3, 3 * sizeof(double));
    /* Start like a fresh process: the reference only rebuilds HEALPix when
     * the radius or resolution moved by > 3e-5 since its previous call
     * (gmap.cpp:89-95), which across cases in one process would keep a stale
     * nside. */
    last_sphere_radius = -1;
    last_hpxmaxres = -1;
    _prepare_grid_kernel(kernel_type, kp, sphere_radius, hpx_max_res);
    memcpy(params_out, kp, 3 * sizeof(double));
    *disc_size = h_GMaps.disc_size;
    *sphere_radius_out = h_GMaps.sphere_radius;
}

void ref_ang2pix(long n, const double *theta, const double *phi, uint64_t *out) {
    for (long i = 0; i < n; ++i) out[i] = h_ang2pix(theta[i], phi[i]);
}
void ref_loc2pix(long n, const double *z, const double *phi, const double *sth, const int *have, uint64_t *out) {
    for (long i = 0; i < n; ++i) out[i] = h_loc2pix(z[i], phi[i], sth[i], have[i] != 0);
}
void ref_pix2ring(long n, const uint64_t *pix, uint64_t *out) {
    for (long i = 0; i < n; ++i) out[i] = h_pix2ring(pix[i]);
}
void ref_ring_info(long n, const uint64_t *ring, uint64_t *startpix, uint64_t *npr, int *shifted) {
    for (long i = 0; i < n; ++i) {
        bool s;
        h_get_ring_info_small(ring[i], startpix[i], npr[i], s);
        shifted[i] = s;
    }
}
void ref_pix2ang(long n, const uint64_t *pix, double *theta, double *phi) {
    for (long i = 0; i < n; ++i) h_pix2ang(pix[i], theta[i], phi[i]);
}
uint64_t ref_set_optimal_nside(double target_res) { return set_optimal_nside(target_res); }

/* Sample keys, sort, permutation and ring lookup table exactly as the
 * reference computes them. keys_out has n+1 entries (sentinel npix last). */
int ref_presort(uint32_t n, const double *lons, const double *lats, const double *data, int order_arg,
                uint64_t *keys_out, double *lons_out, double *lats_out, double *data_out, uint64_t *firstring,
                uint64_t *usedrings, uint32_t *lut_out, uint32_t lut_cap) {
    h_GMaps.data_shape = n;
    h_lons = RALLOC(double, n);
    h_lats = RALLOC(double, n);
    h_data = RALLOC(double, n);
    memcpy(h_lons, lons, n * sizeof(double));
    memcpy(h_lats, lats, n * sizeof(double));
    memcpy(h_data, data, n * sizeof(double));
    if (order_arg == THRUST)
        init_input_with_thrust(order_arg);
    else
        init_input_with_cpu(order_arg);
    fflush(stdout);
    memcpy(keys_out, h_hpx_idx, (n + 1) * sizeof(uint64_t));
    memcpy(lons_out, h_lons, n * sizeof(double));
    memcpy(lats_out, h_lats, n * sizeof(double));
    memcpy(data_out, h_data, n * sizeof(double));
    *firstring = h_Healpix.firstring;
    *usedrings = h_Healpix.usedrings;
    int rc = 0;
    if (h_Healpix.usedrings + 1 > lut_cap)
        rc = -1;
    else
        memcpy(lut_out, h_start_ring, (h_Healpix.usedrings + 1) * sizeof(uint32_t));
    DEALLOC(h_lons); DEALLOC(h_lats); DEALLOC(h_data); DEALLOC(h_hpx_idx); DEALLOC(h_start_ring);
    return rc;
}

/* One reference kernel run over already-sorted inputs (one channel).
 * nx = NAXIS1, ny = NAXIS2; the reference indexes pixels as row*NAXIS2+col
 * (square-map assumption), so callers pass square maps. Block size 32 makes
 * the launch grid exactly block_warp_num*NAXIS2 warps (no idle warps). */
int ref_grid(uint32_t n, const uint64_t *keys, const double *lons, const double *lats, const double *data,
             const double *weights, const uint32_t *lut, uint64_t firstring, uint64_t usedrings, uint32_t nx,
             uint32_t ny, const double *xwcs, const double *ywcs, uint32_t factor, double *cube_out,
             double *wts_out) {
    h_GMaps.data_shape = n;
    h_GMaps.spec_dim = 1;
    h_GMaps.factor = factor;
    h_Healpix.firstring = firstring;
    h_Healpix.usedrings = usedrings;
    h_zyx = RALLOC(uint32_t, 3);
    h_zyx[0] = 1; h_zyx[1] = ny; h_zyx[2] = nx;
    h_GMaps.block_warp_num = (h_zyx[1] - 1) / (32 * h_GMaps.factor) + 1;
    uint32_t num = nx * ny;
    h_lons = RALLOC(double, n); memcpy(h_lons, lons, n * sizeof(double));
    h_lats = RALLOC(double, n); memcpy(h_lats, lats, n * sizeof(double));
    h_data = RALLOC(double, n); memcpy(h_data, data, n * sizeof(double));
    h_weights = RALLOC(double, n); memcpy(h_weights, weights, n * sizeof(double));
    h_hpx_idx = RALLOC(uint64_t, n + 1); memcpy(h_hpx_idx, keys, (n + 1) * sizeof(uint64_t));
    h_start_ring = RALLOC(uint32_t, usedrings + 1); memcpy(h_start_ring, lut, (usedrings + 1) * sizeof(uint32_t));
    h_xwcs = RALLOC(double, num); memcpy(h_xwcs, xwcs, num * sizeof(double));
    h_ywcs = RALLOC(double, num); memcpy(h_ywcs, ywcs, num * sizeof(double));
    init_output();
    data_alloc();
    data_h2d();
    dim3 block(32);
    dim3 grid((h_GMaps.block_warp_num * h_zyx[1] - 1) / (block.x / 32) + 1);
    HCG_EMU_LAUNCH(grid, block, hcgrid, d_lons, d_lats, d_data, d_weights, d_xwcs, d_ywcs, d_datacube,
                   d_weightscube, d_hpx_idx);
    data_d2h();
    memcpy(cube_out, h_datacube, num * sizeof(double));
    memcpy(wts_out, h_weightscube, num * sizeof(double));
    /* data_free() would also free the kernel parameters kept by
     * _prepare_grid_kernel; release everything else the same way. */
    DEALLOC(h_lons); cudaFree(d_lons); DEALLOC(h_lats); cudaFree(d_lats);
    DEALLOC(h_data); cudaFree(d_data); DEALLOC(h_weights); cudaFree(d_weights);
    DEALLOC(h_xwcs); cudaFree(d_xwcs); DEALLOC(h_ywcs); cudaFree(d_ywcs);
    DEALLOC(h_datacube); cudaFree(d_datacube); DEALLOC(h_weightscube); cudaFree(d_weightscube);
    DEALLOC(h_hpx_idx); cudaFree(d_hpx_idx); DEALLOC(h_start_ring); cudaUnbindTexture(tex_start_ring);
    cudaFree(d_start_ring); DEALLOC(h_zyx);
    return 0;
}

/* The reference's complete FITS path (read input + target, WCS through
 * wcslib, sort, kernel, normalise, write). `factor` is HCGrid's
 * coarsening factor (1 = off). */
void ref_solve_gridding(const char *infile, const char *tarfile, const char *outfile, int order_arg, int bdim,
                        uint32_t factor) {
    h_GMaps.factor = factor;
    solve_gridding(infile, tarfile, outfile, NULL, order_arg, bdim);
    fflush(stdout);
}

/* set_WCS through the reference's read_output_map (gmap.cpp:151-250). */
int ref_target_wcs(const char *tarfile, uint32_t *nx, uint32_t *ny, uint32_t *nz, double *xwcs, double *ywcs,
                   long cap) {
    h_GMaps.factor = 1;
    read_output_map(tarfile);
    *nz = h_zyx[0]; *ny = h_zyx[1]; *nx = h_zyx[2];
    long num = (long)h_zyx[1] * h_zyx[2];
    if (num > cap) { DEALLOC(h_zyx); DEALLOC(h_header); return -1; }
    int ok = set_WCS();
    memcpy(xwcs, h_xwcs, num * sizeof(double));
    memcpy(ywcs, h_ywcs, num * sizeof(double));
    DEALLOC(h_xwcs); DEALLOC(h_ywcs); DEALLOC(h_zyx); DEALLOC(h_header);
    return ok;
}

}  // extern "C"
