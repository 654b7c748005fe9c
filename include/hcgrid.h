/*
 * Reference-compatible C++ entry points over the C ABI (hcgrid_c.h).
 *
 * Existing HCGrid driver code (HCGrid/HCGrid.cpp) links against these
 * unchanged: same names, signatures and argument meaning, backed by a
 * default context on CUDA device 0 (HCG_DEVICE overrides). As in the
 * reference, a failure prints a message and exits; callers that want
 * status codes use hcgrid_c.h directly.
 *
 *   _prepare_grid_kernel  HCGrid/gmap.h:121, HCGrid/gmap.cpp:64-99
 *   solve_gridding        HCGrid/gridding.h:99, HCGrid/gridding.cu:484-556
 *                         (FITS in, FITS out; the whole cube is written, plus
 *                         a WEIGHTS image extension when HCG_WRITE_WEIGHTS=1)
 *   solve_gridding (+argc, argv)
 *                         HCGrid+/gridding.h:99 (HDF5 input): reports that
 *                         HDF5 is unsupported in this build and exits.
 */
#ifndef HCGRID_COMPAT_H
#define HCGRID_COMPAT_H

#include <stdint.h>

#include "hcgrid_c.h"

/* The reference driver sets h_GMaps.factor (its coarsening factor) before
 * solve_gridding (HCGrid/HCGrid.cpp:156-161); same member layout as
 * HCGrid/gmap.h:47-61. Only `factor` is read (values > 1 are accepted and
 * every pixel keeps its own disc). Guarded so the reference's own gmap.h
 * can be used instead. */
#ifndef GMAP_H
class GMaps {
  public:
    uint32_t block_warp_num;
    uint32_t factor;
    uint32_t data_shape;
    uint32_t spec_dim;
    uint32_t kernel_type;
    double disc_size;
    double sphere_radius;
    bool bearing_needed;
};
extern GMaps h_GMaps;
/* HCGrid/healpix.h:26; RING only (the reference fails on NESTED). nside is
 * recomputed by _prepare_grid_kernel, as in the reference. */
void _Healpix_init(uint64_t nside, uint32_t scheme);
#endif

/* Kernel and HEALPix setup; kernel_params[0] (sigma, deg) becomes
 * 0.5/sigma^2 in place for GAUSS1D. */
void _prepare_grid_kernel(uint32_t kernel_type, double *kernel_params, double sphere_radius, double hpx_max_res);

/* Read infile (values + lon/lat HDUs) and tarfile (target header), grid on
 * the device, write outfile; sortfile (may be NULL) receives the samples in
 * sorted order. param is HCGrid's order_arg (the device sort is always the
 * stable order of order_arg 2); bDim is a tuning hint. */
void solve_gridding(const char *infile, const char *tarfile, const char *outfile, const char *sortfile,
                    const int &param, const int &bDim);
void solve_gridding(const char *infile, const char *tarfile, const char *outfile, const char *sortfile,
                    const int &param, const int &bDim, int argc, char **argv);

/* The context the two functions above use (created on first use). */
extern "C" hcg_context *hcg_default_context();

#endif
