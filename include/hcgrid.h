/*
 * Reference-compatible C++ entry points over the C ABI (hcgrid_c.h).
 *
 * Existing HCGrid driver code links against these unchanged: the same names,
 * signatures, argument meaning and global variables as the reference, backed
 * by a default context on CUDA device 0 (HCG_DEVICE overrides). As in the
 * reference, a failure prints a message and exits; callers that want status
 * codes use hcgrid_c.h directly. The declarations sit behind the
 * reference's own include guards, so a driver compiled against the
 * reference's headers (HCGrid/gmap.h, gridding.h, healpix.h) links to the
 * same symbols.
 *
 *   _Healpix_init, h_Healpix     HCGrid/healpix.h:16-26, healpix.cu:42-65
 *   _prepare_grid_kernel         HCGrid/gmap.h:121, gmap.cpp:64-99
 *   read_input_map               HCGrid/gmap.h:124, gmap.cpp:102-148
 *   read_output_map              HCGrid/gmap.h:127, gmap.cpp:151-180
 *   set_WCS                      HCGrid/gmap.h:130, gmap.cpp:183-250
 *   write_output_map             HCGrid/gmap.h:133, gmap.cpp:253-323
 *   write_ordered_map            HCGrid/gmap.h:136, gmap.cpp:326-379
 *   init_input_with_cpu/_thrust  HCGrid/gridding.h:53-60, gridding.cu:70-216
 *   init_output                  HCGrid/gridding.h:63, gridding.cu:219-227
 *   data_alloc/h2d/d2h/free      HCGrid/gridding.h:87-96, gridding.cu:406-481
 *   solve_gridding               HCGrid/gridding.h:99, gridding.cu:484-556
 *   h_* globals                  HCGrid/gmap.h:47-107, gmap.cpp:39-61
 *   solve_gridding (+argc, argv) HCGrid+/gridding.h:99 (HDF5 input): reports
 *                                that HDF5 is unsupported in this build and
 *                                exits.
 *
 * The sequence is the reference's: read_input_map, read_output_map,
 * set_WCS, init_output, init_input_with_cpu (the on-device stable sort; the
 * sorted keys, ring table and sorted host arrays come back into h_hpx_idx,
 * h_start_ring, h_lons, h_lats, h_data as the reference leaves them),
 * data_alloc, data_h2d, then data_d2h, which grids on the device (the
 * reference's `hcgrid<<<>>>` launch, a __global__ function a host-compiled
 * driver cannot launch itself) and fills h_datacube with the unnormalised
 * sums and h_weightscube with the weight sums, as the reference's kernel
 * leaves them; write_output_map normalises in place and writes, and
 * data_free releases everything (the retained kernel_params array
 * included). Differences, all supersets of the reference's behaviour: every
 * channel of a multi-channel input is sorted and gridded (the reference
 * sorts and grids channel 0 only), the output map is written with
 * NAXIS1 = nx and NAXIS2 = ny for any shape (the reference swaps them,
 * which only matters for non-square maps), and h_GMaps.factor > 1 is
 * honoured by the reference-compatible coarsening of the device kernel.
 */
#ifndef HCGRID_COMPAT_H
#define HCGRID_COMPAT_H

#include <stdint.h>

#include "hcgrid_c.h"

#ifndef HEALPIX_H
/* HCGrid/healpix.h:16-23, same member layout. */
struct Healpix {
    uint64_t _nside, _order, _nrings, usedrings, firstring;
    uint64_t _max_npix_per_ring;
    uint64_t _npface, _ncap, _npix;
    double _fact1, _fact2, _resolution, _omega;
    uint32_t _scheme;
    bool _params_dirty;
};
extern Healpix h_Healpix;
/* RING only (the reference fails on NESTED). _prepare_grid_kernel sets the
 * optimal nside afterwards, as in the reference. */
void _Healpix_init(uint64_t nside, uint32_t scheme);
#endif

#ifndef GMAP_H
/* HCGrid/gmap.h:47-61, same member layout. The driver sets `factor` (its
 * coarsening factor) before solve_gridding (HCGrid/HCGrid.cpp:156-161). */
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

/* Host arrays with the reference's contents at each step (malloc'd by the
 * library, released by data_free). h_data is [spec_dim][data_shape]. */
extern double *h_lons;
extern double *h_lats;
extern double *h_data;
extern double *h_weights;
extern uint64_t *h_hpx_idx;    /* sorted keys + npix sentinel (init_input_*) */
extern uint32_t *h_start_ring; /* ring lookup table, usedrings + 1 entries */
extern char *h_header;         /* target header cards (read_output_map) */
extern uint32_t *h_zyx;        /* NAXIS3, NAXIS2, NAXIS1 of the target */
extern double *h_xwcs;
extern double *h_ywcs;
extern double *h_datacube;     /* [z][ny][nx]: sums, normalised by write_output_map */
extern double *h_weightscube;
extern double *h_kernel_params; /* the caller's array, retained by _prepare_grid_kernel */
extern double last_sphere_radius;
extern double last_hpxmaxres;

/* Kernel and HEALPix setup; kernel_params[0] (sigma, deg) becomes
 * 0.5/sigma^2 in place for GAUSS1D. */
void _prepare_grid_kernel(uint32_t kernel_type, double *kernel_params, double sphere_radius, double hpx_max_res);
void read_input_map(const char *infile);
void read_output_map(const char *infile);
int set_WCS(); /* 1 ok, 0 failure (unsupported projection) */
void write_output_map(const char *infile);
void write_ordered_map(const char *infile, const char *outfile);
#endif

#ifndef SORTGRID_H
/* sort_param is HCGrid's order_arg; the device sort is always the stable
 * order of order_arg 2 (block_indirect_sort may order equal keys
 * differently; nothing else depends on it). */
void init_input_with_cpu(const int &sort_param);
void init_input_with_thrust(const int &sort_param);
void init_output();
void data_alloc();
void data_h2d();
void data_d2h();
void data_free();
/* Read infile (values + lon/lat HDUs) and tarfile (target header), grid on
 * the device, write outfile; sortfile (may be NULL) receives the samples in
 * sorted order. bDim is a tuning hint. A WEIGHTS image extension is added
 * when HCG_WRITE_WEIGHTS=1. */
void solve_gridding(const char *infile, const char *tarfile, const char *outfile, const char *sortfile,
                    const int &param, const int &bDim);
void solve_gridding(const char *infile, const char *tarfile, const char *outfile, const char *sortfile,
                    const int &param, const int &bDim, int argc, char **argv);
#endif

/* The context the functions above use (created on first use). */
extern "C" hcg_context *hcg_default_context();

#endif
