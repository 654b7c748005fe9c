// Reference-named C++ entry points (include/hcgrid.h) over the C ABI: the
// free functions and global host arrays of HCGrid/gmap.h and gridding.h,
// with the reference's contents at each step of its call sequence
// (HCGrid/gridding.cu:484-556), backed by one default context.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include <string>
#include <vector>

#include "hcgrid.h"

extern "C" {
hcg_status hcg_fits_read_samples(const char *path, uint64_t *n, uint32_t *nchan, double *lon, double *lat,
                                 float *values);
hcg_status hcg_fits_read_header(const char *path, char *header, size_t cap, size_t *len);
hcg_status hcg_fits_write_cube(const char *path, const char *target_header, size_t len, uint32_t nx, uint32_t ny,
                               uint32_t nchan, const float *cube, const float *weights, int bitpix);
hcg_status hcg_fits_write_samples(const char *path, uint64_t n, uint32_t nchan, const double *lon,
                                  const double *lat, const float *values);
}

// ------------------------------------------------------------------ globals
// HCGrid/gmap.cpp:39-61 and healpix.cu:39
Healpix h_Healpix = {};
GMaps h_GMaps = {0, 1, 0, 0, 0, 0.0, 0.0, false};
double *h_lons = nullptr;
double *h_lats = nullptr;
double *h_data = nullptr;
double *h_weights = nullptr;
uint64_t *h_hpx_idx = nullptr;
uint32_t *h_start_ring = nullptr;
char *h_header = nullptr;
uint32_t *h_zyx = nullptr;
double *h_xwcs = nullptr;
double *h_ywcs = nullptr;
double *h_datacube = nullptr;
double *h_weightscube = nullptr;
double *h_kernel_params = nullptr;
double last_sphere_radius = -1;
double last_hpxmaxres = -1;

namespace {

hcg_context *g_ctx = nullptr;

// The device side of the sequence: the field made by init_input_*, the
// target made by data_alloc, the permutation that sorted the host arrays.
struct Session {
    hcg_field *field = nullptr;
    hcg_target *target = nullptr;
    std::vector<uint32_t> perm;
    uint32_t nx = 0, ny = 0;
    bool uploaded = false;
    double kernel_ms = 0.0;
} g_s;

double now_ms() {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec * 1e3 + tv.tv_usec * 1e-3;
}

[[noreturn]] void die(const char *what, hcg_status s) {
    fprintf(stderr, "%s: %s (%s)\n", what, hcg_status_string(s), g_ctx ? hcg_last_error(g_ctx) : "");
    exit(EXIT_FAILURE);
}

void check(hcg_status s, const char *what) {
    if (s != HCG_OK) die(what, s);
}

template <class T>
T *alloc(size_t n) {
    T *p = (T *)malloc((n ? n : 1) * sizeof(T));
    if (!p) {
        fprintf(stderr, "malloc() failed\n");
        exit(EXIT_FAILURE);
    }
    return p;
}

template <class T>
void release(T *&p) {
    free(p);
    p = nullptr;
}

// _update_params (HCGrid/healpix.cu:52-65)
void healpix_from_nside(uint64_t nside) {
    h_Healpix._nside = nside;
    uint64_t order = 0;
    for (uint64_t v = nside; v > 1; v >>= 1) ++order;
    h_Healpix._order = ((1ull << order) == nside) ? order : (uint64_t)-1;
    h_Healpix._nrings = 4 * nside - 1;
    h_Healpix._max_npix_per_ring = 4 * nside;
    h_Healpix._npface = nside * nside;
    h_Healpix._ncap = (h_Healpix._npface - nside) << 1;
    h_Healpix._npix = 12 * h_Healpix._npface;
    h_Healpix._fact2 = 4. / h_Healpix._npix;
    h_Healpix._fact1 = (nside << 1) * h_Healpix._fact2;
    h_Healpix._omega = 4. * 3.1415926535897932384626433832 / h_Healpix._npix;
    h_Healpix._resolution = sqrt(h_Healpix._omega);
}

// integer value of a header card ("KEY     =    value")
bool card_int(const char *hdr, size_t len, const char *key, long &v) {
    const size_t kl = strlen(key);
    for (size_t o = 0; o + 80 <= len; o += 80) {
        if (strncmp(hdr + o, key, kl) == 0 && (kl == 8 || hdr[o + kl] == ' ') && hdr[o + 8] == '=') {
            v = strtol(hdr + o + 10, nullptr, 10);
            return true;
        }
    }
    return false;
}

}  // namespace

extern "C" hcg_context *hcg_default_context() {
    if (!g_ctx) {
        const char *d = getenv("HCG_DEVICE");
        check(hcg_context_create(d ? atoi(d) : 0, nullptr, &g_ctx), "hcg_context_create");
    }
    return g_ctx;
}

void _Healpix_init(uint64_t nside, uint32_t scheme) {
    if (scheme != 2 || nside == 0) {  // RING = 2 (HCGrid/constants.h:73)
        fprintf(stderr, "_Healpix_init: only the RING scheme is supported\n");
        exit(1);
    }
    h_Healpix._scheme = scheme;
    h_Healpix._params_dirty = true;
    healpix_from_nside(nside);
}

void _prepare_grid_kernel(uint32_t kernel_type, double *kernel_params, double sphere_radius, double hpx_max_res) {
    hcg_context *ctx = hcg_default_context();
    check(hcg_prepare_grid_kernel(ctx, kernel_type, kernel_params, sphere_radius, hpx_max_res),
          "_prepare_grid_kernel");
    hcg_info inf;
    check(hcg_get_info(ctx, nullptr, &inf), "_prepare_grid_kernel");
    if (fabs(last_sphere_radius - sphere_radius) > 3e-5 || fabs(last_hpxmaxres - hpx_max_res) > 3e-5) {
        healpix_from_nside(inf.nside);
        last_sphere_radius = sphere_radius;
        last_hpxmaxres = hpx_max_res;
    }
    h_GMaps.kernel_type = kernel_type;
    h_GMaps.bearing_needed = kernel_type == HCG_GAUSS2D;
    h_GMaps.sphere_radius = sphere_radius;
    h_GMaps.disc_size = inf.disc_size;
    h_kernel_params = kernel_params;  // retained, released by data_free as in the reference
}

void read_input_map(const char *infile) {
    uint64_t n = 0;
    uint32_t nchan = 0;
    check(hcg_fits_read_samples(infile, &n, &nchan, nullptr, nullptr, nullptr), "read_input_map");
    std::vector<float> vals((size_t)n * nchan);
    h_lons = alloc<double>(n);
    h_lats = alloc<double>(n);
    check(hcg_fits_read_samples(infile, &n, &nchan, h_lons, h_lats, vals.data()), "read_input_map");
    h_GMaps.data_shape = (uint32_t)n;
    h_GMaps.spec_dim = nchan;
    h_data = alloc<double>(vals.size());
    for (size_t i = 0; i < vals.size(); ++i) h_data[i] = vals[i];  // float32 on disk: exact
    h_weights = alloc<double>(vals.size());
    for (size_t i = 0; i < vals.size(); ++i) h_weights[i] = 1.;
}

void read_output_map(const char *infile) {
    size_t len = 0;
    check(hcg_fits_read_header(infile, nullptr, 0, &len), "read_output_map");
    h_header = alloc<char>(len + 1);
    check(hcg_fits_read_header(infile, h_header, len + 1, &len), "read_output_map");
    long naxes = 0, v[3] = {1, 1, 1};
    if (!card_int(h_header, len, "NAXIS", naxes) || naxes < 2 || naxes > 3 || !card_int(h_header, len, "NAXIS1", v[0]) ||
        !card_int(h_header, len, "NAXIS2", v[1]) || (naxes == 3 && !card_int(h_header, len, "NAXIS3", v[2]))) {
        fprintf(stderr, "read_output_map: %s needs NAXIS 2 or 3 with NAXISn cards\n", infile);
        exit(EXIT_FAILURE);
    }
    h_zyx = alloc<uint32_t>(3);
    h_zyx[0] = (uint32_t)v[2];
    h_zyx[1] = (uint32_t)v[1];
    h_zyx[2] = (uint32_t)v[0];
    const uint32_t f = h_GMaps.factor ? h_GMaps.factor : 1;
    h_GMaps.block_warp_num = (h_zyx[1] - 1) / (32 * f) + 1;
}

int set_WCS() {
    if (!h_header || !h_zyx) return 0;
    const size_t len = strlen(h_header);
    uint32_t nx = 0, ny = 0;
    if (hcg_header_coords(h_header, len, &nx, &ny, nullptr, nullptr) != HCG_OK) return 0;
    h_xwcs = alloc<double>((size_t)nx * ny);
    h_ywcs = alloc<double>((size_t)nx * ny);
    if (hcg_header_coords(h_header, len, &nx, &ny, h_xwcs, h_ywcs) != HCG_OK) return 0;
    g_s.nx = nx;
    g_s.ny = ny;
    return 1;
}

void init_output() {
    const size_t num = (size_t)h_zyx[0] * h_zyx[1] * h_zyx[2];
    h_datacube = alloc<double>(num);
    h_weightscube = alloc<double>(num);
    for (size_t i = 0; i < num; ++i) h_datacube[i] = h_weightscube[i] = 0.;
}

// init_input_with_cpu / _thrust: the sort runs on the device; the host
// arrays are then left as the reference leaves them (gridding.cu:93-136):
// h_hpx_idx sorted with the npix sentinel, h_lons/h_lats/h_data in sorted
// order, h_start_ring and h_Healpix.firstring/usedrings set.
static void init_input_device() {
    const double t0 = now_ms();
    hcg_context *ctx = hcg_default_context();
    const uint64_t n = h_GMaps.data_shape;
    const uint32_t nchan = h_GMaps.spec_dim ? h_GMaps.spec_dim : 1;
    if (g_s.field) hcg_field_destroy(g_s.field);
    g_s.field = nullptr;
    check(hcg_field_create(ctx, n, h_lons, h_lats, h_weights, HCG_MEM_HOST, &g_s.field), "init_input");
    hcg_info inf;
    check(hcg_get_info(ctx, g_s.field, &inf), "init_input");
    h_hpx_idx = alloc<uint64_t>(n + 1);
    h_start_ring = alloc<uint32_t>(inf.usedrings + 1);
    g_s.perm.assign(n, 0);
    check(hcg_field_sorted(g_s.field, h_hpx_idx, g_s.perm.data(), h_start_ring), "init_input");
    h_Healpix.firstring = inf.firstring;
    h_Healpix.usedrings = inf.usedrings;
    std::vector<double> tmp(n);
    for (uint64_t i = 0; i < n; ++i) tmp[i] = h_lons[g_s.perm[i]];
    memcpy(h_lons, tmp.data(), n * sizeof(double));
    for (uint64_t i = 0; i < n; ++i) tmp[i] = h_lats[g_s.perm[i]];
    memcpy(h_lats, tmp.data(), n * sizeof(double));
    for (uint32_t c = 0; c < nchan; ++c) {
        double *d = h_data + (size_t)c * n;
        for (uint64_t i = 0; i < n; ++i) tmp[i] = d[g_s.perm[i]];
        memcpy(d, tmp.data(), n * sizeof(double));
    }
    g_s.uploaded = false;
    printf("%f, ", now_ms() - t0);  // the reference prints its pre-sort time (gridding.cu:145)
}

void init_input_with_cpu(const int &sort_param) {
    (void)sort_param;
    init_input_device();
}

void init_input_with_thrust(const int &sort_param) {
    (void)sort_param;
    init_input_device();
}

void data_alloc() {
    hcg_context *ctx = hcg_default_context();
    if (g_s.target) hcg_target_destroy(g_s.target);
    g_s.target = nullptr;
    check(hcg_target_create(ctx, g_s.nx, g_s.ny, h_xwcs, h_ywcs, HCG_MEM_HOST, &g_s.target), "data_alloc");
}

// The spectra as they are in h_data now (sorted order), back in input order
// for the field, which permutes them on the device.
void data_h2d() {
    const uint64_t n = h_GMaps.data_shape;
    const uint32_t nchan = h_GMaps.spec_dim ? h_GMaps.spec_dim : 1;
    std::vector<float> vals((size_t)n * nchan);
    for (uint32_t c = 0; c < nchan; ++c)
        for (uint64_t i = 0; i < n; ++i) vals[(size_t)c * n + g_s.perm[i]] = (float)h_data[(size_t)c * n + i];
    check(hcg_field_set_spectra(g_s.field, nchan, vals.data(), HCG_LAYOUT_CHANNEL_MAJOR, HCG_MEM_HOST), "data_h2d");
    g_s.uploaded = true;
}

// Grids on the device (the reference's hcgrid<<<>>> launch) and leaves the
// sums as the reference's kernel does: h_datacube = sum(w x) per channel
// plane, h_weightscube = sum(w) (unnormalised; write_output_map divides).
void data_d2h() {
    hcg_context *ctx = hcg_default_context();
    if (!g_s.uploaded) data_h2d();
    const uint32_t nchan = h_GMaps.spec_dim ? h_GMaps.spec_dim : 1;
    const size_t P = (size_t)g_s.nx * g_s.ny;
    std::vector<float> cube(P * nchan), wts(P);
    check(hcg_set_coarsening_factor(ctx, h_GMaps.factor ? h_GMaps.factor : 1), "hcgrid");
    check(hcg_grid(ctx, g_s.field, g_s.target, cube.data(), HCG_LAYOUT_CHANNEL_MAJOR, wts.data(), HCG_MEM_HOST,
                   HCG_ENGINE_AUTO),
          "hcgrid");
    hcg_stats st;
    check(hcg_get_stats(ctx, &st), "hcgrid");
    g_s.kernel_ms = st.ms_total;
    const uint32_t planes = h_zyx[0] < nchan ? h_zyx[0] : nchan;
    for (uint32_t c = 0; c < planes; ++c)
        for (size_t p = 0; p < P; ++p) {
            const double w = wts[p];
            h_weightscube[(size_t)c * P + p] = w;
            h_datacube[(size_t)c * P + p] = w != 0.0 ? (double)cube[(size_t)c * P + p] * w : 0.0;
        }
}

void write_output_map(const char *outfile) {
    const uint32_t nchan = h_zyx[0];
    const size_t P = (size_t)g_s.nx * g_s.ny;
    std::vector<float> cube(P * nchan), wts(P);
    for (size_t i = 0; i < P * nchan; ++i) {
        h_datacube[i] /= h_weightscube[i];  // 0/0 -> NaN for empty pixels, as the reference
        cube[i] = (float)h_datacube[i];
    }
    for (size_t p = 0; p < P; ++p) wts[p] = (float)h_weightscube[p];
    const char *ww = getenv("HCG_WRITE_WEIGHTS");
    check(hcg_fits_write_cube(outfile, h_header, strlen(h_header), g_s.nx, g_s.ny, nchan, cube.data(),
                              (ww && atoi(ww)) ? wts.data() : nullptr, -64),
          "write_output_map");
}

void write_ordered_map(const char *infile, const char *outfile) {
    (void)infile;  // the reference copies infile's headers; the layout written here is the same
    const uint64_t n = h_GMaps.data_shape;
    const uint32_t nchan = h_GMaps.spec_dim ? h_GMaps.spec_dim : 1;
    std::vector<float> vals((size_t)n * nchan);
    for (size_t i = 0; i < vals.size(); ++i) vals[i] = (float)h_data[i];
    check(hcg_fits_write_samples(outfile, n, nchan, h_lons, h_lats, vals.data()), "write_ordered_map");
}

void data_free() {
    release(h_lons);
    release(h_lats);
    release(h_data);
    release(h_weights);
    release(h_xwcs);
    release(h_ywcs);
    release(h_datacube);
    release(h_weightscube);
    release(h_hpx_idx);
    release(h_start_ring);
    release(h_header);
    release(h_zyx);
    release(h_kernel_params);
    if (g_s.target) hcg_target_destroy(g_s.target);
    if (g_s.field) hcg_field_destroy(g_s.field);
    g_s = Session();
}

void solve_gridding(const char *infile, const char *tarfile, const char *outfile, const char *sortfile,
                    const int &param, const int &bDim) {
    (void)bDim;
    const double t0 = now_ms();
    read_input_map(infile);
    read_output_map(tarfile);
    if (!set_WCS()) {
        fprintf(stderr, "set_WCS: %s is not a RA---SIN/DEC--SIN target\n", tarfile);
        exit(EXIT_FAILURE);
    }
    init_output();
    if (param == 3)  // THRUST (HCGrid/constants.h:63)
        init_input_with_thrust(param);
    else
        init_input_with_cpu(param);
    data_alloc();
    data_h2d();
    printf("h_zyx[1]=%u, h_zyx[2]=%u, ", h_zyx[1], h_zyx[2]);
    data_d2h();
    printf("kernel elapsed time=%f, ", g_s.kernel_ms);
    write_output_map(outfile);
    if (sortfile) write_ordered_map(infile, sortfile);
    data_free();
    printf("solving_gridding time=%f\n", now_ms() - t0);
}

void solve_gridding(const char *infile, const char *tarfile, const char *outfile, const char *sortfile,
                    const int &param, const int &bDim, int argc, char **argv) {
    (void)tarfile; (void)outfile; (void)sortfile; (void)param; (void)bDim; (void)argc; (void)argv;
    fprintf(stderr, "solve_gridding: HDF5 input (%s) needs libhdf5, which this build does not include (%s)\n",
            infile, hcg_status_string(HCG_EUNSUPPORTED));
    exit(EXIT_FAILURE);
}
