// Reference-named C++ entry points (include/hcgrid.h) over the C ABI.
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

namespace {

hcg_context *g_ctx = nullptr;

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

}  // namespace

GMaps h_GMaps = {0, 1, 0, 0, 0, 0.0, 0.0, false};

void _Healpix_init(uint64_t nside, uint32_t scheme) {
    if (scheme != 2 || nside == 0) {  // RING = 2 (HCGrid/constants.h:73)
        fprintf(stderr, "_Healpix_init: only the RING scheme is supported\n");
        exit(1);
    }
}

extern "C" hcg_context *hcg_default_context() {
    if (!g_ctx) {
        const char *d = getenv("HCG_DEVICE");
        check(hcg_context_create(d ? atoi(d) : 0, nullptr, &g_ctx), "hcg_context_create");
    }
    return g_ctx;
}

void _prepare_grid_kernel(uint32_t kernel_type, double *kernel_params, double sphere_radius, double hpx_max_res) {
    check(hcg_prepare_grid_kernel(hcg_default_context(), kernel_type, kernel_params, sphere_radius, hpx_max_res),
          "_prepare_grid_kernel");
}

void solve_gridding(const char *infile, const char *tarfile, const char *outfile, const char *sortfile,
                    const int &param, const int &bDim) {
    (void)param;
    (void)bDim;
    double t0 = now_ms();
    hcg_context *ctx = hcg_default_context();
    uint64_t n = 0;
    uint32_t nchan = 0;
    check(hcg_fits_read_samples(infile, &n, &nchan, nullptr, nullptr, nullptr), "read_input_map");
    std::vector<double> lon(n), lat(n);
    std::vector<float> vals((size_t)n * nchan);
    check(hcg_fits_read_samples(infile, &n, &nchan, lon.data(), lat.data(), vals.data()), "read_input_map");
    size_t hlen = 0;
    check(hcg_fits_read_header(tarfile, nullptr, 0, &hlen), "read_output_map");
    std::string hdr(hlen + 1, '\0');
    check(hcg_fits_read_header(tarfile, &hdr[0], hdr.size(), &hlen), "read_output_map");
    double t1 = now_ms();
    hcg_field *f = nullptr;
    check(hcg_field_create(ctx, n, lon.data(), lat.data(), nullptr, HCG_MEM_HOST, &f), "init_input");
    check(hcg_field_set_spectra(f, nchan, vals.data(), HCG_LAYOUT_CHANNEL_MAJOR, HCG_MEM_HOST), "init_input");
    check(hcg_synchronize(ctx), "init_input");
    double t2 = now_ms();
    hcg_target *t = nullptr;
    check(hcg_target_from_header(ctx, hdr.data(), hlen, &t), "set_WCS");
    uint32_t nx = 0, ny = 0;
    check(hcg_target_coords(t, &nx, &ny, nullptr, nullptr), "set_WCS");
    std::vector<float> cube((size_t)nx * ny * nchan), wts((size_t)nx * ny);
    check(hcg_grid(ctx, f, t, cube.data(), HCG_LAYOUT_CHANNEL_MAJOR, wts.data(), HCG_MEM_HOST, HCG_ENGINE_AUTO),
          "hcgrid");
    hcg_stats st;
    check(hcg_get_stats(ctx, &st), "hcgrid");
    const char *ww = getenv("HCG_WRITE_WEIGHTS");
    check(hcg_fits_write_cube(outfile, hdr.data(), hlen, nx, ny, nchan, cube.data(),
                              (ww && atoi(ww)) ? wts.data() : nullptr, -64),
          "write_output_map");
    if (sortfile) {
        std::vector<uint32_t> perm(n);
        check(hcg_field_sorted(f, nullptr, perm.data(), nullptr), "write_ordered_map");
        std::vector<double> sl(n), sb(n);
        std::vector<float> sv((size_t)n * nchan);
        for (uint64_t i = 0; i < n; ++i) {
            sl[i] = lon[perm[i]];
            sb[i] = lat[perm[i]];
            for (uint32_t c = 0; c < nchan; ++c) sv[(size_t)c * n + i] = vals[(size_t)c * n + perm[i]];
        }
        check(hcg_fits_write_samples(sortfile, n, nchan, sl.data(), sb.data(), sv.data()), "write_ordered_map");
    }
    hcg_target_destroy(t);
    hcg_field_destroy(f);
    double t3 = now_ms();
    // the reference prints comma-separated timings (gridding.cu:145,534,555)
    printf("%f, h_zyx[1]=%u, h_zyx[2]=%u, kernel elapsed time=%f, solving_gridding time=%f\n", t2 - t1, ny, nx,
           st.ms_total, t3 - t0);
}

void solve_gridding(const char *infile, const char *tarfile, const char *outfile, const char *sortfile,
                    const int &param, const int &bDim, int argc, char **argv) {
    (void)tarfile; (void)outfile; (void)sortfile; (void)param; (void)bDim; (void)argc; (void)argv;
    fprintf(stderr, "solve_gridding: HDF5 input (%s) needs libhdf5, which this build does not include (%s)\n",
            infile, hcg_status_string(HCG_EUNSUPPORTED));
    exit(EXIT_FAILURE);
}
