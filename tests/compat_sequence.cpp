// A driver written against the reference's lower-level names, called in the
// order of the reference's own solve_gridding (HCGrid/gridding.cu:484-556),
// linked against hcgrid_b200. After each step it dumps the globals the
// reference leaves behind, as raw arrays in <dumpdir>/<name>.bin, for
// tests/test_gpu_compat.py to compare with the reference's golden vectors.
//
//   compat_sequence infile tarfile outfile sortfile dumpdir sigma_deg
//                   sphere_radius_deg hpx_max_res_deg factor
#include <stdio.h>
#include <stdlib.h>
#include <string>

#include "hcgrid.h"

static std::string g_dir;

template <class T>
static void dump(const char *name, const T *p, size_t n) {
    FILE *f = fopen((g_dir + "/" + name + ".bin").c_str(), "wb");
    if (!f || fwrite(p, sizeof(T), n, f) != n) {
        fprintf(stderr, "dump %s failed\n", name);
        exit(2);
    }
    fclose(f);
}

int main(int argc, char **argv) {
    if (argc != 10) {
        fprintf(stderr, "usage: compat_sequence in tar out sort dumpdir sigma r res factor\n");
        return 2;
    }
    g_dir = argv[5];
    _Healpix_init(1, 2);
    double *kp = (double *)calloc(3, sizeof(double));
    kp[0] = atof(argv[6]);
    _prepare_grid_kernel(1, kp, atof(argv[7]), atof(argv[8]));
    h_GMaps.factor = (uint32_t)atoi(argv[9]);
    const double setup[4] = {kp[0], h_GMaps.disc_size, h_GMaps.sphere_radius, h_Healpix._resolution};
    dump("setup", setup, 4);
    const uint64_t hp[2] = {h_Healpix._nside, h_Healpix._npix};
    dump("healpix", hp, 2);

    read_input_map(argv[1]);
    const uint32_t n = h_GMaps.data_shape, nchan = h_GMaps.spec_dim;
    dump("in_lons", h_lons, n);
    read_output_map(argv[2]);
    dump("zyx", h_zyx, 3);
    if (set_WCS() != 1) return 3;
    const size_t P = (size_t)h_zyx[1] * h_zyx[2];
    dump("xwcs", h_xwcs, P);
    dump("ywcs", h_ywcs, P);
    init_output();
    init_input_with_cpu(2);
    dump("hpx_idx", h_hpx_idx, (size_t)n + 1);
    dump("start_ring", h_start_ring, (size_t)h_Healpix.usedrings + 1);
    const uint64_t rings[2] = {h_Healpix.firstring, h_Healpix.usedrings};
    dump("rings", rings, 2);
    dump("sorted_lons", h_lons, n);
    dump("sorted_lats", h_lats, n);
    dump("sorted_data", h_data, (size_t)n * nchan);
    data_alloc();
    data_h2d();
    data_d2h();
    dump("datacube", h_datacube, P * h_zyx[0]);
    dump("weightscube", h_weightscube, P * h_zyx[0]);
    write_output_map(argv[3]);
    write_ordered_map(argv[1], argv[4]);
    data_free();
    // data_free releases every host array, the retained kernel_params included
    if (h_lons || h_lats || h_data || h_hpx_idx || h_start_ring || h_datacube || h_weightscube || h_header ||
        h_zyx || h_kernel_params)
        return 4;
    return 0;
}
