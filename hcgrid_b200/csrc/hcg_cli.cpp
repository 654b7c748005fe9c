// Command line with the reference's flags (HCGrid/HCGrid.cpp:38-197):
//   --fits_path --input_file --target_file --output_file --sorted_file
//   --fits_id --beam_size --order_arg --block_num --register_num --sp_num
//   --coarsening_factor
// File names are <fits_path><name><fits_id>.fits with the output written in
// cfitsio's overwrite mode, as the reference builds them. The kernel is
// GAUSS1D with sigma = FWHM / sqrt(8 ln 2) (FWHM = --beam_size arcsec,
// default 300), sphere_radius = 5 sigma and hpx_max_res = sigma / 2
// (HCGrid.cpp:141-151). --block_num, --register_num and --sp_num are the
// reference's launch-shape hints and are accepted; --coarsening_factor (1-3)
// sets h_GMaps.factor, which groups pixels as the reference's kernel does.
// --sphere_sigmas N changes the 5-sigma radius (e.g. 3 for the README's form).
#include <getopt.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>

#include "hcgrid.h"

int main(int argc, char **argv) {
    const char *path = "", *ifile = nullptr, *tfile = nullptr, *ofile = nullptr, *sfile = nullptr, *num = "",
               *beam = nullptr, *order = "2", *bdim = nullptr, *factor = nullptr, *nsig = nullptr;
    static const struct option opts[] = {
        {"helparg", no_argument, nullptr, 'h'},          {"fits_path", required_argument, nullptr, 'p'},
        {"input_file", required_argument, nullptr, 'i'}, {"target_file", required_argument, nullptr, 't'},
        {"output_file", required_argument, nullptr, 'o'}, {"sorted_file", required_argument, nullptr, 's'},
        {"fits_id", required_argument, nullptr, 'n'},    {"beam_size", required_argument, nullptr, 'b'},
        {"order_arg", required_argument, nullptr, 'd'},  {"block_num", required_argument, nullptr, 'a'},
        {"register_num", required_argument, nullptr, 'r'}, {"sp_num", required_argument, nullptr, 'm'},
        {"coarsening_factor", required_argument, nullptr, 'f'}, {"sphere_sigmas", required_argument, nullptr, 'g'},
        {nullptr, 0, nullptr, 0}};
    int c, idx = 0;
    while ((c = getopt_long_only(argc, argv, "hp:i:t:o:s:n:b:d:a:", opts, &idx)) != -1) {
        switch (c) {
            case 'h':
                fprintf(stderr, "usage: HCGrid --fits_path <dir/> --input_file <name> --target_file <name> "
                                "--output_file <name> [--sorted_file <name>] --fits_id <n> [--beam_size <arcsec>] "
                                "[--order_arg <1-4>] [--block_num <n>] [--sphere_sigmas <k>]\n");
                return 1;
            case 'p': path = optarg; break;
            case 'i': ifile = optarg; break;
            case 't': tfile = optarg; break;
            case 'o': ofile = optarg; break;
            case 's': sfile = optarg; break;
            case 'n': num = optarg; break;
            case 'b': beam = optarg; break;
            case 'd': order = optarg; break;
            case 'a': bdim = optarg; break;
            case 'r': case 'm': break;
            case 'f': factor = optarg; break;
            case 'g': nsig = optarg; break;
            default: return 1;
        }
    }
    if (!ifile || !tfile || !ofile) {
        fprintf(stderr, "HCGrid: --input_file, --target_file and --output_file are required\n");
        return 1;
    }
    std::string in = std::string(path) + ifile + num + ".fits";
    std::string tar = std::string(path) + tfile + num + ".fits";
    std::string out = std::string("!") + path + ofile + num + ".fits";
    std::string sorted = sfile ? std::string("!") + path + sfile + num + ".fits" : "";
    double fwhm = (beam ? atoi(beam) : 300) / 3600.;
    double sigma = fwhm / sqrt(8 * log(2));
    _Healpix_init(1, 2);
    // heap-allocated as the reference's driver does: _prepare_grid_kernel
    // retains it and data_free releases it
    double *kp = (double *)calloc(3, sizeof(double));
    if (!kp) return 1;
    kp[0] = sigma;
    double k = nsig ? atof(nsig) : 5.0;
    _prepare_grid_kernel(HCG_GAUSS1D, kp, k * sigma, sigma / 2.);
    h_GMaps.factor = factor ? (uint32_t)atoi(factor) : 1;
    int ord = atoi(order), bd = bdim ? atoi(bdim) : 64;
    printf("order: %s, num: %s, ", order, num);
    solve_gridding(in.c_str(), tar.c_str(), out.c_str(), sfile ? sorted.c_str() : nullptr, ord, bd);
    return 0;
}
