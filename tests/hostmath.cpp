// Host build of the device HEALPix / correctly rounded cos header, so its
// arithmetic can be checked on CPU cores against the reference's host
// functions (via the oracle) and against quad precision. Compiled by
// tests/test_capi_cpu.py with -ffp-contract=off; the device build performs
// the same explicitly rounded operations.
#include <quadmath.h>
#include <stdint.h>

#include "hcg_math.cuh"

extern "C" {

void hm_ang2pix(uint64_t nside, long n, const double *theta, const double *phi, uint64_t *out, long *hard) {
    hcg::HpxParams h;
    h.nside = nside;
    uint64_t o = 0;
    while ((1ULL << (o + 1)) <= nside) ++o;
    h.order = o;
    uint64_t npface = nside * nside;
    h.ncap = (npface - nside) << 1;
    h.npix = 12 * npface;
    h.fact2 = 4. / h.npix;
    h.fact1 = (nside << 1) * h.fact2;
    h.resolution = 0;
    long hh = 0;
    for (long i = 0; i < n; ++i) {
        int hd;
        out[i] = hcg::ang2pix(h, theta[i], phi[i], hd);
        hh += hd;
    }
    *hard = hh;
}

// Counts of (cr != quad-rounded) for cos and sin, and of cr != libm cos.
void hm_cos_check(long n, const double *theta, long *bad_cos, long *bad_sin, long *diff_libm, long *hard) {
    long bc = 0, bs = 0, dl = 0, hh = 0;
    for (long i = 0; i < n; ++i) {
        double s, c;
        int hd;
        hcg::sincos_cr(theta[i], s, c, hd);
        hh += hd;
        if (c != (double)cosq((__float128)theta[i])) ++bc;
        if (s != (double)sinq((__float128)theta[i])) ++bs;
        if (c != cos(theta[i])) ++dl;
    }
    *bad_cos = bc;
    *bad_sin = bs;
    *diff_libm = dl;
    *hard = hh;
}
}
