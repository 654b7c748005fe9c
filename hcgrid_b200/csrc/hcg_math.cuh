// Exact-rounding HEALPix RING arithmetic and a correctly rounded sin/cos,
// shared by the device kernels and by a host build used to check them.
//
// Pixel indices must equal the reference's host results bit for bit
// (HCGrid/healpix.cu computed with x86-64 libm, no FMA). Every floating
// operation here is therefore an explicitly rounded IEEE operation
// (__dadd_rn, __dmul_rn, ... on the device; plain operators in a host
// translation unit built with -ffp-contract=off), so neither side can fuse
// a multiply into an add.
//
// cos(theta) is evaluated in double-double and rounded once: Cody-Waite
// reduction by a three-part pi/2 (Cody & Waite, "Software Manual for the
// Elementary Functions", 1980), Taylor series of sin and cos in Horner form
// on double-double operands (Dekker 1971 / Knuth two-sum, FMA two-product),
// and a Ziv-style rounding test (Ziv 1991) that counts the cases it cannot
// decide. Host libm's cos is not correctly rounded (about 0.14% of inputs in
// [0, pi] differ from the correctly rounded value by one ulp), so pixel
// indices agree with it except where such a one-ulp difference moves a
// point across a pixel boundary.
#pragma once

#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define HCG_HD __host__ __device__ __forceinline__
#else
#define HCG_HD static inline
#endif

namespace hcg {

// Values of constants.h:75-84 (PI, HALFPI, INV_HALFPI, TWOTHIRD, DEG2RAD,
// RAD2DEG) and of PI - 0.01 as used by ang2pix, as exact binary literals.
constexpr double kPi = 0x1.921fb54442d18p+1;
constexpr double kHalfPi = 0x1.921fb54442d18p+0;
constexpr double kInvHalfPi = 0x1.45f306dc9c883p-1;
constexpr double kTwoThird = 0x1.5555555555555p-1;
constexpr double kDeg2Rad = 0x1.1df46a2529d39p-6;
constexpr double kRad2Deg = 0x1.ca5dc1a63c1f8p+5;
constexpr double kPiMinus001 = 0x1.90d8072fc7f04p+1;
constexpr uint64_t kMaxY = 1073741824ULL;  // 2^30, the reference's invalid-theta pixel
constexpr double kNorthB = 20.0;            // polar full-ring bounds, degrees of theta
constexpr double kSouthB = 160.0;

#if defined(__CUDA_ARCH__)
HCG_HD double dadd(double a, double b) { return __dadd_rn(a, b); }
HCG_HD double dsub(double a, double b) { return __dsub_rn(a, b); }
HCG_HD double dmul(double a, double b) { return __dmul_rn(a, b); }
HCG_HD double ddiv(double a, double b) { return __ddiv_rn(a, b); }
HCG_HD double dsqrt(double a) { return __dsqrt_rn(a); }
HCG_HD double dfma(double a, double b, double c) { return __fma_rn(a, b, c); }
HCG_HD double u2d(uint64_t u) { return __ull2double_rn(u); }
HCG_HD uint64_t d2u(double d) { return __double2ull_rz(d); }
#else
HCG_HD double dadd(double a, double b) { return a + b; }
HCG_HD double dsub(double a, double b) { return a - b; }
HCG_HD double dmul(double a, double b) { return a * b; }
HCG_HD double ddiv(double a, double b) { return a / b; }
HCG_HD double dsqrt(double a) { return sqrt(a); }
HCG_HD double dfma(double a, double b, double c) { return fma(a, b, c); }
HCG_HD double u2d(uint64_t u) { return (double)u; }
HCG_HD uint64_t d2u(double d) { return (uint64_t)d; }
#endif

struct HpxParams {
    uint64_t nside, order, ncap, npix;
    double fact1, fact2, resolution;
};

// ---------------------------------------------------------------------------
// Double-double helpers.

HCG_HD void two_sum(double a, double b, double &s, double &e) {
    s = dadd(a, b);
    double bb = dsub(s, a);
    e = dadd(dsub(a, dsub(s, bb)), dsub(b, bb));
}
HCG_HD void fast_two_sum(double a, double b, double &s, double &e) {
    s = dadd(a, b);
    e = dsub(b, dsub(s, a));
}
HCG_HD void dd_add(double ah, double al, double bh, double bl, double &sh, double &sl) {
    double s, e, t, f;
    two_sum(ah, bh, s, e);
    two_sum(al, bl, t, f);
    e = dadd(e, t);
    fast_two_sum(s, e, s, e);
    e = dadd(e, f);
    fast_two_sum(s, e, sh, sl);
}
HCG_HD void dd_mul(double ah, double al, double bh, double bl, double &ph, double &pl) {
    double p = dmul(ah, bh);
    double e = dfma(ah, bh, -p);
    e = dfma(ah, bl, e);
    e = dfma(al, bh, e);
    fast_two_sum(p, e, ph, pl);
}

// (-1)^j / (2j)! and (-1)^j / (2j+1)! as double-double (exact rationals
// rounded to hi + lo), j = 0..14.
#define HCG_DD_COEFFS                                                                      \
    static const double kCos[15][2] = {{1.0, 0.0},                                         \
                                       {-0.5, 0.0},                                        \
                                       {0.041666666666666664, 2.3129646346357427e-18},     \
                                       {-0.001388888888888889, 5.300543954373577e-20},     \
                                       {2.48015873015873e-05, 2.1511947866775882e-23},     \
                                       {-2.755731922398589e-07, -2.3767714622250297e-23},  \
                                       {2.08767569878681e-09, -1.20734505911326e-25},      \
                                       {-1.1470745597729725e-11, -2.0655512752830745e-28}, \
                                       {4.779477332387385e-14, 4.399205485834081e-31},     \
                                       {-1.5619206968586225e-16, -1.1910679660273754e-32}, \
                                       {4.110317623312165e-19, 1.4412973378659527e-36},    \
                                       {-8.896791392450574e-22, 7.911402614872376e-38},    \
                                       {1.6117375710961184e-24, -3.6846573564509766e-41},  \
                                       {-2.4795962632247976e-27, 1.2953730964765229e-43},  \
                                       {3.279889237069838e-30, 1.5117542744029879e-46}};   \
    static const double kSin[15][2] = {{1.0, 0.0},                                         \
                                       {-0.16666666666666666, -9.25185853854297e-18},      \
                                       {0.008333333333333333, 1.1564823173178714e-19},     \
                                       {-0.0001984126984126984, -1.7209558293420705e-22},  \
                                       {2.7557319223985893e-06, -1.858393274046472e-22},   \
                                       {-2.505210838544172e-08, 1.448814070935912e-24},    \
                                       {1.6059043836821613e-10, 1.2585294588752098e-26},   \
                                       {-7.647163731819816e-13, -7.03872877733453e-30},    \
                                       {2.8114572543455206e-15, 1.6508842730861433e-31},   \
                                       {-8.22063524662433e-18, -2.2141894119604265e-34},   \
                                       {1.9572941063391263e-20, -1.3643503830087908e-36},  \
                                       {-3.868170170630684e-23, 8.843177655482344e-40},    \
                                       {6.446950284384474e-26, -1.9330404233703465e-42},   \
                                       {-9.183689863795546e-29, -1.4303150396787322e-45},  \
                                       {1.1309962886447716e-31, 1.0498015412959506e-47}};

// pi/2 = kPio2Hi + kPio2Mid + kPio2Lo to about 2^-163.
constexpr double kPio2Hi = 0x1.921fb54442d18p+0;
constexpr double kPio2Mid = 0x1.1a62633145c07p-54;
constexpr double kPio2Lo = -0x1.f1976b7ed8fbcp-110;

// Round a normalised double-double to double and report whether the
// rounding could not be decided (|lo| within 2^-99 |hi| of half an ulp).
HCG_HD double dd_round(double h, double l, int &hard) {
    double toward = (l >= 0) ? INFINITY : -INFINITY;
    double gap = dsub(nextafter(h, toward), h);
    double d = dsub(fabs(l), fabs(gap) * 0.5);
    hard = (l != 0.0) && (fabs(d) <= ldexp(fabs(h), -99));
    return h;
}

// sin and cos of theta in [0, pi], correctly rounded unless `hard` is set.
HCG_HD void sincos_cr(double theta, double &s, double &c, int &hard) {
    HCG_DD_COEFFS
    int k;
    double rh, rl;
    if (theta < 0x1.921fb54442d18p-1) {
        k = 0; rh = theta; rl = 0.0;
    } else if (theta < 0x1.2d97c7f3321d2p+1) {
        k = 1;
        dd_add(dsub(theta, kPio2Hi), 0.0, -kPio2Mid, -kPio2Lo, rh, rl);  // theta - kPio2Hi is exact
    } else {
        k = 2;
        dd_add(dsub(theta, 2.0 * kPio2Hi), 0.0, -2.0 * kPio2Mid, -2.0 * kPio2Lo, rh, rl);
    }
    double xh, xl;
    dd_mul(rh, rl, rh, rl, xh, xl);
    double ch = kCos[14][0], cl = kCos[14][1];
    double sh = kSin[14][0], sl = kSin[14][1];
    for (int j = 13; j >= 0; --j) {
        dd_mul(ch, cl, xh, xl, ch, cl);
        dd_add(ch, cl, kCos[j][0], kCos[j][1], ch, cl);
        dd_mul(sh, sl, xh, xl, sh, sl);
        dd_add(sh, sl, kSin[j][0], kSin[j][1], sh, sl);
    }
    dd_mul(sh, sl, rh, rl, sh, sl);  // sin r = r * S(r^2)
    double oc_h, oc_l, os_h, os_l;
    if (k == 0) { oc_h = ch; oc_l = cl; os_h = sh; os_l = sl; }
    else if (k == 1) { oc_h = -sh; oc_l = -sl; os_h = ch; os_l = cl; }
    else { oc_h = -ch; oc_l = -cl; os_h = -sh; os_l = -sl; }
    int h1, h2;
    c = dd_round(oc_h, oc_l, h1);
    s = dd_round(os_h, os_l, h2);
    hard = h1 | h2;
}

HCG_HD double cos_cr(double theta, int &hard) {
    double s, c;
    sincos_cr(theta, s, c, hard);
    return c;
}

// ---------------------------------------------------------------------------
// HEALPix RING functions, same arithmetic as HCGrid/healpix.cu and helpers.cu.

HCG_HD uint64_t isqrt(uint64_t arg) { return d2u(dsqrt(dadd(u2d(arg), 0.5))); }  // helpers.cu:67-69

HCG_HD double fmodulo(double v1, double v2) {  // helpers.cu:83-95
    if (v1 >= 0) return (v1 < v2) ? v1 : fmod(v1, v2);
    double tmp = dadd(fmod(v1, v2), v2);
    return (tmp == v2) ? 0. : tmp;
}

HCG_HD void ring_info(const HpxParams &h, uint64_t ring, uint64_t &startpix, uint64_t &npr) {  // healpix.cu:68-86
    if (ring < h.nside) {
        npr = 4 * ring;
        startpix = 2 * ring * (ring - 1);
    } else if (ring < 3 * h.nside) {
        npr = 4 * h.nside;
        startpix = h.ncap + (ring - h.nside) * npr;
    } else {
        uint64_t nr = 4 * h.nside - ring;
        npr = 4 * nr;
        startpix = h.npix - 2 * nr * (nr + 1);
    }
}

HCG_HD uint64_t pix2ring(const HpxParams &h, uint64_t pix) {  // healpix.cu:108-115
    if (pix < h.ncap) return (1 + isqrt(1 + 2 * pix)) >> 1;
    if (pix < h.npix - h.ncap) return (pix - h.ncap) / (4 * h.nside) + h.nside;
    return 4 * h.nside - ((1 + isqrt(2 * (h.npix - pix) - 1)) >> 1);
}

HCG_HD uint64_t loc2pix(const HpxParams &h, double z, double phi, double sth, bool have_sth) {  // healpix.cu:126-165
    double za = fabs(z);
    double tt = fmodulo(dmul(phi, kInvHalfPi), 4.0);
    double ns = u2d(h.nside);
    if (za <= kTwoThird) {
        uint64_t nl4 = 4 * h.nside;
        double temp1 = dmul(ns, dadd(0.5, tt));
        double temp2 = dmul(dmul(ns, z), 0.75);
        uint64_t jp = d2u(dsub(temp1, temp2));
        uint64_t jm = d2u(dadd(temp1, temp2));
        uint64_t ir = h.nside + 1 + jp - jm;
        uint64_t kshift = 1 - (ir & 1);
        uint64_t t1 = jp + jm + kshift + 1 + nl4 + nl4 - h.nside;
        uint64_t ip = (h.order > 0) ? ((t1 >> 1) & (nl4 - 1)) : ((t1 >> 1) % nl4);
        return h.ncap + (ir - 1) * nl4 + ip;
    }
    double tp = dsub(tt, u2d(d2u(tt)));
    double tmp;
    if ((za < 0.99) || (!have_sth))
        tmp = dmul(ns, dsqrt(dmul(3., dsub(1., za))));
    else
        tmp = ddiv(dmul(ns, sth), dsqrt(ddiv(dadd(1., za), 3.)));
    uint64_t jp = d2u(dmul(tp, tmp));
    uint64_t jm = d2u(dmul(dsub(1.0, tp), tmp));
    uint64_t ir = jp + jm + 1;
    uint64_t ip = d2u(dmul(tt, u2d(ir)));
    if (z > 0) return 2 * ir * (ir - 1) + ip;
    return h.npix - 2 * ir * (ir + 1) + ip;
}

// healpix.cu:208-216, with the correctly rounded cos/sin.
HCG_HD uint64_t ang2pix(const HpxParams &h, double theta, double phi, int &hard) {
    hard = 0;
    if (!(theta >= 0 && theta <= kPi)) return kMaxY;
    double s, c;
    sincos_cr(theta, s, c, hard);
    if ((theta < 0.01) || (theta > kPiMinus001)) return loc2pix(h, c, phi, s, true);
    return loc2pix(h, c, phi, 0., false);
}

// healpix.cu:227-273: location of a pixel centre (z, phi, sin theta).
HCG_HD void pix2loc(const HpxParams &h, uint64_t pix, double &z, double &phi, double &sth, bool &have_sth) {
    have_sth = false;
    sth = 0.0;
    if (pix < h.ncap) {
        uint64_t iring = (1 + isqrt(1 + 2 * pix)) >> 1;
        uint64_t iphi = (pix + 1) - 2 * iring * (iring - 1);
        double tmp = dmul(u2d(iring * iring), h.fact2);
        z = dsub(1.0, tmp);
        if (z > 0.99) { sth = dsqrt(dmul(tmp, dsub(2., tmp))); have_sth = true; }
        phi = ddiv(dmul(dsub(u2d(iphi), 0.5), kHalfPi), u2d(iring));
    } else if (pix < h.npix - h.ncap) {
        uint64_t nl4 = 4 * h.nside;
        uint64_t ip = pix - h.ncap;
        uint64_t itmp = ip >> (h.order + 2);
        uint64_t iring = itmp + h.nside;
        uint64_t iphi = ip - nl4 * itmp + 1;
        double fodd = (((iring + h.nside) & 1) > 0) ? 1.0 : 0.5;
        z = dmul(dsub(dmul(2., u2d(h.nside)), u2d(iring)), h.fact1);
        phi = dmul(dmul(dmul(dsub(u2d(iphi), fodd), kPi), 0.75), h.fact1);
    } else {
        uint64_t ip = h.npix - pix;
        uint64_t iring = (1 + isqrt(2 * ip - 1)) >> 1;
        uint64_t iphi = 4 * iring + 1 - (ip - 2 * iring * (iring - 1));
        double tmp = dmul(u2d(iring * iring), h.fact2);
        z = dsub(tmp, 1.0);
        if (z < -0.99) { sth = dsqrt(dmul(tmp, dsub(2., tmp))); have_sth = true; }
        phi = ddiv(dmul(dsub(u2d(iphi), 0.5), kHalfPi), u2d(iring));
    }
}

}  // namespace hcg
