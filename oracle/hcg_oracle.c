/*
 * CPU restatement of HCGrid's gridding path -- TEST INFRASTRUCTURE ONLY.
 *
 * The checker for the CUDA path (see hcg_oracle.h). Restates, in plain C
 * with the host libm, the reference's HEALPix RING functions
 * (HCGrid/healpix.cu), numeric helpers (HCGrid/helpers.cu), kernel setup
 * (HCGrid/gmap.cpp:64-99), pre-sort and ring lookup table
 * (HCGrid/gridding.cu:70-136) and the `hcgrid` kernel body
 * (HCGrid/gridding.cu:277-403) in FP64. Built with -ffp-contract=off so
 * every product and sum rounds separately, as on x86-64 without FMA.
 *
 * Pinned against the reference's own code compiled for the host
 * (oracle/_ref) by tests/test_oracle_vs_ref.py and against the golden
 * vectors in tests/golden/.
 */
#include "hcg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Same numeric constants as constants.h:75-84 (value-for-value; the
 * window and ring arithmetic must round identically). */
#define PI (3.1415926535897932384626433832)
#define TWOTHIRD (2.0 / 3.0)
#define HALFPI (PI / 2.)
#define INV_HALFPI (1. / HALFPI)
#define NORTH_B (20)
#define SOUTH_B (160)
#define DEG2RAD (PI / 180.)
#define RAD2DEG (180. / PI)

/* helpers.cu:40-64 -- floor(log2(arg)), 0 for arg == 0. */
uint64_t orc_ilog2(uint64_t arg) {
    uint64_t r = 0;
    while (arg > 1) { arg >>= 1; ++r; }
    return r;
}

/* helpers.cu:67-69 */
uint64_t orc_isqrt(uint64_t arg) { return (uint64_t)sqrt((double)arg + 0.5); }

/* helpers.cu:83-95 */
double orc_fmodulo(double v1, double v2) {
    if (v1 >= 0) return (v1 < v2) ? v1 : fmod(v1, v2);
    double tmp = fmod(v1, v2) + v2;
    return (tmp == v2) ? 0. : tmp;
}

/* helpers.cu:98-102 (the reference shifts an int; nside stays < 2^31). */
uint64_t orc_set_optimal_nside(double target_res) {
    uint64_t nside = (uint64_t)(sqrt(PI / 3.) / target_res + 0.5);
    return 1ULL << (orc_ilog2(nside) + 1);
}

/* helpers.cu:105-114 */
uint64_t orc_nside_to_order(uint64_t nside) {
    if (nside == 0) return ORC_MAX_Y;
    if (nside & (nside - 1)) return (uint64_t)-1;
    return orc_ilog2(nside);
}

/* healpix.cu:42-65 */
void orc_healpix_init(orc_healpix *h, uint64_t nside) {
    h->nside = nside;
    h->order = orc_nside_to_order(nside);
    h->nrings = 4 * nside - 1;
    h->npface = nside * nside;
    h->ncap = (h->npface - nside) << 1;
    h->npix = 12 * h->npface;
    h->fact2 = 4. / h->npix;
    h->fact1 = (nside << 1) * h->fact2;
    h->omega = 4. * PI / h->npix;
    h->resolution = sqrt(h->omega);
}

/* healpix.cu:87-105 */
void orc_ring_info(const orc_healpix *h, uint64_t ring, uint64_t *startpix, uint64_t *npr, int *shifted) {
    if (ring < h->nside) {
        *shifted = 1;
        *npr = 4 * ring;
        *startpix = 2 * ring * (ring - 1);
    } else if (ring < 3 * h->nside) {
        *shifted = ((ring - h->nside) & 1) == 0;
        *npr = 4 * h->nside;
        *startpix = h->ncap + (ring - h->nside) * *npr;
    } else {
        uint64_t nr = 4 * h->nside - ring;
        *shifted = 1;
        *npr = 4 * nr;
        *startpix = h->npix - 2 * nr * (nr + 1);
    }
}

/* healpix.cu:116-123 */
uint64_t orc_pix2ring(const orc_healpix *h, uint64_t pix) {
    if (pix < h->ncap) return (1 + orc_isqrt(1 + 2 * pix)) >> 1;
    if (pix < h->npix - h->ncap) return (pix - h->ncap) / (4 * h->nside) + h->nside;
    return 4 * h->nside - ((1 + orc_isqrt(2 * (h->npix - pix) - 1)) >> 1);
}

/* healpix.cu:166-205 */
uint64_t orc_loc2pix(const orc_healpix *h, double z, double phi, double sth, int have_sth) {
    double za = fabs(z);
    double tt = orc_fmodulo(phi * INV_HALFPI, 4.0);
    if (za <= TWOTHIRD) {
        uint64_t nl4 = 4 * h->nside;
        double temp1 = h->nside * (0.5 + tt);
        double temp2 = h->nside * z * 0.75;
        uint64_t jp = (uint64_t)(temp1 - temp2);
        uint64_t jm = (uint64_t)(temp1 + temp2);
        uint64_t ir = h->nside + 1 + jp - jm;
        uint64_t kshift = 1 - (ir & 1);
        uint64_t t1 = jp + jm + kshift + 1 + nl4 + nl4 - h->nside;
        uint64_t ip = (h->order > 0) ? ((t1 >> 1) & (nl4 - 1)) : ((t1 >> 1) % nl4);
        return h->ncap + (ir - 1) * nl4 + ip;
    } else {
        double tp = tt - (double)((uint64_t)tt);
        double tmp;
        if ((za < 0.99) || (!have_sth))
            tmp = h->nside * sqrt(3. * (1. - za));
        else
            tmp = h->nside * sth / sqrt((1. + za) / 3.);
        uint64_t jp = (uint64_t)(tp * tmp);
        uint64_t jm = (uint64_t)((1.0 - tp) * tmp);
        uint64_t ir = jp + jm + 1;
        uint64_t ip = (uint64_t)(tt * ir);
        if (z > 0) return 2 * ir * (ir - 1) + ip;
        return h->npix - 2 * ir * (ir + 1) + ip;
    }
}

/* healpix.cu:217-224 */
uint64_t orc_ang2pix(const orc_healpix *h, double theta, double phi) {
    if (!(theta >= 0 && theta <= PI)) return ORC_MAX_Y;
    if ((theta < 0.01) || (theta > PI - 0.01)) return orc_loc2pix(h, cos(theta), phi, sin(theta), 1);
    return orc_loc2pix(h, cos(theta), phi, 0., 0);
}

/* healpix.cu:274-320 */
void orc_pix2loc(const orc_healpix *h, uint64_t pix, double *z, double *phi, double *sth, int *have_sth) {
    *have_sth = 0;
    if (pix < h->ncap) {
        uint64_t iring = (1 + orc_isqrt(1 + 2 * pix)) >> 1;
        uint64_t iphi = (pix + 1) - 2 * iring * (iring - 1);
        double tmp = (iring * iring) * h->fact2;
        *z = 1.0 - tmp;
        if (*z > 0.99) { *sth = sqrt(tmp * (2. - tmp)); *have_sth = 1; }
        *phi = (iphi - 0.5) * HALFPI / iring;
    } else if (pix < h->npix - h->ncap) {
        uint64_t ip = pix - h->ncap;
        uint64_t itmp = ip >> (h->order + 2); /* order is unsigned: the >= 0 branch is always taken */
        uint64_t nl4 = 4 * h->nside;
        uint64_t iring = itmp + h->nside;
        uint64_t iphi = ip - nl4 * itmp + 1;
        double fodd = (((iring + h->nside) & 1) > 0) ? 1.0 : 0.5;
        *z = (2. * h->nside - iring) * h->fact1;
        *phi = (iphi - fodd) * PI * 0.75 * h->fact1;
    } else {
        uint64_t ip = h->npix - pix;
        uint64_t iring = (1 + orc_isqrt(2 * ip - 1)) >> 1;
        uint64_t iphi = 4 * iring + 1 - (ip - 2 * iring * (iring - 1));
        double tmp = (iring * iring) * h->fact2;
        *z = tmp - 1.0;
        if (*z < -0.99) { *sth = sqrt(tmp * (2. - tmp)); *have_sth = 1; }
        *phi = (iphi - 0.5) * HALFPI / iring;
    }
}

/* healpix.cu:336-348 */
void orc_pix2ang(const orc_healpix *h, uint64_t pix, double *theta, double *phi) {
    double z, sth = 0.0;
    int have;
    orc_pix2loc(h, pix, &z, phi, &sth, &have);
    *theta = have ? atan2(sth, z) : acos(z);
}

/* gmap.cpp:64-99. The reference only rebuilds HEALPix when sphere_radius or
 * hpx_max_res moved by more than 3e-5 since the last call; a fresh state
 * (hpx.nside == 0) always builds. */
int orc_prepare_grid_kernel(orc_gmaps *g, uint32_t kernel_type, double *params, double sphere_radius,
                            double hpx_max_res) {
    static double last_r = -1, last_res = -1;
    const int taper_fix = (kernel_type & ORC_TAPER_FIX) != 0;
    kernel_type &= ~ORC_TAPER_FIX;
    if (taper_fix && kernel_type != ORC_TAPERED_SINC) return -1;
    g->taper_fix = taper_fix;
    if (kernel_type == ORC_GAUSS1D) {
        params[0] = 0.5 / pow(params[0], 2.);
        g->bearing_needed = 0;
    } else if (kernel_type == ORC_GAUSS2D) {
        g->bearing_needed = 1;
    } else if (kernel_type == ORC_TAPERED_SINC) {
        g->bearing_needed = 0;
    } else {
        return -1;
    }
    g->kernel_type = kernel_type;
    memcpy(g->params, params, 3 * sizeof(double));
    if (g->hpx.nside == 0 || fabs(last_r - sphere_radius) > 3e-5 || fabs(last_res - hpx_max_res) > 3e-5) {
        orc_healpix_init(&g->hpx, orc_set_optimal_nside(DEG2RAD * hpx_max_res));
        last_r = sphere_radius;
        last_res = hpx_max_res;
    }
    g->sphere_radius = sphere_radius;
    g->disc_size = (DEG2RAD * sphere_radius + g->hpx.resolution);
    return 0;
}

/* gridding.cu:77-82 */
void orc_sample_keys(const orc_healpix *h, long n, const double *lons, const double *lats, uint64_t *keys) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        double theta = HALFPI - DEG2RAD * lats[i];
        double phi = DEG2RAD * lons[i];
        keys[i] = orc_ang2pix(h, theta, phi);
    }
}

static const uint64_t *g_sort_keys;
static int cmp_stable(const void *a, const void *b) {
    uint32_t i = *(const uint32_t *)a, j = *(const uint32_t *)b;
    if (g_sort_keys[i] < g_sort_keys[j]) return -1;
    if (g_sort_keys[i] > g_sort_keys[j]) return 1;
    return (i < j) ? -1 : (i > j);
}

/* gridding.cu:84-92 with order_arg 2 (boost parallel_stable_sort): order by
 * key, equal keys in input order. */
void orc_stable_sort(long n, const uint64_t *keys, uint64_t *sorted_keys, uint32_t *perm) {
    for (long i = 0; i < n; ++i) perm[i] = (uint32_t)i;
    g_sort_keys = keys;
    qsort(perm, (size_t)n, sizeof(uint32_t), cmp_stable);
    for (long i = 0; i < n; ++i) sorted_keys[i] = keys[perm[i]];
}

/* gridding.cu:260-275 (unsigned arithmetic kept: left may wrap). */
static uint32_t search_last_less(const uint64_t *values, uint32_t left, uint32_t right, uint64_t key) {
    if (right <= left) return right;
    uint32_t low = left, mid, up = right - 1;
    while (low < up) {
        mid = low + ((up - low + 1) >> 1);
        if (values[mid] < key)
            low = mid;
        else
            up = mid - 1;
    }
    return (values[low] < key) ? low : right;
}

/* gridding.cu:118-136. Returns the number of LUT entries (usedrings + 1),
 * or -1 when lut_cap is too small. */
long orc_ring_lut(const orc_healpix *h, long n, const uint64_t *sorted_keys, uint64_t *firstring,
                  uint64_t *usedrings, uint32_t *lut, long lut_cap) {
    uint64_t first = orc_pix2ring(h, sorted_keys[0]);
    uint32_t count = (uint32_t)(1 + orc_pix2ring(h, sorted_keys[n - 1]) - first);
    *firstring = first;
    *usedrings = count;
    if ((long)count + 1 > lut_cap) return -1;
    lut[0] = 0;
    uint32_t ring_idx = 0;
    for (uint64_t k = 1; k < count; ++k) {
        uint64_t startpix, npr;
        int shifted;
        orc_ring_info(h, k + first, &startpix, &npr, &shifted);
        uint32_t c = search_last_less(sorted_keys, ring_idx, (uint32_t)n, startpix);
        if (c == (uint32_t)n) c = ring_idx - 1;
        ring_idx = c + 1;
        lut[k] = ring_idx;
    }
    lut[count] = (uint32_t)n;
    return (long)count + 1;
}

/* helpers.cu:128-130 */
static double true_angular_distance(double l1, double b1, double l2, double b2) {
    return 2 * asin(sqrt(pow(sin((b1 - b2) / 2.), 2) + cos(b1) * cos(b2) * pow(sin((l1 - l2) / 2.), 2)));
}

/* helpers.cu:133-137: great-circle bearing of (l2, b2) seen from (l1, b1),
 * radians. */
static double great_circle_bearing(double l1, double b1, double l2, double b2) {
    double l_diff = l2 - l1;
    double cos_b2 = cos(b2);
    return atan2(cos_b2 * sin(l_diff), cos(b1) * sin(b2) - sin(b1) * cos_b2 * cos(l_diff));
}

/* gridding.cu:229-235 */
static double sinc(double x) { return fabs(x) < 1.e-10 ? 1. : sin(x) / x; }

/* gridding.cu:237-257: the grid kernel at `distance` degrees and `bearing`
 * radians. GAUSS1D takes the transformed 0.5 / sigma^2; GAUSS2D
 * (sigma_maj, sigma_min, PA) and TAPERED_SINC (sigma, a, b) take their
 * parameters as given. The reference's taper is exp(pow(-(arg / a), 2)) =
 * exp(+(arg / a)^2); taper_fix takes exp(-(arg / a)^2). */
static double kernel_func(const orc_gmaps *g, double distance, double bearing) {
    const double *p = g->params;
    if (g->kernel_type == ORC_GAUSS1D) return exp(-distance * distance * p[0]);
    if (g->kernel_type == ORC_GAUSS2D) {
        double ellarg = pow(p[0], 2.0) * pow(sin(bearing - p[2]), 2.0) + pow(p[1], 2.0) * pow(cos(bearing - p[2]), 2.0);
        double Earg = pow(distance / p[0] / p[1], 2.0) / 2. * ellarg;
        return exp(-Earg);
    }
    double arg = PI * distance / p[0];
    double t = pow(-(arg / p[1]), 2.0);
    return sinc(arg / p[2]) * exp(g->taper_fix ? -t : t);
}

typedef struct {
    uint64_t uring, dring;
    double l1, b1, disc_theta, disc_phi;
    int polar;
} pixel_setup;

/* gridding.cu:298-323 */
static void setup_pixel(const orc_gmaps *g, uint64_t firstring, uint64_t usedrings, double xw, double yw,
                        pixel_setup *ps) {
    const orc_healpix *h = &g->hpx;
    ps->l1 = xw * DEG2RAD;
    ps->b1 = yw * DEG2RAD;
    double disc_theta = HALFPI - ps->b1;
    double disc_phi = ps->l1;
    double utheta = disc_theta - g->disc_size;
    if (utheta * RAD2DEG < 0) utheta = 0;
    uint64_t uring = orc_pix2ring(h, orc_ang2pix(h, utheta, disc_phi));
    if (uring < firstring) uring = firstring;
    utheta = disc_theta + g->disc_size;
    uint64_t dring = orc_pix2ring(h, orc_ang2pix(h, utheta, disc_phi));
    if (dring >= firstring + usedrings) dring = firstring + usedrings - 1;
    ps->uring = uring;
    ps->dring = dring;
    ps->disc_theta = disc_theta;
    ps->disc_phi = disc_phi;
    ps->polar = (disc_theta * RAD2DEG <= NORTH_B || disc_theta * RAD2DEG >= SOUTH_B);
}

/* gridding.cu:329-367 for one ring: the [lo, hi) candidate interval the
 * kernel walks. Returns 0 for a normal ring, 1 for the ring that the
 * reference would spin on forever (lpix/rpix outside the ring: A3). */
static int ring_window(const orc_gmaps *g, long n, const uint64_t *keys, const uint32_t *lut, uint64_t firstring,
                       const pixel_setup *ps, uint64_t uring, uint32_t *lo, uint32_t *hi) {
    const orc_healpix *h = &g->hpx;
    uint32_t start_int = lut[uring - firstring];
    uint32_t end_int = lut[uring - firstring + 1];
    uint64_t startpix, npr;
    int shifted;
    orc_ring_info(h, uring, &startpix, &npr, &shifted);
    double utheta, uphi;
    orc_pix2ang(h, startpix, &utheta, &uphi);
    uint64_t lpix = orc_ang2pix(h, utheta, ps->disc_phi - g->disc_size);
    if (ps->polar) lpix = startpix;
    *lo = *hi = start_int;
    if (!(lpix >= startpix && lpix < startpix + npr)) return 1;
    uint64_t rpix = orc_ang2pix(h, utheta, ps->disc_phi + g->disc_size);
    if (ps->polar) rpix = startpix + npr - 1;
    if (!(rpix >= startpix && rpix < startpix + npr)) return 1;
    uint32_t idx = search_last_less(keys, start_int - 1, end_int, lpix) + 1;
    if (idx > end_int) idx = (uint32_t)n;
    uint32_t j = idx;
    while (j < (uint32_t)n && !(keys[j] > rpix)) ++j;
    *lo = idx;
    *hi = j;
    return 0;
}

long orc_pixel_windows(const orc_gmaps *g, long n, const uint64_t *sorted_keys, const uint32_t *lut,
                       uint64_t firstring, uint64_t usedrings, double xwcs, double ywcs, uint64_t *uring,
                       uint64_t *dring, uint32_t *lo, uint32_t *hi, long cap, long *a3) {
    pixel_setup ps;
    setup_pixel(g, firstring, usedrings, xwcs, ywcs, &ps);
    *uring = ps.uring;
    *dring = ps.dring;
    *a3 = 0;
    long k = 0;
    for (uint64_t r = ps.uring; r <= ps.dring; ++r, ++k) {
        if (k >= cap) return -1;
        *a3 += ring_window(g, n, sorted_keys, lut, firstring, &ps, r, &lo[k], &hi[k]);
    }
    return k;
}

static double hav(double x) { double s = sin(x / 2.); return s * s; }

void orc_grid(const orc_gmaps *g, long n, const uint64_t *sorted_keys, const uint32_t *lut, uint64_t firstring,
              uint64_t usedrings, const double *lons, const double *lats, const double *weights, const double *data,
              long nchan, long npix_map, const double *xwcs, const double *ywcs, int mode, double *cube_out,
              double *wts_out, orc_stats *stats) {
    orc_grid_ex(g, n, sorted_keys, lut, firstring, usedrings, lons, lats, weights, data, nchan, npix_map, xwcs, ywcs,
                mode, cube_out, wts_out, NULL, stats);
}

void orc_grid_ex(const orc_gmaps *g, long n, const uint64_t *sorted_keys, const uint32_t *lut, uint64_t firstring,
                 uint64_t usedrings, const double *lons, const double *lats, const double *weights,
                 const double *data, long nchan, long npix_map, const double *xwcs, const double *ywcs, int mode,
                 double *cube_out, double *wts_out, double *wabs_out, orc_stats *stats) {
    const orc_healpix *h = &g->hpx;
    long long visited = 0, within = 0, a3 = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : visited, within, a3)
    for (long p = 0; p < npix_map; ++p) {
        double *acc = cube_out + p * nchan;
        double wsum = 0.0, wabs = 0.0;
        for (long c = 0; c < nchan; ++c) acc[c] = 0.0;
        pixel_setup ps;
        setup_pixel(g, firstring, usedrings, xwcs[p], ywcs[p], &ps);
        if (mode == 0) {
            for (uint64_t r = ps.uring; r <= ps.dring; ++r) {
                uint32_t lo, hi;
                if (ring_window(g, n, sorted_keys, lut, firstring, &ps, r, &lo, &hi)) { ++a3; continue; }
                for (uint32_t i = lo; i < hi; ++i) {
                    double l2 = lons[i] * DEG2RAD;
                    double b2 = lats[i] * DEG2RAD;
                    double sdist = true_angular_distance(ps.l1, ps.b1, l2, b2) * RAD2DEG;
                    double sbear = g->bearing_needed ? great_circle_bearing(ps.l1, ps.b1, l2, b2) : 0.;
                    ++visited;
                    if (sdist < g->sphere_radius) {
                        double tweight = weights[i] * kernel_func(g, sdist, sbear);
                        const double *x = data + (long)i * nchan;
                        for (long c = 0; c < nchan; ++c) acc[c] += x[c] * tweight;
                        wsum += tweight;
                        wabs += fabs(tweight);
                        ++within;
                    }
                }
            }
        } else {
            /* Exact disc: every sample of every ring that can hold a point
             * within sphere_radius, pre-filtered by the haversine bound
             * hav(dl) <= hav(r) / (cos b1 cos b2). */
            double r = g->sphere_radius * DEG2RAD;
            double rr = r + h->resolution;
            double th0 = ps.disc_theta - rr, th1 = ps.disc_theta + rr;
            uint64_t r0 = orc_pix2ring(h, orc_ang2pix(h, th0 < 0 ? 0 : th0, 0.0));
            uint64_t r1 = orc_pix2ring(h, orc_ang2pix(h, th1 > PI ? PI : th1, 0.0));
            if (r0 < firstring) r0 = firstring;
            if (r1 >= firstring + usedrings) r1 = firstring + usedrings - 1;
            double cbmin = fmin(sin(th0 < 0 ? 0 : th0), sin(th1 > PI ? PI : th1));
            if (th0 <= HALFPI && th1 >= HALFPI) cbmin = fmin(cbmin, 1.0);
            double cb1 = cos(ps.b1);
            double limit = (cbmin > 1e-6 && cb1 > 1e-6) ? hav(r) / (cbmin * cb1) * 1.000001 + 1e-300 : 2.0;
            for (uint64_t ring = r0; ring <= r1 && r0 <= r1; ++ring) {
                uint32_t lo = lut[ring - firstring], hi = lut[ring - firstring + 1];
                for (uint32_t i = lo; i < hi; ++i) {
                    double l2 = lons[i] * DEG2RAD;
                    double b2 = lats[i] * DEG2RAD;
                    if (limit < 1.0 && hav(ps.l1 - l2) > limit) continue;
                    double sdist = true_angular_distance(ps.l1, ps.b1, l2, b2) * RAD2DEG;
                    double sbear = g->bearing_needed ? great_circle_bearing(ps.l1, ps.b1, l2, b2) : 0.;
                    ++visited;
                    if (sdist < g->sphere_radius) {
                        double tweight = weights[i] * kernel_func(g, sdist, sbear);
                        const double *x = data + (long)i * nchan;
                        for (long c = 0; c < nchan; ++c) acc[c] += x[c] * tweight;
                        wsum += tweight;
                        wabs += fabs(tweight);
                        ++within;
                    }
                }
            }
        }
        wts_out[p] = wsum;
        if (wabs_out) wabs_out[p] = wabs;
    }
    if (stats) {
        stats->pairs_visited = visited;
        stats->pairs_within = within;
        stats->a3_events = a3;
    }
}

void orc_normalize(long npix_map, long nchan, const double *cube, const double *wts, double *out) {
    for (long p = 0; p < npix_map; ++p)
        for (long c = 0; c < nchan; ++c) out[p * nchan + c] = cube[p * nchan + c] / wts[p];
}

/* Bulk forms for the tests. */
void orc_ang2pix_many(const orc_healpix *h, long n, const double *theta, const double *phi, uint64_t *out) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) out[i] = orc_ang2pix(h, theta[i], phi[i]);
}
void orc_pix2ring_many(const orc_healpix *h, long n, const uint64_t *pix, uint64_t *out) {
    for (long i = 0; i < n; ++i) out[i] = orc_pix2ring(h, pix[i]);
}
void orc_pix2ang_many(const orc_healpix *h, long n, const uint64_t *pix, double *theta, double *phi) {
    for (long i = 0; i < n; ++i) orc_pix2ang(h, pix[i], &theta[i], &phi[i]);
}
void orc_ring_info_many(const orc_healpix *h, long n, const uint64_t *ring, uint64_t *startpix, uint64_t *npr) {
    for (long i = 0; i < n; ++i) {
        int s;
        orc_ring_info(h, ring[i], &startpix[i], &npr[i], &s);
    }
}
