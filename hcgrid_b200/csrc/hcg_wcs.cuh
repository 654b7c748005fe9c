// SIN (orthographic) pixel -> celestial coordinates, shared by the host
// (hcg_header_coords) and the device (hcg_target_from_header). FITS linear
// transformation then the zenithal SIN deprojection and native-to-celestial
// rotation of Calabretta & Greisen (2002), "Paper II" (eqs. 2, 59-60 with
// xi = eta = 0, and 2 for the rotation); degrees in and out, longitude
// normalised to [0, 360). Outside the projection (r > 1) gives NaN.
#pragma once

#include <math.h>

#include "hcg_math.cuh"

namespace hcg {

constexpr double kWcsD2R = 0x1.1df46a2529d39p-6;
constexpr double kWcsR2D = 0x1.ca5dc1a63c1f8p+5;

struct SinWcs {
    double crpix1, crpix2;
    double cdelt[2];
    double pc[2][2];
    double ap, sdp, cdp, pp;  // CRVAL1 (rad), sin/cos CRVAL2, LONPOLE (rad)
};

HCG_HD void sin_pix2world(const SinWcs &w, double p1, double p2, double &lon, double &lat) {
    double q1 = p1 - w.crpix1, q2 = p2 - w.crpix2;
    double x = w.cdelt[0] * (w.pc[0][0] * q1 + w.pc[0][1] * q2);
    double y = w.cdelt[1] * (w.pc[1][0] * q1 + w.pc[1][1] * q2);
    double r = sqrt(x * x + y * y) * kWcsD2R;
    if (r > 1.0) {
        lon = lat = NAN;
        return;
    }
    double phi = (r == 0.0) ? 0.0 : atan2(x, -y);
    double ct = r, st = sqrt((1.0 - r) * (1.0 + r));  // cos, sin of the native latitude
    double dphi = phi - w.pp;
    double cd = cos(dphi);
    double sdelta = st * w.sdp + ct * w.cdp * cd;
    double yv = -ct * sin(dphi);
    double xv = st * w.cdp - ct * w.sdp * cd;
    double a = fmod((w.ap + atan2(yv, xv)) * kWcsR2D, 360.0);
    if (a < 0) a += 360.0;
    lon = a;
    lat = atan2(sdelta, sqrt(xv * xv + yv * yv)) * kWcsR2D;  // (xv, yv) = cos(delta) (cos, sin) of d-alpha
}

}  // namespace hcg
