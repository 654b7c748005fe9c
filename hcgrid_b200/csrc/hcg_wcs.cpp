// Target pixel centres from a FITS header: the part of the reference's
// read_output_map + set_WCS (HCGrid/gmap.cpp:151-250, wcslib wcspih/wcsp2s)
// that the gridding path needs. Implements the FITS linear transformation
// (CRPIX, PCi_j or CDi_j, CDELT) followed by the zenithal SIN projection and
// the native-to-celestial rotation of Calabretta & Greisen (2002), "Paper II",
// for RA---SIN/DEC--SIN (and GLON/GLAT, ELON/ELAT) axes. Pixel (xx+1, yy+1)
// is evaluated for xx < NAXIS1, yy < NAXIS2, stored at yy*NAXIS1 + xx, as
// set_WCS does. Points outside the projection come out as NaN.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <string>
#include <vector>

#include "hcg_internal.h"
#include "hcg_wcs.cuh"

namespace hcg {
namespace {

std::map<std::string, std::string> parse_cards(const char *hdr, size_t len) {
    std::map<std::string, std::string> kv;
    for (size_t off = 0; off + 80 <= len || (off < len && len - off >= 8); off += 80) {
        std::string card(hdr + off, std::min<size_t>(80, len - off));
        std::string key = card.substr(0, std::min<size_t>(8, card.size()));
        while (!key.empty() && key.back() == ' ') key.pop_back();
        if (key == "END") break;
        if (card.size() < 10 || card[8] != '=' || card[9] != ' ') continue;
        std::string v = card.substr(10);
        size_t i = v.find_first_not_of(' ');
        if (i == std::string::npos) continue;
        v = v.substr(i);
        if (v[0] == '\'') {
            size_t j = v.find('\'', 1);
            v = v.substr(1, j == std::string::npos ? std::string::npos : j - 1);
            while (!v.empty() && v.back() == ' ') v.pop_back();
        } else {
            size_t j = v.find('/');
            if (j != std::string::npos) v = v.substr(0, j);
            while (!v.empty() && v.back() == ' ') v.pop_back();
        }
        kv[key] = v;
    }
    return kv;
}

double num(const std::map<std::string, std::string> &kv, const char *k, double dflt, bool &have) {
    auto it = kv.find(k);
    if (it == kv.end()) { have = false; return dflt; }
    have = true;
    return strtod(it->second.c_str(), nullptr);
}

}  // namespace

int parse_sin_header(const char *header, size_t len, uint32_t &nx, uint32_t &ny, SinWcs &w, std::string &why) {
    auto kv = parse_cards(header, len);
    bool h;
    nx = (uint32_t)num(kv, "NAXIS1", 0, h);
    if (!h) { why = "NAXIS1 missing"; return HCG_EINVAL; }
    ny = (uint32_t)num(kv, "NAXIS2", 0, h);
    if (!h) { why = "NAXIS2 missing"; return HCG_EINVAL; }
    std::string t1 = kv.count("CTYPE1") ? kv["CTYPE1"] : "", t2 = kv.count("CTYPE2") ? kv["CTYPE2"] : "";
    if (t1.size() < 8 || t2.size() < 8 || t1.substr(4, 4) != "-SIN" || t2.substr(4, 4) != "-SIN") {
        why = "only SIN projections are supported (CTYPE1='" + t1 + "', CTYPE2='" + t2 + "')";
        return HCG_EUNSUPPORTED;
    }
    w.crpix1 = num(kv, "CRPIX1", 0, h);
    w.crpix2 = num(kv, "CRPIX2", 0, h);
    double crval1 = num(kv, "CRVAL1", 0, h), crval2 = num(kv, "CRVAL2", 0, h);
    w.pc[0][0] = 1; w.pc[0][1] = 0; w.pc[1][0] = 0; w.pc[1][1] = 1;
    w.cdelt[0] = w.cdelt[1] = 1;
    bool hc;
    num(kv, "CD1_1", 0, hc);
    if (hc) {
        w.pc[0][0] = num(kv, "CD1_1", 0, h); w.pc[0][1] = num(kv, "CD1_2", 0, h);
        w.pc[1][0] = num(kv, "CD2_1", 0, h); w.pc[1][1] = num(kv, "CD2_2", 0, h);
    } else {
        w.cdelt[0] = num(kv, "CDELT1", 1, h);
        w.cdelt[1] = num(kv, "CDELT2", 1, h);
        w.pc[0][0] = num(kv, "PC1_1", 1, h); w.pc[0][1] = num(kv, "PC1_2", 0, h);
        w.pc[1][0] = num(kv, "PC2_1", 0, h); w.pc[1][1] = num(kv, "PC2_2", 1, h);
    }
    bool hxi, heta;
    double xi = num(kv, "PV2_1", 0, hxi), eta = num(kv, "PV2_2", 0, heta);
    if ((hxi && xi != 0.0) || (heta && eta != 0.0)) { why = "SIN with PV2_1/PV2_2 (slant) is not supported"; return HCG_EUNSUPPORTED; }
    // Zenithal projection: (phi0, theta0) = (0, 90), so the celestial pole of
    // the native frame is the reference point; LONPOLE defaults to 180 deg
    // when CRVAL2 < 90 (Paper II, sec. 2.5).
    double lonpole = num(kv, "LONPOLE", crval2 < 90.0 ? 180.0 : 0.0, h);
    w.ap = crval1 * kWcsD2R;
    w.sdp = sin(crval2 * kWcsD2R);
    w.cdp = cos(crval2 * kWcsD2R);
    w.pp = lonpole * kWcsD2R;
    return HCG_OK;
}

int sin_target_coords(const char *header, size_t len, uint32_t &nx, uint32_t &ny, std::vector<double> &X,
                      std::vector<double> &Y, std::string &why) {
    SinWcs w;
    int st = parse_sin_header(header, len, nx, ny, w, why);
    if (st != HCG_OK) return st;
    X.resize((size_t)nx * ny);
    Y.resize((size_t)nx * ny);
    for (uint32_t yy = 0; yy < ny; ++yy)
        for (uint32_t xx = 0; xx < nx; ++xx) {
            size_t o = (size_t)yy * nx + xx;
            sin_pix2world(w, xx + 1.0, yy + 1.0, X[o], Y[o]);
        }
    return HCG_OK;
}

}  // namespace hcg
