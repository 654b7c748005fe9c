// FITS input/output of the gridding path, host side.
//
// Formats follow the reference (HCGrid/gmap.cpp):
//   input map   read_input_map (102-148): primary HDU image NAXIS1 x NAXIS2
//               [x NAXIS3] holds the values (N = NAXIS1*NAXIS2 samples, channel
//               slowest); the second HDU image holds N longitudes followed by N
//               latitudes (degrees).
//   target      read_output_map (151-180): the primary header, NAXIS1/2/3.
//   output      write_output_map (253-323): an image whose header copies the
//               target's cards after the first six (SIMPLE ... NAXIS3), holding
//               the normalised map. Here the whole cube is written (HCGrid+
//               writes channel 0 only, HCGrid+/gmap.cpp:353-361) and, optionally,
//               the weight map as an IMAGE extension (the reference writes none).
// Data are big-endian; BITPIX 8/16/32/64/-32/-64 and BSCALE/BZERO are read.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "hcg_internal.h"

namespace {

constexpr size_t kBlock = 2880, kCard = 80;

struct Hdu {
    std::string header;  // cards up to and including END
    int bitpix = 0;
    std::vector<long long> naxes;
    double bscale = 1.0, bzero = 0.0;
    size_t data_off = 0;
    long long count() const {
        if (naxes.empty()) return 0;
        long long n = 1;
        for (long long a : naxes) n *= a;
        return n;
    }
};

bool card_value(const std::string &hdr, const char *key, std::string &out) {
    for (size_t o = 0; o + kCard <= hdr.size(); o += kCard) {
        std::string k = hdr.substr(o, 8);
        while (!k.empty() && k.back() == ' ') k.pop_back();
        if (k == "END") break;
        if (k != key || hdr[o + 8] != '=') continue;
        std::string v = hdr.substr(o + 10, 70);
        size_t i = v.find_first_not_of(' ');
        if (i == std::string::npos) return false;
        v = v.substr(i);
        if (v[0] == '\'') {
            size_t j = v.find('\'', 1);
            out = v.substr(1, j == std::string::npos ? std::string::npos : j - 1);
        } else {
            size_t j = v.find('/');
            out = v.substr(0, j);
        }
        while (!out.empty() && out.back() == ' ') out.pop_back();
        return true;
    }
    return false;
}

bool read_file(const char *path, std::vector<unsigned char> &buf) {
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    buf.resize(sz > 0 ? (size_t)sz : 0);
    bool ok = sz >= 0 && fread(buf.data(), 1, buf.size(), f) == buf.size();
    fclose(f);
    return ok;
}

bool parse(const std::vector<unsigned char> &b, std::vector<Hdu> &hdus) {
    size_t off = 0;
    while (off + kBlock <= b.size()) {
        Hdu h;
        bool end = false;
        while (!end && off + kBlock <= b.size()) {
            for (size_t i = 0; i < kBlock / kCard; ++i) {
                const char *c = (const char *)b.data() + off + i * kCard;
                h.header.append(c, kCard);
                if (strncmp(c, "END", 3) == 0 && c[3] == ' ') { end = true; break; }
            }
            off += kBlock;
        }
        if (!end) return false;
        std::string v;
        if (!card_value(h.header, "BITPIX", v)) return false;
        h.bitpix = atoi(v.c_str());
        int nax = card_value(h.header, "NAXIS", v) ? atoi(v.c_str()) : 0;
        for (int a = 1; a <= nax; ++a) {
            std::string key = "NAXIS" + std::to_string(a);
            if (!card_value(h.header, key.c_str(), v)) return false;
            h.naxes.push_back(atoll(v.c_str()));
        }
        if (card_value(h.header, "BSCALE", v)) h.bscale = atof(v.c_str());
        if (card_value(h.header, "BZERO", v)) h.bzero = atof(v.c_str());
        long long pcount = card_value(h.header, "PCOUNT", v) ? atoll(v.c_str()) : 0;
        long long gcount = card_value(h.header, "GCOUNT", v) ? atoll(v.c_str()) : 1;
        h.data_off = off;
        size_t nbytes = (size_t)(abs(h.bitpix) / 8) * (size_t)gcount * (size_t)(pcount + h.count());
        if (off + nbytes > b.size()) return false;
        off += (nbytes + kBlock - 1) / kBlock * kBlock;
        hdus.push_back(std::move(h));
    }
    return !hdus.empty();
}

double load_be(const unsigned char *p, int bitpix) {
    unsigned char t[8];
    int nb = abs(bitpix) / 8;
    for (int i = 0; i < nb; ++i) t[i] = p[nb - 1 - i];
    switch (bitpix) {
        case 8: return (double)p[0];
        case 16: { int16_t v; memcpy(&v, t, 2); return v; }
        case 32: { int32_t v; memcpy(&v, t, 4); return v; }
        case 64: { int64_t v; memcpy(&v, t, 8); return (double)v; }
        case -32: { float v; memcpy(&v, t, 4); return v; }
        case -64: { double v; memcpy(&v, t, 8); return v; }
    }
    return 0.0;
}

double value(const std::vector<unsigned char> &b, const Hdu &h, long long i) {
    double v = load_be(b.data() + h.data_off + (size_t)i * (abs(h.bitpix) / 8), h.bitpix);
    return (h.bscale == 1.0 && h.bzero == 0.0) ? v : v * h.bscale + h.bzero;
}

void put_card(std::string &hdr, const std::string &text) {
    std::string c = text.substr(0, kCard);
    c.resize(kCard, ' ');
    hdr += c;
}

std::string int_card(const char *key, long long v) {
    char buf[81];
    snprintf(buf, sizeof buf, "%-8s= %20lld", key, v);
    return buf;
}

void pad_write(FILE *f, const std::string &hdr) {
    std::string h = hdr;
    put_card(h, "END");
    h.resize((h.size() + kBlock - 1) / kBlock * kBlock, ' ');
    fwrite(h.data(), 1, h.size(), f);
}

template <class T>
void write_data(FILE *f, const T *v, size_t n, int bitpix) {
    std::vector<unsigned char> out;
    size_t nb = (size_t)abs(bitpix) / 8;
    out.resize(n * nb);
    for (size_t i = 0; i < n; ++i) {
        unsigned char t[8];
        if (bitpix == -64) {
            double d = (double)v[i];
            memcpy(t, &d, 8);
        } else {
            float d = (float)v[i];
            memcpy(t, &d, 4);
        }
        for (size_t k = 0; k < nb; ++k) out[i * nb + k] = t[nb - 1 - k];
    }
    size_t padded = (out.size() + kBlock - 1) / kBlock * kBlock;
    out.resize(padded, 0);
    fwrite(out.data(), 1, out.size(), f);
}

}  // namespace

extern "C" {

hcg_status hcg_fits_read_samples(const char *path, uint64_t *n, uint32_t *nchan, double *lon, double *lat,
                                 float *values) {
    if (!path || !n || !nchan) return HCG_EINVAL;
    std::vector<unsigned char> b;
    std::vector<Hdu> h;
    if (!read_file(path, b) || !parse(b, h) || h.size() < 2) return HCG_EIO;
    const Hdu &d = h[0], &c = h[1];
    if (d.naxes.size() < 2) return HCG_EIO;
    long long N = d.naxes[0] * d.naxes[1];
    long long z = d.naxes.size() >= 3 ? d.naxes[2] : 1;
    if (c.count() < 2 * N) return HCG_EIO;
    *n = (uint64_t)N;
    *nchan = (uint32_t)z;
    if (lon && lat)
        for (long long i = 0; i < N; ++i) {
            lon[i] = value(b, c, i);
            lat[i] = value(b, c, N + i);
        }
    if (values)
        for (long long i = 0; i < N * z; ++i) values[i] = (float)value(b, d, i);
    return HCG_OK;
}

hcg_status hcg_fits_read_header(const char *path, char *header, size_t cap, size_t *len) {
    if (!path || !len) return HCG_EINVAL;
    std::vector<unsigned char> b;
    std::vector<Hdu> h;
    if (!read_file(path, b) || !parse(b, h)) return HCG_EIO;
    *len = h[0].header.size();
    if (header) {
        if (cap < h[0].header.size() + 1) return HCG_EINVAL;
        memcpy(header, h[0].header.data(), h[0].header.size());
        header[h[0].header.size()] = 0;
    }
    return HCG_OK;
}

hcg_status hcg_fits_write_cube(const char *path, const char *target_header, size_t len, uint32_t nx, uint32_t ny,
                               uint32_t nchan, const float *cube, const float *weights, int bitpix) {
    if (!path || !target_header || !cube || (bitpix != -32 && bitpix != -64)) return HCG_EINVAL;
    const char *p = path[0] == '!' ? path + 1 : path;  // cfitsio's overwrite prefix
    FILE *f = fopen(p, "wb");
    if (!f) return HCG_EIO;
    std::string hdr;
    put_card(hdr, "SIMPLE  =                    T");
    put_card(hdr, int_card("BITPIX", bitpix));
    put_card(hdr, int_card("NAXIS", 3));
    put_card(hdr, int_card("NAXIS1", nx));
    put_card(hdr, int_card("NAXIS2", ny));
    put_card(hdr, int_card("NAXIS3", nchan));
    if (weights) put_card(hdr, "EXTEND  =                    T");
    // the target's remaining cards, as write_output_map copies them (gmap.cpp:277-301)
    for (size_t o = 0; o + kCard <= len; o += kCard) {
        std::string card(target_header + o, kCard);
        std::string k = card.substr(0, 8);
        while (!k.empty() && k.back() == ' ') k.pop_back();
        if (k == "END") break;
        if (k == "SIMPLE" || k == "BITPIX" || k == "NAXIS" || k == "NAXIS1" || k == "NAXIS2" || k == "NAXIS3" ||
            k == "EXTEND" || k == "CHECKSUM" || k == "DATASUM" || card[0] == '#')
            continue;
        put_card(hdr, card);
    }
    pad_write(f, hdr);
    write_data(f, cube, (size_t)nx * ny * nchan, bitpix);
    if (weights) {
        std::string e;
        put_card(e, "XTENSION= 'IMAGE   '");
        put_card(e, int_card("BITPIX", -32));
        put_card(e, int_card("NAXIS", 2));
        put_card(e, int_card("NAXIS1", nx));
        put_card(e, int_card("NAXIS2", ny));
        put_card(e, int_card("PCOUNT", 0));
        put_card(e, int_card("GCOUNT", 1));
        put_card(e, "EXTNAME = 'WEIGHTS '");
        pad_write(f, e);
        write_data(f, weights, (size_t)nx * ny, -32);
    }
    bool ok = !ferror(f);
    fclose(f);
    return ok ? HCG_OK : HCG_EIO;
}

hcg_status hcg_fits_write_samples(const char *path, uint64_t n, uint32_t nchan, const double *lon,
                                  const double *lat, const float *values) {
    if (!path || !lon || !lat || !values || n == 0 || nchan == 0) return HCG_EINVAL;
    const char *p = path[0] == '!' ? path + 1 : path;
    FILE *f = fopen(p, "wb");
    if (!f) return HCG_EIO;
    std::string hdr;
    put_card(hdr, "SIMPLE  =                    T");
    put_card(hdr, int_card("BITPIX", -32));
    put_card(hdr, int_card("NAXIS", nchan > 1 ? 3 : 2));
    put_card(hdr, int_card("NAXIS1", 1));
    put_card(hdr, int_card("NAXIS2", (long long)n));
    if (nchan > 1) put_card(hdr, int_card("NAXIS3", nchan));
    put_card(hdr, "EXTEND  =                    T");
    pad_write(f, hdr);
    write_data(f, values, (size_t)n * nchan, -32);
    std::string e;
    put_card(e, "XTENSION= 'IMAGE   '");
    put_card(e, int_card("BITPIX", -64));
    put_card(e, int_card("NAXIS", 2));
    put_card(e, int_card("NAXIS1", (long long)n));
    put_card(e, int_card("NAXIS2", 2));
    put_card(e, int_card("PCOUNT", 0));
    put_card(e, int_card("GCOUNT", 1));
    pad_write(f, e);
    std::vector<double> c(2 * n);
    memcpy(c.data(), lon, n * sizeof(double));
    memcpy(c.data() + n, lat, n * sizeof(double));
    write_data(f, c.data(), 2 * n, -64);
    bool ok = !ferror(f);
    fclose(f);
    return ok ? HCG_OK : HCG_EIO;
}

}  // extern "C"
