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
// Headers are read block by block and data units converted straight from the
// file into the caller's arrays by several threads (pread of 4 MB pieces);
// writes convert in parallel 64 MB at a time.
#include <fcntl.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <string>
#include <thread>
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

// Threads for `bytes` of conversion: one per 4 MB, at most the cores (16).
unsigned io_threads(uint64_t bytes) {
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(hw, bytes >> 22));
}

// fn(begin, end) over [0, n) split evenly across `nt` threads.
template <class F>
void parallel_ranges(uint64_t n, unsigned nt, F fn) {
    if (nt <= 1 || n < 2) {
        fn(0, n);
        return;
    }
    std::vector<std::thread> th;
    const uint64_t per = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; ++t) {
        const uint64_t a = std::min<uint64_t>(n, t * per), b = std::min<uint64_t>(n, a + per);
        if (a < b) th.emplace_back(fn, a, b);
    }
    for (auto &x : th) x.join();
}

bool read_at(int fd, void *dst, size_t n, uint64_t off) {
    char *p = (char *)dst;
    while (n) {
        const ssize_t r = pread(fd, p, n, (off_t)off);
        if (r <= 0) return false;
        p += r;
        n -= (size_t)r;
        off += (uint64_t)r;
    }
    return true;
}

struct File {
    int fd = -1;
    uint64_t size = 0;
    explicit File(const char *path) {
        fd = open(path, O_RDONLY);
        struct stat st;
        if (fd >= 0 && fstat(fd, &st) == 0) size = (uint64_t)st.st_size;
    }
    ~File() {
        if (fd >= 0) close(fd);
    }
};

// Headers and data offsets of the first `max_hdus` HDUs.
bool parse(const File &f, std::vector<Hdu> &hdus, size_t max_hdus) {
    uint64_t off = 0;
    char blk[kBlock];
    while (off + kBlock <= f.size && hdus.size() < max_hdus) {
        Hdu h;
        bool end = false;
        while (!end && off + kBlock <= f.size) {
            if (!read_at(f.fd, blk, kBlock, off)) return false;
            for (size_t i = 0; i < kBlock / kCard; ++i) {
                const char *c = blk + i * kCard;
                h.header.append(c, kCard);
                if (strncmp(c, "END", 3) == 0 && c[3] == ' ') { end = true; break; }
            }
            off += kBlock;
        }
        if (!end) return false;
        std::string v;
        if (!card_value(h.header, "BITPIX", v)) return false;
        h.bitpix = atoi(v.c_str());
        if (h.bitpix != 8 && h.bitpix != 16 && h.bitpix != 32 && h.bitpix != 64 && h.bitpix != -32 && h.bitpix != -64)
            return false;
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
        uint64_t nbytes = (uint64_t)(abs(h.bitpix) / 8) * (uint64_t)gcount * (uint64_t)(pcount + h.count());
        if (off + nbytes > f.size) return false;
        off += (nbytes + kBlock - 1) / kBlock * kBlock;
        hdus.push_back(std::move(h));
    }
    return !hdus.empty();
}

// n big-endian values of `bitpix` at src, scaled as the header says, into dst.
template <class Out>
void decode(const unsigned char *src, uint64_t n, const Hdu &h, Out *dst) {
    const bool scaled = !(h.bscale == 1.0 && h.bzero == 0.0);
    auto put = [&](uint64_t i, double v) { dst[i] = (Out)(scaled ? v * h.bscale + h.bzero : v); };
    switch (h.bitpix) {
        case 8:
            for (uint64_t i = 0; i < n; ++i) put(i, (double)src[i]);
            break;
        case 16:
            for (uint64_t i = 0; i < n; ++i) {
                uint16_t u;
                memcpy(&u, src + 2 * i, 2);
                put(i, (double)(int16_t)__builtin_bswap16(u));
            }
            break;
        case 32:
            for (uint64_t i = 0; i < n; ++i) {
                uint32_t u;
                memcpy(&u, src + 4 * i, 4);
                put(i, (double)(int32_t)__builtin_bswap32(u));
            }
            break;
        case 64:
            for (uint64_t i = 0; i < n; ++i) {
                uint64_t u;
                memcpy(&u, src + 8 * i, 8);
                put(i, (double)(int64_t)__builtin_bswap64(u));
            }
            break;
        case -32:
            for (uint64_t i = 0; i < n; ++i) {
                uint32_t u;
                memcpy(&u, src + 4 * i, 4);
                u = __builtin_bswap32(u);
                float x;
                memcpy(&x, &u, 4);
                put(i, (double)x);
            }
            break;
        case -64:
            for (uint64_t i = 0; i < n; ++i) {
                uint64_t u;
                memcpy(&u, src + 8 * i, 8);
                u = __builtin_bswap64(u);
                double x;
                memcpy(&x, &u, 8);
                put(i, x);
            }
            break;
    }
}

// Values [first, first + n) of an HDU's data unit into dst, several threads
// each reading its own range in 4 MB pieces.
template <class Out>
bool read_values(const File &f, const Hdu &h, uint64_t first, uint64_t n, Out *dst) {
    const uint64_t es = (uint64_t)abs(h.bitpix) / 8;
    std::atomic<bool> ok{true};
    parallel_ranges(n, io_threads(n * es), [&](uint64_t a, uint64_t b) {
        const uint64_t piece = std::max<uint64_t>(1, (4u << 20) / es);
        std::vector<unsigned char> buf((size_t)(std::min(piece, b - a) * es));
        for (uint64_t i = a; i < b && ok;) {
            const uint64_t m = std::min(piece, b - i);
            if (!read_at(f.fd, buf.data(), (size_t)(m * es), h.data_off + (first + i) * es)) {
                ok = false;
                return;
            }
            decode(buf.data(), m, h, dst + i);
            i += m;
        }
    });
    return ok;
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

// n values as big-endian `bitpix` (-32 or -64) and the zero padding of the
// data unit; converted in parallel 64 MB at a time.
template <class T>
bool write_data(FILE *f, const T *v, size_t n, int bitpix) {
    const size_t nb = (size_t)abs(bitpix) / 8, chunk = (64u << 20) / nb;
    std::vector<unsigned char> out(std::min(n, chunk) * nb);
    for (size_t i0 = 0; i0 < n; i0 += chunk) {
        const size_t m = std::min(chunk, n - i0);
        parallel_ranges(m, io_threads(m * nb), [&](uint64_t a, uint64_t b) {
            for (uint64_t i = a; i < b; ++i) {
                if (bitpix == -64) {
                    const double d = (double)v[i0 + i];
                    uint64_t u;
                    memcpy(&u, &d, 8);
                    u = __builtin_bswap64(u);
                    memcpy(&out[i * 8], &u, 8);
                } else {
                    const float d = (float)v[i0 + i];
                    uint32_t u;
                    memcpy(&u, &d, 4);
                    u = __builtin_bswap32(u);
                    memcpy(&out[i * 4], &u, 4);
                }
            }
        });
        if (fwrite(out.data(), 1, m * nb, f) != m * nb) return false;
    }
    const size_t pad = (kBlock - (n * nb) % kBlock) % kBlock;
    const std::vector<unsigned char> zero(pad, 0);
    return pad == 0 || fwrite(zero.data(), 1, pad, f) == pad;
}

}  // namespace

extern "C" {

hcg_status hcg_fits_read_samples(const char *path, uint64_t *n, uint32_t *nchan, double *lon, double *lat,
                                 float *values) {
    if (!path || !n || !nchan) return HCG_EINVAL;
    File f(path);
    std::vector<Hdu> h;
    if (f.fd < 0 || !parse(f, h, 2) || h.size() < 2) return HCG_EIO;
    const Hdu &d = h[0], &c = h[1];
    if (d.naxes.size() < 2) return HCG_EIO;
    long long N = d.naxes[0] * d.naxes[1];
    long long z = d.naxes.size() >= 3 ? d.naxes[2] : 1;
    if (c.count() < 2 * N) return HCG_EIO;
    *n = (uint64_t)N;
    *nchan = (uint32_t)z;
    if (lon && lat && (!read_values(f, c, 0, (uint64_t)N, lon) || !read_values(f, c, (uint64_t)N, (uint64_t)N, lat)))
        return HCG_EIO;
    if (values && !read_values(f, d, 0, (uint64_t)(N * z), values)) return HCG_EIO;
    return HCG_OK;
}

hcg_status hcg_fits_read_header(const char *path, char *header, size_t cap, size_t *len) {
    if (!path || !len) return HCG_EINVAL;
    File f(path);
    std::vector<Hdu> h;
    if (f.fd < 0 || !parse(f, h, 1)) return HCG_EIO;
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
    bool wrote = write_data(f, cube, (size_t)nx * ny * nchan, bitpix);
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
        wrote = write_data(f, weights, (size_t)nx * ny, -32) && wrote;
    }
    bool ok = wrote && !ferror(f);
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
    bool wrote = write_data(f, values, (size_t)n * nchan, -32);
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
    wrote = write_data(f, c.data(), 2 * n, -64) && wrote;
    bool ok = wrote && !ferror(f);
    fclose(f);
    return ok ? HCG_OK : HCG_EIO;
}

}  // extern "C"
