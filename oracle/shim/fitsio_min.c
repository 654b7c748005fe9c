/*
 * Minimal FITS reader/writer behind the cfitsio subset in fitsio.h.
 * TEST INFRASTRUCTURE ONLY (see fitsio.h). FITS: 2880-byte records of
 * 80-character cards, big-endian data, one header + data unit per HDU.
 */
#include "fitsio.h"

#include <ctype.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define BLK 2880
#define CARD 80
#define MAX_HDU 16
#define MAX_OUT_CARDS 4096

typedef struct {
    size_t hdr_off, ncards, data_off;
    int bitpix, naxis;
    long naxes[9];
    double bscale, bzero;
} hdu_t;

struct hcg_fitsfile {
    int writing;
    /* read side */
    unsigned char *buf;
    size_t size;
    int nhdu, cur;
    hdu_t hdu[MAX_HDU];
    /* write side */
    char *path;
    int out_nhdu;
    FILE *out;
    char (*cards)[CARD];
    int ncards;
    int out_bitpix, out_naxis;
    long out_naxes[9];
    double *out_data;
    long long out_n;
};

static void card_key(const char *card, char key[9]) {
    int i;
    for (i = 0; i < 8; ++i) key[i] = card[i];
    key[8] = 0;
    for (i = 7; i >= 0 && key[i] == ' '; --i) key[i] = 0;
}

static int card_value(const char *card, char *val, size_t cap) {
    /* value field: columns 11-80 for "KEY     = value / comment" */
    if (card[8] != '=' || card[9] != ' ') return 0;
    const char *p = card + 10;
    const char *end = card + CARD;
    while (p < end && *p == ' ') ++p;
    size_t n = 0;
    if (p < end && *p == '\'') {
        ++p;
        while (p < end && n + 1 < cap) {
            if (*p == '\'') {
                if (p + 1 < end && p[1] == '\'') { val[n++] = '\''; p += 2; continue; }
                break;
            }
            val[n++] = *p++;
        }
    } else {
        while (p < end && *p != '/' && n + 1 < cap) val[n++] = *p++;
    }
    val[n] = 0;
    while (n > 0 && val[n - 1] == ' ') val[--n] = 0;
    return 1;
}

static const char *find_card(const fitsfile *f, int h, const char *key) {
    const hdu_t *u = &f->hdu[h];
    for (size_t i = 0; i < u->ncards; ++i) {
        const char *c = (const char *)f->buf + u->hdr_off + i * CARD;
        char k[9];
        card_key(c, k);
        if (strcmp(k, key) == 0) return c;
    }
    return NULL;
}

static int parse_hdus(fitsfile *f) {
    size_t off = 0;
    f->nhdu = 0;
    while (off + BLK <= f->size && f->nhdu < MAX_HDU) {
        hdu_t *u = &f->hdu[f->nhdu];
        memset(u, 0, sizeof(*u));
        u->hdr_off = off;
        u->bscale = 1.0;
        size_t ncards = 0;
        int found_end = 0;
        while (off + BLK <= f->size && !found_end) {
            for (int i = 0; i < BLK / CARD; ++i) {
                const char *c = (const char *)f->buf + off + (size_t)i * CARD;
                ++ncards;
                if (strncmp(c, "END", 3) == 0 && (c[3] == ' ')) { found_end = 1; break; }
            }
            off += BLK;
        }
        if (!found_end) return -1;
        u->ncards = ncards;
        u->data_off = off;
        f->nhdu++;
        char v[80];
        const char *c;
        int h = f->nhdu - 1;
        if ((c = find_card(f, h, "BITPIX")) && card_value(c, v, sizeof v)) u->bitpix = atoi(v);
        if ((c = find_card(f, h, "NAXIS")) && card_value(c, v, sizeof v)) u->naxis = atoi(v);
        long long n = u->naxis > 0 ? 1 : 0;
        for (int a = 1; a <= u->naxis && a <= 9; ++a) {
            char key[9];
            snprintf(key, sizeof key, "NAXIS%d", a);
            if ((c = find_card(f, h, key)) && card_value(c, v, sizeof v)) u->naxes[a - 1] = atol(v);
            n *= u->naxes[a - 1];
        }
        if ((c = find_card(f, h, "BSCALE")) && card_value(c, v, sizeof v)) u->bscale = atof(v);
        if ((c = find_card(f, h, "BZERO")) && card_value(c, v, sizeof v)) u->bzero = atof(v);
        long pcount = 0, gcount = 1;
        if ((c = find_card(f, h, "PCOUNT")) && card_value(c, v, sizeof v)) pcount = atol(v);
        if ((c = find_card(f, h, "GCOUNT")) && card_value(c, v, sizeof v)) gcount = atol(v);
        size_t nbytes = (size_t)(abs(u->bitpix) / 8) * (size_t)gcount * (size_t)(pcount + n);
        off += (nbytes + BLK - 1) / BLK * BLK;
    }
    return f->nhdu > 0 ? 0 : -1;
}

int fits_open_file(fitsfile **fptr, const char *filename, int iomode, int *status) {
    (void)iomode;
    if (*status) return *status;
    FILE *fp = fopen(filename, "rb");
    if (!fp) return *status = FILE_NOT_OPENED;
    fitsfile *f = (fitsfile *)calloc(1, sizeof(fitsfile));
    fseek(fp, 0, SEEK_END);
    f->size = (size_t)ftell(fp);
    fseek(fp, 0, SEEK_SET);
    f->buf = (unsigned char *)malloc(f->size ? f->size : 1);
    if (fread(f->buf, 1, f->size, fp) != f->size) { fclose(fp); free(f->buf); free(f); return *status = FILE_NOT_OPENED; }
    fclose(fp);
    if (parse_hdus(f)) { free(f->buf); free(f); return *status = FILE_NOT_OPENED; }
    f->cur = 0;
    *fptr = f;
    return 0;
}

int fits_create_file(fitsfile **fptr, const char *filename, int *status) {
    if (*status) return *status;
    const char *p = filename;
    if (*p == '!') ++p; /* cfitsio's overwrite prefix */
    FILE *out = fopen(p, "wb");
    if (!out) return *status = FILE_NOT_CREATED;
    fitsfile *f = (fitsfile *)calloc(1, sizeof(fitsfile));
    f->writing = 1;
    f->out = out;
    f->cards = (char (*)[CARD])calloc(MAX_OUT_CARDS, CARD);
    *fptr = f;
    return 0;
}

static void put_card(fitsfile *f, const char *text) {
    if (f->ncards >= MAX_OUT_CARDS) return;
    char *c = f->cards[f->ncards++];
    memset(c, ' ', CARD);
    size_t n = strlen(text);
    if (n > CARD) n = CARD;
    memcpy(c, text, n);
}

static void be_store(unsigned char *dst, const void *src, int nbytes) {
    const unsigned char *s = (const unsigned char *)src;
    for (int i = 0; i < nbytes; ++i) dst[i] = s[nbytes - 1 - i];
}

static void flush_hdu(fitsfile *f) {
    if (!f->ncards) return;
    put_card(f, "END");
    size_t hbytes = (size_t)f->ncards * CARD;
    size_t hpad = (hbytes + BLK - 1) / BLK * BLK;
    unsigned char *h = (unsigned char *)malloc(hpad);
    memset(h, ' ', hpad);
    memcpy(h, f->cards, hbytes);
    fwrite(h, 1, hpad, f->out);
    free(h);
    long long n = f->out_naxis > 0 ? 1 : 0;
    for (int a = 0; a < f->out_naxis; ++a) n *= f->out_naxes[a];
    size_t dbytes = (size_t)n * 8;
    size_t dpad = (dbytes + BLK - 1) / BLK * BLK;
    if (dpad) {
        unsigned char *d = (unsigned char *)calloc(dpad, 1);
        for (long long i = 0; i < n && i < f->out_n; ++i) be_store(d + i * 8, &f->out_data[i], 8);
        fwrite(d, 1, dpad, f->out);
        free(d);
    }
    free(f->out_data);
    f->out_data = NULL;
    f->out_n = 0;
    f->ncards = 0;
    f->out_nhdu++;
}

int fits_create_img(fitsfile *fptr, int bitpix, int naxis, long *naxes, int *status) {
    if (*status) return *status;
    if (bitpix != DOUBLE_IMG) return *status = BAD_DATATYPE;
    flush_hdu(fptr);
    char buf[81];
    if (fptr->out_nhdu == 0) {
        snprintf(buf, sizeof buf, "%-8s= %20s", "SIMPLE", "T");
    } else {
        snprintf(buf, sizeof buf, "%-8s= %-20s", "XTENSION", "'IMAGE   '");
    }
    put_card(fptr, buf);
    snprintf(buf, sizeof buf, "%-8s= %20d", "BITPIX", bitpix);
    put_card(fptr, buf);
    snprintf(buf, sizeof buf, "%-8s= %20d", "NAXIS", naxis);
    put_card(fptr, buf);
    long long n = 1;
    for (int a = 0; a < naxis; ++a) {
        char key[9];
        snprintf(key, sizeof key, "NAXIS%d", a + 1);
        snprintf(buf, sizeof buf, "%-8s= %20ld", key, naxes[a]);
        put_card(fptr, buf);
        fptr->out_naxes[a] = naxes[a];
        n *= naxes[a];
    }
    if (fptr->out_nhdu > 0) {
        snprintf(buf, sizeof buf, "%-8s= %20d", "PCOUNT", 0);
        put_card(fptr, buf);
        snprintf(buf, sizeof buf, "%-8s= %20d", "GCOUNT", 1);
        put_card(fptr, buf);
    }
    fptr->out_bitpix = bitpix;
    fptr->out_naxis = naxis;
    fptr->out_data = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    fptr->out_n = n;
    return 0;
}

int fits_write_record(fitsfile *fptr, const char *card, int *status) {
    if (*status) return *status;
    if (strncmp(card, "END", 3) == 0 && (card[3] == ' ' || card[3] == 0)) return 0;
    put_card(fptr, card);
    return 0;
}

int fits_write_img(fitsfile *fptr, int datatype, long long firstelem, long long nelem, void *array, int *status) {
    if (*status) return *status;
    if (datatype != TDOUBLE) return *status = BAD_DATATYPE;
    if (firstelem < 1 || firstelem - 1 + nelem > fptr->out_n) return *status = BAD_ELEM_NUM;
    memcpy(fptr->out_data + (firstelem - 1), array, (size_t)nelem * sizeof(double));
    return 0;
}

int fits_copy_header(fitsfile *infptr, fitsfile *outfptr, int *status) {
    if (*status) return *status;
    flush_hdu(outfptr);
    const hdu_t *u = &infptr->hdu[infptr->cur];
    outfptr->out_naxis = u->naxis;
    long long n = u->naxis > 0 ? 1 : 0;
    for (int a = 0; a < u->naxis; ++a) { outfptr->out_naxes[a] = u->naxes[a]; n *= u->naxes[a]; }
    for (size_t i = 0; i < u->ncards; ++i) {
        char c[CARD + 1];
        memcpy(c, infptr->buf + u->hdr_off + i * CARD, CARD);
        c[CARD] = 0;
        if (strncmp(c, "END", 3) == 0 && c[3] == ' ') break;
        if (strncmp(c, "BITPIX  ", 8) == 0) {
            char b[81];
            snprintf(b, sizeof b, "%-8s= %20d", "BITPIX", DOUBLE_IMG);
            put_card(outfptr, b);
            continue;
        }
        put_card(outfptr, c);
    }
    outfptr->out_bitpix = DOUBLE_IMG;
    outfptr->out_data = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    outfptr->out_n = n;
    return 0;
}

int fits_write_col(fitsfile *fptr, int datatype, int colnum, long long firstrow, long long firstelem,
                   long long nelem, void *array, int *status) {
    (void)fptr; (void)datatype; (void)colnum; (void)firstrow; (void)firstelem; (void)nelem; (void)array;
    if (*status) return *status;
    return *status = NOT_TABLE; /* cfitsio refuses column writes on an IMAGE HDU as well */
}

int fits_close_file(fitsfile *fptr, int *status) {
    if (!fptr) return *status;
    if (fptr->writing) {
        flush_hdu(fptr);
        fclose(fptr->out);
        free(fptr->cards);
    } else {
        free(fptr->buf);
    }
    free(fptr);
    return *status;
}

int fits_movabs_hdu(fitsfile *fptr, int hdunum, int *hdutype, int *status) {
    if (*status) return *status;
    if (hdunum < 1 || hdunum > fptr->nhdu) return *status = BAD_HDU_NUM;
    fptr->cur = hdunum - 1;
    if (hdutype) *hdutype = IMAGE_HDU;
    return 0;
}

int fits_read_key_lng(fitsfile *fptr, const char *keyname, long *value, char *comm, int *status) {
    (void)comm;
    if (*status) return *status;
    const char *c = find_card(fptr, fptr->cur, keyname);
    char v[80];
    if (!c || !card_value(c, v, sizeof v)) return *status = KEY_NO_EXIST;
    *value = atol(v);
    return 0;
}

int fits_read_keys_lng(fitsfile *fptr, const char *keyroot, int nstart, int nmax, long *value, int *nfound,
                       int *status) {
    if (*status) return *status;
    *nfound = 0;
    for (int i = 0; i < nmax; ++i) {
        char key[16];
        snprintf(key, sizeof key, "%s%d", keyroot, nstart + i);
        const char *c = find_card(fptr, fptr->cur, key);
        char v[80];
        if (c && card_value(c, v, sizeof v)) {
            value[i] = atol(v);
            *nfound = i + 1;
        }
    }
    return 0;
}

static double be_load(const unsigned char *p, int bitpix) {
    unsigned char t[8];
    int nb = abs(bitpix) / 8;
    for (int i = 0; i < nb; ++i) t[i] = p[nb - 1 - i];
    switch (bitpix) {
        case 8: return (double)p[0];
        case 16: { int16_t v; memcpy(&v, t, 2); return (double)v; }
        case 32: { int32_t v; memcpy(&v, t, 4); return (double)v; }
        case 64: { int64_t v; memcpy(&v, t, 8); return (double)v; }
        case -32: { float v; memcpy(&v, t, 4); return (double)v; }
        case -64: { double v; memcpy(&v, t, 8); return v; }
    }
    return 0.0;
}

int fits_read_img(fitsfile *fptr, int datatype, long long firstelem, long long nelem, void *nulval, void *array,
                  int *anynul, int *status) {
    (void)nulval;
    if (*status) return *status;
    if (datatype != TDOUBLE) return *status = BAD_DATATYPE;
    const hdu_t *u = &fptr->hdu[fptr->cur];
    long long n = u->naxis > 0 ? 1 : 0;
    for (int a = 0; a < u->naxis; ++a) n *= u->naxes[a];
    if (firstelem < 1 || firstelem - 1 + nelem > n) return *status = BAD_ELEM_NUM;
    int nb = abs(u->bitpix) / 8;
    double *out = (double *)array;
    for (long long i = 0; i < nelem; ++i) {
        const unsigned char *p = fptr->buf + u->data_off + (size_t)(firstelem - 1 + i) * nb;
        double v = be_load(p, u->bitpix);
        out[i] = (u->bscale == 1.0 && u->bzero == 0.0) ? v : v * u->bscale + u->bzero;
    }
    if (anynul) *anynul = 0;
    return 0;
}

int fits_hdr2str(fitsfile *fptr, int nocomments, char **exclist, int nexc, char **header, int *nkeys, int *status) {
    (void)exclist; (void)nexc;
    if (*status) return *status;
    const hdu_t *u = &fptr->hdu[fptr->cur];
    char *s = (char *)malloc(u->ncards * CARD + 1);
    size_t k = 0;
    int nk = 0;
    for (size_t i = 0; i < u->ncards; ++i) {
        const char *c = (const char *)fptr->buf + u->hdr_off + i * CARD;
        int is_end = strncmp(c, "END", 3) == 0 && c[3] == ' ';
        if (nocomments && (strncmp(c, "COMMENT ", 8) == 0 || strncmp(c, "HISTORY ", 8) == 0)) continue;
        int blank = 1;
        for (int j = 0; j < CARD; ++j) if (c[j] != ' ') { blank = 0; break; }
        if (blank) continue;
        memcpy(s + k, c, CARD);
        k += CARD;
        ++nk;
        if (is_end) break;
    }
    s[k] = 0;
    *header = s;
    *nkeys = nk - 1; /* the END record is appended but not counted */
    return 0;
}

void fits_report_error(FILE *stream, int status) {
    fprintf(stream, "FITS shim error status %d\n", status);
}
