/*
 * Minimal stand-in for the cfitsio calls that the reference's gmap.cpp makes
 * (HCGrid/gmap.cpp:102-379). TEST INFRASTRUCTURE ONLY: cfitsio itself is not
 * in this image (the reference's cfitsio-3.47 tarball is listed as missing),
 * so oracle/Makefile builds the reference's FITS path against this subset.
 *
 * Supported: primary and IMAGE-extension HDUs, BITPIX 8/16/32/64/-32/-64
 * with BSCALE/BZERO on read; DOUBLE_IMG output; header-string export.
 * Names and argument meanings follow the public cfitsio API.
 */
#ifndef HCG_SHIM_FITSIO_H
#define HCG_SHIM_FITSIO_H

#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hcg_fitsfile fitsfile;

#define READONLY 0
#define READWRITE 1
#define TDOUBLE 82
#define DOUBLE_IMG (-64)
#define FLOAT_IMG (-32)
#define IMAGE_HDU 0
#define FILE_NOT_OPENED 104
#define FILE_NOT_CREATED 105
#define KEY_NO_EXIST 202
#define NOT_TABLE 235
#define BAD_HDU_NUM 301
#define BAD_DATATYPE 410
#define BAD_ELEM_NUM 308
#define MEMORY_ALLOCATION 113

int fits_open_file(fitsfile **fptr, const char *filename, int iomode, int *status);
int fits_create_file(fitsfile **fptr, const char *filename, int *status);
int fits_close_file(fitsfile *fptr, int *status);
int fits_movabs_hdu(fitsfile *fptr, int hdunum, int *hdutype, int *status);
int fits_read_key_lng(fitsfile *fptr, const char *keyname, long *value, char *comm, int *status);
int fits_read_keys_lng(fitsfile *fptr, const char *keyroot, int nstart, int nmax, long *value, int *nfound,
                       int *status);
int fits_read_img(fitsfile *fptr, int datatype, long long firstelem, long long nelem, void *nulval, void *array,
                  int *anynul, int *status);
int fits_hdr2str(fitsfile *fptr, int nocomments, char **exclist, int nexc, char **header, int *nkeys, int *status);
int fits_create_img(fitsfile *fptr, int bitpix, int naxis, long *naxes, int *status);
int fits_write_record(fitsfile *fptr, const char *card, int *status);
int fits_write_img(fitsfile *fptr, int datatype, long long firstelem, long long nelem, void *array, int *status);
int fits_copy_header(fitsfile *infptr, fitsfile *outfptr, int *status);
int fits_write_col(fitsfile *fptr, int datatype, int colnum, long long firstrow, long long firstelem,
                   long long nelem, void *array, int *status);
void fits_report_error(FILE *stream, int status);

#ifdef __cplusplus
}
#endif
#endif
