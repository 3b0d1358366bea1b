/*
 * Header-only Matrix Market banner / size routines with the interface of the NIST "Matrix Market
 * I/O library for ANSI C" (mmio.h), which the reference vendors under ext/mmio and its demo
 * (demo/cdemo.c:51-73) calls: mm_read_banner, the mm_is_* / mm_set_* typecode macros,
 * mm_read_mtx_array_size, mm_typecode_to_str.  A program written for the reference compiles
 * against this header (-I include/mmio_shim) with nothing else to link.  Everything is
 * `static inline`: no symbol is exported, and a real mmio library can still be linked.
 *
 * MM_typecode is the library's four characters: [0] 'M' matrix; [1] 'C' coordinate / 'A' array;
 * [2] 'R' real / 'C' complex / 'P' pattern / 'I' integer; [3] 'G' general / 'S' symmetric /
 * 'H' hermitian / 'K' skew-symmetric.  Routines return 0 or one of the MM_* error codes.
 *
 * Whole files (values included, dense or coordinate) are read faster by isvd_?MtxRead in
 * <isvd/b200.h>, which parses the values on all host threads.
 */
#ifndef ISVD_MMIO_SHIM_H_
#define ISVD_MMIO_SHIM_H_

#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#if defined(__cplusplus)
extern "C" {
#endif

#define MM_MAX_LINE_LENGTH 1025
#define MatrixMarketBanner "%%MatrixMarket"
#define MM_MAX_TOKEN_LENGTH 64

typedef char MM_typecode[4];

/* error codes */
#define MM_COULD_NOT_READ_FILE  11
#define MM_PREMATURE_EOF        12
#define MM_NOT_MTX              13
#define MM_NO_HEADER            14
#define MM_UNSUPPORTED_TYPE     15
#define MM_LINE_TOO_LONG        16
#define MM_COULD_NOT_WRITE_FILE 17

/* banner words */
#define MM_MTX_STR        "matrix"
#define MM_ARRAY_STR      "array"
#define MM_DENSE_STR      "array"
#define MM_COORDINATE_STR "coordinate"
#define MM_SPARSE_STR     "coordinate"
#define MM_COMPLEX_STR    "complex"
#define MM_REAL_STR       "real"
#define MM_INT_STR        "integer"
#define MM_GENERAL_STR    "general"
#define MM_SYMM_STR       "symmetric"
#define MM_HERM_STR       "hermitian"
#define MM_SKEW_STR       "skew-symmetric"
#define MM_PATTERN_STR    "pattern"

/* typecode queries */
#define mm_is_matrix(tc)     ((tc)[0] == 'M')
#define mm_is_sparse(tc)     ((tc)[1] == 'C')
#define mm_is_coordinate(tc) ((tc)[1] == 'C')
#define mm_is_dense(tc)      ((tc)[1] == 'A')
#define mm_is_array(tc)      ((tc)[1] == 'A')
#define mm_is_complex(tc)    ((tc)[2] == 'C')
#define mm_is_real(tc)       ((tc)[2] == 'R')
#define mm_is_pattern(tc)    ((tc)[2] == 'P')
#define mm_is_integer(tc)    ((tc)[2] == 'I')
#define mm_is_symmetric(tc)  ((tc)[3] == 'S')
#define mm_is_general(tc)    ((tc)[3] == 'G')
#define mm_is_skew(tc)       ((tc)[3] == 'K')
#define mm_is_hermitian(tc)  ((tc)[3] == 'H')

/* typecode setters (take a pointer to the typecode) */
#define mm_set_matrix(tcp)     ((*(tcp))[0] = 'M')
#define mm_set_coordinate(tcp) ((*(tcp))[1] = 'C')
#define mm_set_array(tcp)      ((*(tcp))[1] = 'A')
#define mm_set_dense(tcp)      mm_set_array(tcp)
#define mm_set_sparse(tcp)     mm_set_coordinate(tcp)
#define mm_set_complex(tcp)    ((*(tcp))[2] = 'C')
#define mm_set_real(tcp)       ((*(tcp))[2] = 'R')
#define mm_set_pattern(tcp)    ((*(tcp))[2] = 'P')
#define mm_set_integer(tcp)    ((*(tcp))[2] = 'I')
#define mm_set_symmetric(tcp)  ((*(tcp))[3] = 'S')
#define mm_set_general(tcp)    ((*(tcp))[3] = 'G')
#define mm_set_skew(tcp)       ((*(tcp))[3] = 'K')
#define mm_set_hermitian(tcp)  ((*(tcp))[3] = 'H')
#define mm_clear_typecode(tcp) ((*(tcp))[0] = (*(tcp))[1] = (*(tcp))[2] = ' ', (*(tcp))[3] = 'G')
#define mm_initialize_typecode(tcp) mm_clear_typecode(tcp)

/* Case-insensitive equality of a banner word. */
static inline int isvd_mm_word_is(const char *w, const char *ref) {
  for (; *w && *ref; ++w, ++ref)
    if (tolower((unsigned char)*w) != *ref) return 0;
  return *w == 0 && *ref == 0;
}

/* 1 when the typecode is one the format allows. */
static inline int mm_is_valid(MM_typecode tc) {
  if (!mm_is_matrix(tc)) return 0;
  if (mm_is_dense(tc) && mm_is_pattern(tc)) return 0;
  if (mm_is_real(tc) && mm_is_hermitian(tc)) return 0;
  if (mm_is_pattern(tc) && (mm_is_hermitian(tc) || mm_is_skew(tc))) return 0;
  return 1;
}

/* Reads the banner line "%%MatrixMarket matrix <format> <field> <symmetry>" into *tc. */
static inline int mm_read_banner(FILE *f, MM_typecode *tc) {
  char line[MM_MAX_LINE_LENGTH];
  char w[5][MM_MAX_TOKEN_LENGTH];
  mm_clear_typecode(tc);
  if (!f || !fgets(line, (int)sizeof(line), f)) return MM_PREMATURE_EOF;
  if (sscanf(line, "%63s %63s %63s %63s %63s", w[0], w[1], w[2], w[3], w[4]) != 5) return MM_PREMATURE_EOF;
  if (strcmp(w[0], MatrixMarketBanner) != 0) return MM_NO_HEADER;
  if (!isvd_mm_word_is(w[1], MM_MTX_STR)) return MM_UNSUPPORTED_TYPE;
  mm_set_matrix(tc);
  if (isvd_mm_word_is(w[2], MM_SPARSE_STR)) mm_set_coordinate(tc);
  else if (isvd_mm_word_is(w[2], MM_DENSE_STR)) mm_set_array(tc);
  else return MM_UNSUPPORTED_TYPE;
  if (isvd_mm_word_is(w[3], MM_REAL_STR)) mm_set_real(tc);
  else if (isvd_mm_word_is(w[3], MM_COMPLEX_STR)) mm_set_complex(tc);
  else if (isvd_mm_word_is(w[3], MM_PATTERN_STR)) mm_set_pattern(tc);
  else if (isvd_mm_word_is(w[3], MM_INT_STR)) mm_set_integer(tc);
  else return MM_UNSUPPORTED_TYPE;
  if (isvd_mm_word_is(w[4], MM_GENERAL_STR)) mm_set_general(tc);
  else if (isvd_mm_word_is(w[4], MM_SYMM_STR)) mm_set_symmetric(tc);
  else if (isvd_mm_word_is(w[4], MM_HERM_STR)) mm_set_hermitian(tc);
  else if (isvd_mm_word_is(w[4], MM_SKEW_STR)) mm_set_skew(tc);
  else return MM_UNSUPPORTED_TYPE;
  return 0;
}

/* Skips comment ('%') and blank lines, then reads `count` integers of the size line. */
static inline int isvd_mm_read_size_line(FILE *f, int count, int *a, int *b, int *c) {
  char line[MM_MAX_LINE_LENGTH];
  for (;;) {
    if (!fgets(line, (int)sizeof(line), f)) return MM_PREMATURE_EOF;
    const char *q = line;
    while (*q && isspace((unsigned char)*q)) ++q;
    if (*q && *q != '%') break;
  }
  const int got = count == 2 ? sscanf(line, "%d %d", a, b) : sscanf(line, "%d %d %d", a, b, c);
  return got == count ? 0 : MM_PREMATURE_EOF;
}

static inline int mm_read_mtx_array_size(FILE *f, int *M, int *N) {
  if (M) *M = 0;
  if (N) *N = 0;
  return isvd_mm_read_size_line(f, 2, M, N, NULL);
}

static inline int mm_read_mtx_crd_size(FILE *f, int *M, int *N, int *nz) {
  if (M) *M = 0;
  if (N) *N = 0;
  if (nz) *nz = 0;
  return isvd_mm_read_size_line(f, 3, M, N, nz);
}

/* "matrix <format> <field> <symmetry>" for a typecode (a new string the caller may free), or
 * NULL for an invalid code. */
static inline char *mm_typecode_to_str(MM_typecode tc) {
  const char *fmt = mm_is_sparse(tc) ? MM_SPARSE_STR : mm_is_dense(tc) ? MM_DENSE_STR : NULL;
  const char *field = mm_is_real(tc) ? MM_REAL_STR : mm_is_complex(tc) ? MM_COMPLEX_STR
                    : mm_is_pattern(tc) ? MM_PATTERN_STR : mm_is_integer(tc) ? MM_INT_STR : NULL;
  const char *sym = mm_is_general(tc) ? MM_GENERAL_STR : mm_is_symmetric(tc) ? MM_SYMM_STR
                  : mm_is_hermitian(tc) ? MM_HERM_STR : mm_is_skew(tc) ? MM_SKEW_STR : NULL;
  if (!mm_is_matrix(tc) || !fmt || !field || !sym) return NULL;
  const size_t len = strlen(MM_MTX_STR) + strlen(fmt) + strlen(field) + strlen(sym) + 4;
  char *s = (char *)malloc(len);
  if (s) snprintf(s, len, "%s %s %s %s", MM_MTX_STR, fmt, field, sym);
  return s;
}

static inline int mm_write_banner(FILE *f, MM_typecode tc) {
  char *s = mm_typecode_to_str(tc);
  if (!s) return MM_UNSUPPORTED_TYPE;
  const int ok = fprintf(f, "%s %s\n", MatrixMarketBanner, s) > 0;
  free(s);
  return ok ? 0 : MM_COULD_NOT_WRITE_FILE;
}

static inline int mm_write_mtx_array_size(FILE *f, int M, int N) {
  return fprintf(f, "%d %d\n", M, N) > 0 ? 0 : MM_COULD_NOT_WRITE_FILE;
}

static inline int mm_write_mtx_crd_size(FILE *f, int M, int N, int nz) {
  return fprintf(f, "%d %d %d\n", M, N, nz) > 0 ? 0 : MM_COULD_NOT_WRITE_FILE;
}

#if defined(__cplusplus)
}
#endif

#endif /* ISVD_MMIO_SHIM_H_ */
