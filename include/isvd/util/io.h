/* I/O utilities (reference src/include/c/isvd/util/io.h:19-21; util/io.c:22-45): read one value
 * from a text stream, as demo/cdemo.c:60-64 does for each entry of a Matrix Market array.  A
 * stream that holds no value there records ISVD_GPU_ERROR_ARGUMENT (the reference asserts) and
 * leaves *varp unchanged.  For whole files, isvd_?MtxRead (<isvd/b200.h>) parses in parallel. */
#ifndef ISVD_UTIL_IO_H_
#define ISVD_UTIL_IO_H_

#include <stdio.h>

#include <isvd/def.h>

#if defined(__cplusplus)
extern "C" {
#endif

void isvd_iFget( FILE *stream, isvd_int_t   *varp );
void isvd_sFget( FILE *stream, isvd_s_val_t *varp );
void isvd_dFget( FILE *stream, isvd_d_val_t *varp );

#if defined(__cplusplus)
}
#endif

#endif  /* ISVD_UTIL_IO_H_ */
