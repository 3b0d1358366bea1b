/* Host memory helpers (reference src/include/c/isvd/util/memory.h:19-43; la/util/memory.c:30-127).
 * Buffers are 64-byte aligned; isvd_Free releases any of them. */
#ifndef ISVD_UTIL_MEMORY_H_
#define ISVD_UTIL_MEMORY_H_

#include <isvd/def.h>

#if defined(__cplusplus)
extern "C" {
#endif

isvd_int_t*   isvd_iMalloc( const size_t num );
isvd_s_val_t* isvd_sMalloc( const size_t num );
isvd_d_val_t* isvd_dMalloc( const size_t num );

void isvd_Free( void *ptr );

void isvd_iMemset0( isvd_int_t   *ptr, const size_t num );
void isvd_sMemset0( isvd_s_val_t *ptr, const size_t num );
void isvd_dMemset0( isvd_d_val_t *ptr, const size_t num );

void isvd_iMemcpy( isvd_int_t   *dst, const isvd_int_t   *src, const size_t num );
void isvd_sMemcpy( isvd_s_val_t *dst, const isvd_s_val_t *src, const size_t num );
void isvd_dMemcpy( isvd_d_val_t *dst, const isvd_d_val_t *src, const size_t num );

#if defined(__cplusplus)
}
#endif

#endif  /* ISVD_UTIL_MEMORY_H_ */
