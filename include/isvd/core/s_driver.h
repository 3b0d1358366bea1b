/*
 * iSVD driver, single precision (reference src/include/c/isvd/core/@x@_driver.h:21-28;
 * core/driver/@x@_isvd.c:106-282).
 */
#ifndef ISVD_CORE_S_DRIVER_H_
#define ISVD_CORE_S_DRIVER_H_

#include <isvd/def.h>
#include <isvd/core/param.h>

#if defined(__cplusplus)
extern "C" {
#endif

/* Replaces isvd_sIsvd (reference core/driver/@x@_isvd.c:106).
 * Selectors (case-insensitive): alg_s "GP" | "GP_gpu"; alg_o "TS" | "GR" (and "TS_gpu", "GR_gpu");
 * alg_i "KN" | "WY" | "HR" (and "_gpu" forms); alg_p "TS" | "GR" | "SY" | "TS_gpu" | "GR_gpu" | "SY_gpu".
 * All four stages run on the GPU.  a, s, ut, vt may be host or device pointers. */
void isvd_sIsvd(
    const isvd_Param param,
    const char *alg_s, const char *alg_o, const char *alg_i, const char *alg_p,
    const isvd_s_val_t *argv[4], const isvd_int_t argc[4], isvd_s_val_t *retv[4], const isvd_int_t retc[4],
    double time[4], FILE *stream,
    const char dista, const char ordera, const isvd_s_val_t *a, const isvd_int_t lda,
    isvd_s_val_t *s, isvd_s_val_t *ut, const isvd_int_t ldut, isvd_s_val_t *vt, const isvd_int_t ldvt,
    const isvd_int_t seed, const mpi_int_t ut_root, const mpi_int_t vt_root
);

#if defined(__cplusplus)
}
#endif

#endif  /* ISVD_CORE_S_DRIVER_H_ */
