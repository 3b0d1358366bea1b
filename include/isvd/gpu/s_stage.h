/*
 * GPU-named stages, single precision (reference src/include/c/isvd/gpu/@x@_stage.h:28-90).
 * Same implementation as the CPU-named stages in <isvd/core/s_stage.h>; kept so that
 * selector strings and direct calls written for isvd_gpu_magma keep working.
 */
#ifndef ISVD_GPU_S_STAGE_H_
#define ISVD_GPU_S_STAGE_H_

#include <isvd/def.h>
#include <isvd/core/param.h>

#if defined(__cplusplus)
extern "C" {
#endif

/* Replaces isvd_sSketchGaussianProjection_gpu (reference gpu/stage/@x@_sketch_gaussian_projection_gpu.c). */
void isvd_sSketchGaussianProjection_gpu(
    const isvd_Param param, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_s_val_t *retv, const isvd_int_t retc,
    const char dista, const char ordera, const isvd_s_val_t *a, const isvd_int_t lda,
    isvd_s_val_t *yst, const isvd_int_t ldyst, const isvd_int_t seed, const mpi_int_t mpi_root
);

/* Replaces isvd_sPostprocessTallSkinnyQr_gpu (reference gpu/stage/@x@_postprocess_tall_skinny_qr_gpu.c). */
void isvd_sPostprocessTallSkinnyQr_gpu(
    const isvd_Param param, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_s_val_t *retv, const isvd_int_t retc,
    const char dista, const char ordera,
    const isvd_s_val_t *a, const isvd_int_t lda, const isvd_s_val_t *qt, const isvd_int_t ldqt,
    isvd_s_val_t *s, isvd_s_val_t *ut, const isvd_int_t ldut, isvd_s_val_t *vt, const isvd_int_t ldvt,
    const mpi_int_t ut_root, const mpi_int_t vt_root
);

/* Replaces isvd_sPostprocessGramian_gpu (reference gpu/stage/@x@_postprocess_gramian_gpu.c). */
void isvd_sPostprocessGramian_gpu(
    const isvd_Param param, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_s_val_t *retv, const isvd_int_t retc,
    const char dista, const char ordera,
    const isvd_s_val_t *a, const isvd_int_t lda, const isvd_s_val_t *qt, const isvd_int_t ldqt,
    isvd_s_val_t *s, isvd_s_val_t *ut, const isvd_int_t ldut, isvd_s_val_t *vt, const isvd_int_t ldvt,
    const mpi_int_t ut_root, const mpi_int_t vt_root
);

/* Replaces isvd_sPostprocessSymmetric_gpu (reference gpu/stage/@x@_postprocess_symmetric_gpu.c). */
void isvd_sPostprocessSymmetric_gpu(
    const isvd_Param param, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_s_val_t *retv, const isvd_int_t retc,
    const char dista, const char ordera,
    const isvd_s_val_t *a, const isvd_int_t lda, const isvd_s_val_t *qt, const isvd_int_t ldqt,
    isvd_s_val_t *s, isvd_s_val_t *ut, const isvd_int_t ldut, isvd_s_val_t *vt, const isvd_int_t ldvt,
    const mpi_int_t ut_root, const mpi_int_t vt_root
);

#if defined(__cplusplus)
}
#endif

#endif  /* ISVD_GPU_S_STAGE_H_ */
