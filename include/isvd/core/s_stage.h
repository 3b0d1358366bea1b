/*
 * iSVD stages, single precision (reference src/include/c/isvd/core/@x@_stage.h:21-77).
 *
 * Every routine takes (param, argv, argc, retv, retc, ...): argc < 0 is a default-argument
 * query into retv; argv == NULL / argc == 0 means defaults.  Layouts follow the reference:
 * yst is m_b x Nl row-major, qt is m_b x l row-major, ut/vt row-major, a per dista/ordera.
 * Pointers may be host or device memory; the computation runs on the GPU.
 */
#ifndef ISVD_CORE_S_STAGE_H_
#define ISVD_CORE_S_STAGE_H_

#include <isvd/def.h>
#include <isvd/core/param.h>

#if defined(__cplusplus)
extern "C" {
#endif

/* Replaces isvd_sSketchGaussianProjection (reference core/stage/@x@_sketch_gaussian_projection.c:46):
 * Y = A * Omega for all N sketches, Omega drawn on the GPU (Philox4x32-10 + Box-Muller) from seed. */
void isvd_sSketchGaussianProjection(
    const isvd_Param param, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_s_val_t *retv, const isvd_int_t retc,
    const char dista, const char ordera, const isvd_s_val_t *a, const isvd_int_t lda,
    isvd_s_val_t *yst, const isvd_int_t ldyst, const isvd_int_t seed, const mpi_int_t mpi_root
);

/* Replaces isvd_sOrthogonalizeTallSkinnyQr (reference core/stage/@x@_orthogonalize_tall_skinny_qr.c:36). */
void isvd_sOrthogonalizeTallSkinnyQr(
    const isvd_Param param, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_s_val_t *retv, const isvd_int_t retc,
    isvd_s_val_t *yst, const isvd_int_t ldyst
);

/* Replaces isvd_sOrthogonalizeGramian (reference core/stage/@x@_orthogonalize_gramian.c:33). */
void isvd_sOrthogonalizeGramian(
    const isvd_Param param, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_s_val_t *retv, const isvd_int_t retc,
    isvd_s_val_t *yst, const isvd_int_t ldyst
);

/* Replaces isvd_sIntegrateKolmogorovNagumo (reference core/stage/@x@_integrate_kolmogorov_nagumo.c:42).
 * argv {maxit = 256, tol = 1e-4}; retv {iterations, error}. */
void isvd_sIntegrateKolmogorovNagumo(
    const isvd_Param param, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_s_val_t *retv, const isvd_int_t retc,
    const isvd_s_val_t *yst, const isvd_int_t ldyst, isvd_s_val_t *qt, const isvd_int_t ldqt
);

/* Replaces isvd_sIntegrateWenYin (reference core/stage/@x@_integrate_wen_yin.c:56).
 * argv {maxit 256, tol 1e-3, tau0 1, taumax 1e14, taumin 1e-14, taumaxit 20, beta .5, sigma 1e-4, eta .85};
 * retv {iterations, mu}. */
void isvd_sIntegrateWenYin(
    const isvd_Param param, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_s_val_t *retv, const isvd_int_t retc,
    const isvd_s_val_t *yst, const isvd_int_t ldyst, isvd_s_val_t *qt, const isvd_int_t ldqt
);

/* Replaces isvd_sIntegrateHierarchicalReduction (reference core/stage/@x@_integrate_hierarchical_reduction.c:36).
 * Overwrites yst, as the reference does. */
void isvd_sIntegrateHierarchicalReduction(
    const isvd_Param param, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_s_val_t *retv, const isvd_int_t retc,
    isvd_s_val_t *yst, const isvd_int_t ldyst, isvd_s_val_t *qt, const isvd_int_t ldqt
);

/* Replaces isvd_sPostprocessTallSkinnyQr (reference core/stage/@x@_postprocess_tall_skinny_qr.c:67). */
void isvd_sPostprocessTallSkinnyQr(
    const isvd_Param param, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_s_val_t *retv, const isvd_int_t retc,
    const char dista, const char ordera,
    const isvd_s_val_t *a, const isvd_int_t lda, const isvd_s_val_t *qt, const isvd_int_t ldqt,
    isvd_s_val_t *s, isvd_s_val_t *ut, const isvd_int_t ldut, isvd_s_val_t *vt, const isvd_int_t ldvt,
    const mpi_int_t ut_root, const mpi_int_t vt_root
);

/* Replaces isvd_sPostprocessGramian (reference core/stage/@x@_postprocess_gramian.c:64). */
void isvd_sPostprocessGramian(
    const isvd_Param param, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_s_val_t *retv, const isvd_int_t retc,
    const char dista, const char ordera,
    const isvd_s_val_t *a, const isvd_int_t lda, const isvd_s_val_t *qt, const isvd_int_t ldqt,
    isvd_s_val_t *s, isvd_s_val_t *ut, const isvd_int_t ldut, isvd_s_val_t *vt, const isvd_int_t ldvt,
    const mpi_int_t ut_root, const mpi_int_t vt_root
);

/* Replaces isvd_sPostprocessSymmetric (reference core/stage/@x@_postprocess_symmetric.c:64). */
void isvd_sPostprocessSymmetric(
    const isvd_Param param, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_s_val_t *retv, const isvd_int_t retc,
    const char dista, const char ordera,
    const isvd_s_val_t *a, const isvd_int_t lda, const isvd_s_val_t *qt, const isvd_int_t ldqt,
    isvd_s_val_t *s, isvd_s_val_t *ut, const isvd_int_t ldut, isvd_s_val_t *vt, const isvd_int_t ldvt,
    const mpi_int_t ut_root, const mpi_int_t vt_root
);

#if defined(__cplusplus)
}
#endif

#endif  /* ISVD_CORE_S_STAGE_H_ */
