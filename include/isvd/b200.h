/*
 * B200 extensions of the iSVD API.  None of these has a counterpart in the reference
 * library; they add what the reference cannot express: status codes, a precision mode,
 * a caller-supplied Gaussian test matrix, and status-returning drivers.
 */
#ifndef ISVD_B200_H_
#define ISVD_B200_H_

#include <stddef.h>

#include <isvd/def.h>
#include <isvd/core/param.h>

#if defined(__cplusplus)
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define ISVD_GPU_SUCCESS            0
#define ISVD_GPU_ERROR_ARGUMENT     1  /* invalid argument (selector, layout char, size, leading dim) */
#define ISVD_GPU_ERROR_CUDA         2  /* a CUDA runtime call failed */
#define ISVD_GPU_ERROR_MEMORY       3  /* device or pinned allocation failed */
#define ISVD_GPU_ERROR_TIMEOUT      4  /* a bounded device-side wait expired */
#define ISVD_GPU_ERROR_NUMERICAL    5  /* non-finite values or a matrix iteration that did not converge */
#define ISVD_GPU_ERROR_UNSUPPORTED  6  /* configuration not implemented (e.g. MPI size > 1) */

/* Status of the most recent failing call on this thread (0 if none since the last clear).
 * The void entry points of the reference API report failures here and print the message
 * to stderr, mirroring the reference's print-and-return behaviour for bad arguments. */
int  isvd_gpu_get_last_error( void );
const char *isvd_gpu_get_error_string( void );
void isvd_gpu_clear_error( void );

/* ---------------------------------------------------------------- precision */
#define ISVD_GPU_PRECISION_NATIVE   0  /* products in the routine's own type (FP64 for isvd_d*, FP32 for isvd_s*) */
#define ISVD_GPU_PRECISION_MIXED    1  /* bf16 split products (2 or 3 planes per operand) on tcgen05 tensor
                                          cores, FP32 accumulation; l x l steps (eigensolves, inverse square
                                          roots, small SVDs) in FP64 */

/* Process-wide default precision.  Initial value: ISVD_GPU_PRECISION_NATIVE, or the value
 * of the environment variable ISVD_GPU_PRECISION ("native" / "mixed") at first use. */
void isvd_gpu_set_precision( int mode );
int  isvd_gpu_get_precision( void );

/* ---------------------------------------------------------------- Omega passed in
 * Gaussian projection sketching with a caller-supplied test matrix Omega (n x Nl,
 * row-major, leading dimension ldomega >= Nl; the rows of this rank's column block for
 * dista = 'C').  This is how the reference's own Omega (MKL/LAPACK stream, drawn as
 * r[j*Nl + c] = Omega(j, c), la/vsl/@x@_rng_gaussian_driver.c:16-41) is replayed. */
void isvd_sSketchGaussianProjectionOmega(
    const isvd_Param param, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_s_val_t *retv,
    const isvd_int_t retc, const char dista, const char ordera, const isvd_s_val_t *a, const isvd_int_t lda,
    const isvd_s_val_t *omega, const isvd_int_t ldomega, isvd_s_val_t *yst, const isvd_int_t ldyst
);
void isvd_dSketchGaussianProjectionOmega(
    const isvd_Param param, const isvd_d_val_t *argv, const isvd_int_t argc, isvd_d_val_t *retv,
    const isvd_int_t retc, const char dista, const char ordera, const isvd_d_val_t *a, const isvd_int_t lda,
    const isvd_d_val_t *omega, const isvd_int_t ldomega, isvd_d_val_t *yst, const isvd_int_t ldyst
);

/* ---------------------------------------------------------------- status-returning drivers
 * Same arguments as isvd_?Isvd plus an optional Omega (NULL: drawn on the GPU from seed)
 * and an explicit precision (-1: the process default).  Returns an ISVD_GPU_* status. */
int isvd_sIsvd_ex(
    const isvd_Param param,
    const char *alg_s, const char *alg_o, const char *alg_i, const char *alg_p,
    const isvd_s_val_t *argv[4], const isvd_int_t argc[4], isvd_s_val_t *retv[4], const isvd_int_t retc[4],
    double time[4], FILE *stream,
    const char dista, const char ordera, const isvd_s_val_t *a, const isvd_int_t lda,
    isvd_s_val_t *s, isvd_s_val_t *ut, const isvd_int_t ldut, isvd_s_val_t *vt, const isvd_int_t ldvt,
    const isvd_int_t seed, const mpi_int_t ut_root, const mpi_int_t vt_root,
    const isvd_s_val_t *omega, const isvd_int_t ldomega, const int precision
);
int isvd_dIsvd_ex(
    const isvd_Param param,
    const char *alg_s, const char *alg_o, const char *alg_i, const char *alg_p,
    const isvd_d_val_t *argv[4], const isvd_int_t argc[4], isvd_d_val_t *retv[4], const isvd_int_t retc[4],
    double time[4], FILE *stream,
    const char dista, const char ordera, const isvd_d_val_t *a, const isvd_int_t lda,
    isvd_d_val_t *s, isvd_d_val_t *ut, const isvd_int_t ldut, isvd_d_val_t *vt, const isvd_int_t ldvt,
    const isvd_int_t seed, const mpi_int_t ut_root, const mpi_int_t vt_root,
    const isvd_d_val_t *omega, const isvd_int_t ldomega, const int precision
);

/* Stream on which the library enqueues its work (a cudaStream_t of the current device; NULL
 * restores the library's own non-blocking stream).  Every entry point still returns only after
 * its work on that stream has completed.  Device-memory operands are read in that stream's order:
 * when another stream produced them, either that work has completed before the call (e.g.
 * cudaStreamSynchronize) or the library runs on the producing stream (isvd_gpu_set_stream). */
void  isvd_gpu_set_stream( void *stream );
void *isvd_gpu_get_stream( void );

/* Number of kernels this library has launched since the process started (all devices).
 * Used by benchmarks to report how much of a timed region ran in this library's kernels. */
unsigned long long isvd_gpu_kernel_launch_count( void );

/* Kernel timing.  When enabled, every tcgen05 GEMM launch is bracketed by CUDA events on the
 * library stream and accumulated under its stage tag ("sketch", "block_gram", "gram_full",
 * "project").  isvd_gpu_profile_get returns 0 and fills the total milliseconds, the number of
 * launches and the executed bf16 tensor flops (all plane products) of a tag, or -1 if absent.
 * Enabling it adds a host synchronisation after each such launch: use it outside timed runs. */
void isvd_gpu_profile_enable( int on );
void isvd_gpu_profile_reset( void );
int  isvd_gpu_profile_get( const char *tag, double *ms, unsigned long long *launches, double *flops );

/* ---------------------------------------------------------------- batched solves
 * Many independent matrices of uneven sizes and ranks solved together (no counterpart in the
 * reference): GP / GR / KN / GR with one MPI rank, products in the element type on CUDA cores and
 * FP64 l x l steps, every stage as grouped launches over all matrices.  A batch fixes the shapes
 * (matrix i: m[i] x n[i], rank k[i], oversampling p[i], l = k + p <= 96 and l <= min(m, n); N sketches
 * each) and owns the workspace; NULL on failure (see isvd_gpu_get_last_error).
 * isvd_?BatchIsvd solves every matrix: a[i] (row-major, lda[i] >= n[i]), s[i] (l values), ut[i]
 * (m[i] x l, ldut[i] >= l, k[i] valid columns), vt[i] (n[i] x l, ldvt[i] >= l), all device memory;
 * seed[i] draws the Gaussian test matrix as isvd_?Isvd with that seed; argv / argc: the
 * Kolmogorov-Nagumo arguments {maxit, tol} (defaults 256, 1e-4).  Each matrix stops at its own
 * convergence; iterations[i] and errors[i] (may be NULL) receive the KN iteration count (maxit + 1
 * when exhausted) and error.  The work before and after the iterations is captured as CUDA graphs
 * on the second solve with the same buffers and replayed by later ones.  Returns an ISVD_GPU_* status. */
typedef struct isvd_gpu_batch isvd_gpu_batch;
isvd_gpu_batch *isvd_sBatchCreate(
    const isvd_int_t count, const isvd_int_t *m, const isvd_int_t *n, const isvd_int_t *k, const isvd_int_t *p,
    const isvd_int_t N
);
isvd_gpu_batch *isvd_dBatchCreate(
    const isvd_int_t count, const isvd_int_t *m, const isvd_int_t *n, const isvd_int_t *k, const isvd_int_t *p,
    const isvd_int_t N
);
int isvd_sBatchIsvd(
    isvd_gpu_batch *batch, const isvd_s_val_t *const *a, const isvd_int_t *lda, isvd_s_val_t *const *s,
    isvd_s_val_t *const *ut, const isvd_int_t *ldut, isvd_s_val_t *const *vt, const isvd_int_t *ldvt,
    const isvd_int_t *seed, const isvd_s_val_t *argv, const isvd_int_t argc, isvd_int_t *iterations,
    isvd_s_val_t *errors
);
int isvd_dBatchIsvd(
    isvd_gpu_batch *batch, const isvd_d_val_t *const *a, const isvd_int_t *lda, isvd_d_val_t *const *s,
    isvd_d_val_t *const *ut, const isvd_int_t *ldut, isvd_d_val_t *const *vt, const isvd_int_t *ldvt,
    const isvd_int_t *seed, const isvd_d_val_t *argv, const isvd_int_t argc, isvd_int_t *iterations,
    isvd_d_val_t *errors
);
void isvd_gpu_batch_destroy( isvd_gpu_batch *batch );

/* ---------------------------------------------------------------- truncated-SVD adjoint
 * Gradient of a scalar loss L(U, s, V) with respect to A, where A ~ U diag(s) V' are the k leading
 * singular triplets of A (m x n; s descending, distinct, and s_k > s_(k+1)).  No counterpart in the
 * reference.  Inputs: A stored per ordera ('R' / 'C', leading dimension lda); s (k); U as ut and V
 * as vt, row-major m x k and n x k (the layout of isvd_?Isvd's ut / vt outputs, leading dimensions
 * >= k); the cotangents ds = dL/ds (k), dut = dL/dU (m x k), dvt = dL/dV (n x k), each may be NULL
 * (zero).  Output: da = dL/dA (m x n, stored per ordera, leading dimension ldda).
 *   dA = U J V' + Lam S V' + U Lam' Aperp + U S Gam' + Aperp Gam V',   Aperp = (I - UU') A (I - VV'),
 *   J = diag(ds) + (F o (U'dU - dU'U)) S + S (F o (V'dV - dV'V)),  F_ij = 1 / (s_j^2 - s_i^2),
 *   Lam S^2 - Aperp Aperp' Lam = (I - UU') dU,   Gam S^2 - Aperp' Aperp Gam = (I - VV') dV,
 * the last two solved column by column by conjugate gradients (at most cg_iters iterations each,
 * relative residual tol); cg_iters = 0 uses Lam = (I - UU') dU S^-2 (exact when rank(A) = k).
 * *iterations (may be NULL) receives the CG iterations used (both systems together).  Buffers may
 * be host or device memory.  In MIXED precision (isvd_gpu_set_precision) isvd_sSvdAdjoint runs the
 * products by A and A' on the tensor cores (A in two bf16 planes, the other operand in three);
 * NATIVE keeps them in FP32 on CUDA cores.  Returns an ISVD_GPU_* status. */
int isvd_sSvdAdjoint(
    const isvd_int_t m, const isvd_int_t n, const isvd_int_t k, const char ordera,
    const isvd_s_val_t *a, const isvd_int_t lda, const isvd_s_val_t *s,
    const isvd_s_val_t *ut, const isvd_int_t ldut, const isvd_s_val_t *vt, const isvd_int_t ldvt,
    const isvd_s_val_t *ds, const isvd_s_val_t *dut, const isvd_int_t lddut,
    const isvd_s_val_t *dvt, const isvd_int_t lddvt, isvd_s_val_t *da, const isvd_int_t ldda,
    const int cg_iters, const double tol, int *iterations
);
int isvd_dSvdAdjoint(
    const isvd_int_t m, const isvd_int_t n, const isvd_int_t k, const char ordera,
    const isvd_d_val_t *a, const isvd_int_t lda, const isvd_d_val_t *s,
    const isvd_d_val_t *ut, const isvd_int_t ldut, const isvd_d_val_t *vt, const isvd_int_t ldvt,
    const isvd_d_val_t *ds, const isvd_d_val_t *dut, const isvd_int_t lddut,
    const isvd_d_val_t *dvt, const isvd_int_t lddvt, isvd_d_val_t *da, const isvd_int_t ldda,
    const int cg_iters, const double tol, int *iterations
);

/* ---------------------------------------------------------------- Matrix Market files
 * The file format of the reference's data files (*.mtx) and demo/cdemo.c:51-73 (read there through the
 * NIST mmio library and one isvd_dFget per value).  isvd_?MtxRead stores the size of the matrix in
 * `path` in *m, *n and, when a != NULL, its values in a (ordera 'C': a[i + j*lda], lda >= m;
 * 'R': a[i*lda + j], lda >= n).  Formats "array" (dense, column-major values) and "coordinate"
 * (1-based triplets; omitted entries are zero), fields real / integer / pattern, symmetries
 * general / symmetric / skew-symmetric (mirrored).  The values of a dense file are parsed on all
 * host threads.  isvd_?MtxWrite writes a as "matrix array real general", each value in the
 * shortest decimal form that reads back to it exactly.  Both return an ISVD_GPU_* status
 * (ISVD_GPU_ERROR_ARGUMENT with the reason for a file that cannot be read, written or parsed).
 * No device work. */
int isvd_sMtxRead( const char *path, isvd_int_t *m, isvd_int_t *n, isvd_s_val_t *a, const isvd_int_t lda,
                   const char ordera );
int isvd_dMtxRead( const char *path, isvd_int_t *m, isvd_int_t *n, isvd_d_val_t *a, const isvd_int_t lda,
                   const char ordera );
int isvd_sMtxWrite( const char *path, const isvd_int_t m, const isvd_int_t n, const isvd_s_val_t *a,
                    const isvd_int_t lda, const char ordera );
int isvd_dMtxWrite( const char *path, const isvd_int_t m, const isvd_int_t n, const isvd_d_val_t *a,
                    const isvd_int_t lda, const char ordera );

/* ---------------------------------------------------------------- several ranks without MPI
 * Row-block execution over P processes (one GPU each) whose only exchange is a sum-AllReduce
 * that the caller supplies (NCCL, MPI, gloo ...).  It stands in for the reference's own MPI
 * collectives (MPI_Allreduce in core/stage/@x@_integrate_kolmogorov_nagumo.c:160,178,
 * @x@_integrate_wen_yin.c:206-345, @x@_postprocess_gramian.c:146, ...), which this single-rank
 * build does not call.  After isvd_gpu_set_allreduce(fn, user, nranks, rank, on_device):
 *   - isvd_getMpiSize / isvd_getMpiRank return nranks / rank, so isvd_createParam gives the
 *     reference's row blocks (this rank holds rows [rowidxbegin, rowidxend) = nrow_proc rows);
 *   - with dista 'R' the driver (and the sketch, orthogonalization and integration stages) take
 *     this rank's rows of A, yst and qt, and exchange through fn: the N block Grams (Gramian
 *     orthogonalization; each CholeskyQR pass and the top rows for the sign rule of the
 *     tall-skinny QR), G = Qs'Qs (KN, WY: one exchange per solve
 *     instead of two per iteration; every rank then runs the same iterations on the same G), the
 *     products Q(i)'Q(i+h) of each level of the hierarchical reduction, Z = A'Qbar (Gramian,
 *     tall-skinny QR and symmetric postprocessing; every rank then factors the same Z) and the
 *     l x l W = Qbar'AQbar (symmetric postprocessing);
 *   - outputs as the reference's: ut_root = -1 leaves this rank's rows of U in ut, ut_root >= 0
 *     gathers all m rows on that rank; vt_root = -1 leaves this rank's column block of V
 *     (rows [colidxbegin, colidxend)) in vt, vt_root >= 0 all n rows on that rank (the other
 *     ranks keep their own rows / column block, as after the reference's MPI_Gather);
 *   - fn(buf, count, dtype, stream, user) sums `count` values of type dtype (ISVD_GPU_DTYPE_F32 /
 *     ISVD_GPU_DTYPE_F64) at buf over the ranks, in place.  on_device = 1: buf is device memory
 *     and fn enqueues the reduction on `stream` (a cudaStream_t); on_device = 0: buf is pinned host
 *     memory (the library copies through it and synchronises around the call);
 *   - with dista 'C' (column blocks) each rank passes all m rows of its columns
 *     [colidxbegin, colidxend) of A (and, to the _ex driver, all n rows of Omega): Y = sum of the
 *     ranks' A_j Omega_j is exchanged once (m x Nl) and each rank keeps its rows of Y; the
 *     projection gathers Qbar (m x l) and Z (n x l) through fn as sums of zero-padded copies;
 *   - with nranks > 1 the postprocessing stage called on its own returns
 *     ISVD_GPU_ERROR_UNSUPPORTED.
 * nranks = 1 or fn = NULL returns to single-process execution.  Every rank must make the same
 * calls in the same order. */
#define ISVD_GPU_DTYPE_F32 0
#define ISVD_GPU_DTYPE_F64 1
typedef void (*isvd_gpu_allreduce_fn)( void *buf, size_t count, int dtype, void *stream, void *user );
void isvd_gpu_set_allreduce( isvd_gpu_allreduce_fn fn, void *user, int nranks, int rank, int on_device );

/* ---------------------------------------------------------------- no device allocation
 * Kolmogorov-Nagumo integration in FP64 that allocates no device memory: no cudaMalloc or
 * cudaFree, no stream-ordered pool, no allocating library routine.  It has no counterpart in the
 * reference (whose isvd_dIntegrateKolmogorovNagumo, core/stage/@x@_integrate_kolmogorov_nagumo.c:
 * 97-137, mallocs its workspace on every call); it is for callers that must not allocate once
 * they run, e.g. a process whose device memory is all held by its own pool allocator.
 * Arguments, argv / retv and results as isvd_dIntegrateKolmogorovNagumo, except:
 *   - yst and qt must be device (or managed) memory of the current device;
 *   - the work is enqueued on `stream` (a cudaStream_t of the current device; NULL is the legacy
 *     default stream) and the call returns once it has completed; FP64 whatever the precision mode;
 *   - every intermediate lives in one statically allocated device array of 8 MiB (1,048,576
 *     doubles) per device.  Sizes that do not fit -- (N l)^2 + 5 N l^2 + 13 l^2 + 96 doubles, each
 *     term rounded up to 32 -- or l > 160 are rejected with ISVD_GPU_ERROR_ARGUMENT and a message
 *     (N l = 512 with l = 64 fits; N l = 1024 does not).
 *   - one rank only: with ranks joined by isvd_gpu_set_allreduce, or param.mpi_size != 1, it returns
 *     ISVD_GPU_ERROR_UNSUPPORTED (it never sums the Gram over ranks);
 *   - the call is synchronous: it reads the iteration error back on the host after every iteration
 *     and returns only once all of its work on `stream` has completed.
 * The first call on each device sets up: it looks up the array's address (which loads the device
 * code that holds it), reads the SM count and resolves every kernel the entry point can launch, so
 * that with lazy module loading no later call, whatever its shape, loads code; make that first call
 * before any stream capture on the device.  Nothing in the array has to be zero on entry: each call
 * clears its own status and barrier words.  The array is shared by all calls on a device, so
 * overlapping calls would race on it; each call holds the library's process-wide lock until its
 * work has completed, which makes calls from several threads or streams run one after another.
 * Returns an ISVD_GPU_* status. */
int isvd_dIntegrateKolmogorovNagumo_noalloc(
    const isvd_Param param, const isvd_d_val_t *argv, const isvd_int_t argc, isvd_d_val_t *retv,
    const isvd_int_t retc, const isvd_d_val_t *yst, const isvd_int_t ldyst, isvd_d_val_t *qt,
    const isvd_int_t ldqt, void *stream
);

#if defined(__cplusplus)
}
#endif

#endif  /* ISVD_B200_H_ */
