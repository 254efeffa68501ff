/*
 * mnpbem_b200 -- C ABI of the B200 boundary-element hot path.
 *
 * Plain C types only: device pointers are raw addresses of caller-owned
 * device memory (the library never frees caller memory), host pointers are
 * host memory, sizes are int64_t, streams are cudaStream_t passed as void*.
 * Every entry point returns 0 on success or one of the MNPB_E* codes; the
 * message of the last failure on the calling thread is returned by
 * mnpb_last_error().  No entry point falls back to the CPU.
 *
 * Layouts (all column-major, "ld" = leading dimension in elements):
 *   c128 matrix  : interleaved complex double, element (i,j) at 2*(j*ld+i)
 *   c32p matrix  : planar complex float, a real plane then an imaginary
 *                  plane, each n x n with leading dimension ld; the planes
 *                  are `plane` elements apart
 *   batches      : `batch` matrices `stride` elements apart
 *
 * The reference (PyMNPBEM) has no native interface; each entry point below
 * names the reference Python function whose arithmetic it replaces.  The
 * Python classes in mnpbem_b200/ (BEMRet, BEMStat, CompGreenRet, ...) keep
 * the reference call surface and call these functions through ctypes.
 */
#ifndef MNPBEM_B200_H
#define MNPBEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MNPB_OK 0
#define MNPB_EINVAL 1      /* invalid argument (null pointer, bad size)     */
#define MNPB_ECUDA 2       /* CUDA runtime / launch error                  */
#define MNPB_ESINGULAR 3   /* exactly zero pivot met during factorisation  */
#define MNPB_ENOCONV 4     /* iterative method did not reach its tolerance */
#define MNPB_ETIMEOUT 5    /* a bounded device-side wait gave up           */
#define MNPB_ENOMEM 6      /* workspace too small                          */

/* Library version (major*10000 + minor*100 + patch). */
int mnpb_version(void);

/* Text of the last error on the calling thread ("" if none). */
const char *mnpb_last_error(void);

/* Number of kernel launches issued by this library since load (host-side
 * counter; used to report how many of the library's kernels ran). */
int64_t mnpb_launch_count(void);

/* Device-time profiling of the library's own launches: between
 * mnpb_prof_begin() and mnpb_prof_end() every launch of a profiled kernel is
 * bracketed by CUDA events on its stream.  mnpb_prof_end synchronises and
 * returns, per kernel class (0 assembly, 1 refinement quadrature, 2 FP64
 * GEMM, 3 LU panel, 4 small triangular solves, 5 row/column swaps,
 * 6 element-wise, 7 tensor-core GEMM, 8 far field, 9 FP32 GEMM, 10 matvec,
 * 11 one-launch triangular solves, 12 tensor-core operand packing,
 * 13 refinement element-wise),
 * the summed device time in ms, the summed algorithmic work (flops or bytes,
 * see the kernel) and the number of launches. */
int mnpb_prof_begin(void);
int mnpb_prof_end(int ncls, double *ms, double *work, int64_t *count);
/* Write every launch of the last profiled interval to a CSV file
 * (class, ms, work, shape tag). */
int mnpb_prof_dump(const char *path);

/* ---------------------------------------------------------------------------
 * Geometry set-up (once per particle mesh)
 * ------------------------------------------------------------------------- */

/* Near/self classification of face pairs, host side, integer-exact.
 * Replaces mnpbem/greenfun/refine_utils.py:29 refinematrix (and its twin
 * mnpbem/greenfun/utils.py:43).  pos*: n x 3 row-major doubles, rad*:
 * boundary-element radii (rad1 may be NULL: sources without a radius, such as
 * points, are measured in units of rad2, the reference's fallback at
 * refine_utils.py:97-101).  Writes CSR rows (row_ptr n1+1), column indices
 * and kinds (1 near, 2 self) for up to `cap` pairs; *nnz receives the total
 * count.  Returns MNPB_ENOMEM (after setting *nnz) if cap is too small. */
int mnpb_refinematrix(int64_t n1, int64_t n2, const double *pos1, const double *pos2,
                      const double *rad1, const double *rad2, double abs_cutoff,
                      double rel_cutoff, int64_t cap, int64_t *nnz, int64_t *row_ptr,
                      int32_t *cols, int8_t *kinds);

/* Refined Green-function Taylor coefficients on the GPU (FP64).
 * Replaces mnpbem/greenfun/greenret_refined.py:122-516 (_refine_diagonal and
 * _refine_offdiagonal, deriv='cart', order 5) and the static refinement of
 * mnpbem/greenfun/compgreen_stat.py:327-416.
 * Device inputs: face data pos/nvec/tvec1/tvec2 (n x 3 row-major), pair list
 * rows/cols/kinds (nref), face-quadrature points qpos (P x 3), weights qw and
 * per-face offsets qoff (n+1), polar points ppos/pw/poff likewise.
 * Device outputs: g (nref x 6), f (nref x 3 x 6) real Taylor coefficients,
 * gstat, fstat (nref) static G and F values of the refined pairs. */
int mnpb_refine_coefficients(void *stream, int64_t n, const double *pos, const double *nvec,
                             const double *tvec1, const double *tvec2, int64_t nref,
                             const int32_t *rows, const int32_t *cols, const int8_t *kinds,
                             const double *qpos, const double *qw, const int64_t *qoff,
                             const double *ppos, const double *pw, const int64_t *poff,
                             double *g, double *f, double *gstat, double *fstat);

/* Adds the closed-surface correction corr_i nvec_i to f[:, :, 0] of the self
 * pairs, corr_i = -2 pi cdir_i - fsum_i on faces with cdir_i = +-1 (the
 * normal direction of their closed surface; 0 = not closed; cdir may be
 * NULL), and writes fn[:, m] = nvec_row . f[:, :, m].
 * Replaces mnpbem/greenfun/compgreen_ret.py:376-400 (_apply_diag_corrections)
 * and the nvec contraction of greenret_refined.py:769-774. */
int mnpb_refine_finalize(void *stream, int64_t n, int64_t nref, const int32_t *rows,
                         const int32_t *cols, const double *nvec, const double *cdir,
                         const double *fsum, double *f, double *fn);

/* Closed-surface sums f_j = sum_i a_i F_ij / a_j of the refined static F over
 * the closed surface of face j (rows grp_lo[j]..grp_hi[j]-1).  Replaces
 * mnpbem/greenfun/compgreen_ret.py:302-356 (_fun_closed).  The refined pairs
 * are passed column-sorted (CSC: cptr n+1, crows, cfstat). */
int mnpb_closure_sums(void *stream, int64_t n, const double *pos, const double *nvec,
                      const double *area, const int64_t *grp_lo, const int64_t *grp_hi,
                      const int64_t *cptr, const int32_t *crows, const double *cfstat,
                      double *fsum);

/* Full refined quasistatic F (n x n real, column-major) with the closure
 * term -2 pi cdir_i - fsum_i added on the diagonal of closed faces.  Replaces
 * mnpbem/greenfun/compgreen_stat.py:219-294 (+ _handle_closed_surfaces).
 * Refined pairs in CSR (rptr, rcols, rfstat). */
int mnpb_static_matrix(void *stream, int64_t n, const double *pos, const double *nvec,
                       const double *area, const int64_t *rptr, const int32_t *rcols,
                       const double *rfstat, const double *cdir, const double *fsum, double *F,
                       int64_t ld);

/* ---------------------------------------------------------------------------
 * Per-wavelength retarded assembly (batched over wavelengths)
 * ------------------------------------------------------------------------- */

/* Writes G1, H1, G2, H2 for `batch` wavelengths.  Replaces
 * mnpbem/bem/bem_ret.py:407-423 with mnpbem/greenfun/compgreen_ret.py:739-858
 * and greenret_refined.py:654-810 (G = a/d, F = n.r (ik-1/d)/d^2 a, refined
 * overlay sum_n c_n (ik)^n, phase exp(ikd), H = F +- 2 pi on the diagonal).
 * Particle blocks: nparts particles, face offsets poff (nparts+1, host).
 * kblk (device): batch x 2 x nparts x nparts complex wavenumbers (re,im)
 * for side 1 (G1/H1) and side 2 (G2/H2); sblk (device, same shape) real
 * signs (+1, -1 or 0 = block absent).
 * Refined pairs: nref, rows, cols, g (nref x 6), fn (nref x 6) where
 * fn[:, m] = n_row . f[:, :, m].
 * out_mode 0: c128 outputs (G1,H1,G2,H2 pointers, ld, stride).
 * out_mode 1: c32p outputs (planar float; plane offset `plane`). */
int mnpb_assemble_ret(void *stream, int64_t n, int64_t batch, const double *pos,
                      const double *nvec, const double *area, int nparts, const int64_t *poff,
                      const double *kblk, const double *sblk, int64_t nref, const int32_t *rows,
                      const int32_t *cols, const double *g, const double *fn, int out_mode,
                      void *G1, void *H1, void *G2, void *H2, int64_t ld, int64_t stride,
                      int64_t plane);

/* ---------------------------------------------------------------------------
 * Dense retarded solve (BEMRet), FP64, batched over wavelengths
 * ------------------------------------------------------------------------- */

/* Workspace bytes needed by mnpb_bemret_init_f64 for (n, batch). */
int64_t mnpb_bemret_workspace_f64(int64_t n, int64_t batch);

/* In place: G1 -> LU(G1), G2 -> LU(G2), H1 -> Sigma1 = H1 G1^-1,
 * H2 -> Sigma (combined, LU-factorised), D -> Delta^-1.
 * Replaces mnpbem/bem/bem_ret.py:437-523 (init).  eps (device, batch x 2
 * complex): inside / outside dielectric constants (scalar per wavelength);
 * kvac (device, batch) vacuum wavenumbers 2 pi / enei; nvec (device n x 3)
 * face normals of batch entry b at nvec + b * nvec_stride (stride 0: one
 * particle for every entry, a wavelength sweep; stride 3 n: a batch of
 * different particles with the same face count -- this holds for
 * mnpb_bemret_excitation, _solve_f64, _init_mixed and _solve_refine too).
 * piv (device int32, [3][batch][n]) receives the pivots of G1, G2, Sigma.
 * All matrices c128, leading dimension ld, batch stride `stride`.  When G2
 * follows G1 (G2 == G1 + batch*stride) and H2 follows H1 the two halves are
 * factorised together, as one batch of 2 x batch matrices.
 * info (device int32, [2][batch]) receives the first zero pivot (1-based) or 0. */
int mnpb_bemret_init_f64(void *stream, int64_t n, int64_t batch, double *G1, double *G2,
                         double *H1, double *H2, double *D, int64_t ld, int64_t stride,
                         const double *eps, const double *kvac, const double *nvec, int64_t nvec_stride,
                         int32_t *piv, int32_t *info, void *work, int64_t work_bytes);

/* Excitation variables phi, a, alpha, De (x_in layout of the solve) from
 * the potentials of a batch of excitations.  Replaces
 * mnpbem/bem/bem_ret.py:1360-1429 (_excitation).  pots (device c128,
 * [batch][16][nrhs][n]): phi1, phi1p, a1 (x,y,z), a1p (x,y,z), phi2, phi2p,
 * a2 (x,y,z), a2p (x,y,z). */
/* Entries of different face counts in one batch: entry e keeps its n_e x n_e
 * matrices (n_of_entry, device int32) in the top-left corner of npad x npad
 * buffers; everything else becomes identity padding -- G1 = G2 = H1 = I,
 * H2 = 0 on the pad block, no coupling -- in the c128 matrices (ld, stride)
 * and their planar FP32 copies (ldp, planep, stridep).  The factorisations
 * and solves then treat the entries as one batch and return zeros on the
 * pad (with zero normals and zero right-hand sides there).  No reference
 * counterpart (the reference solves one particle at a time). */
int mnpb_pad_entries(void *stream, int64_t npad, int64_t batch, const int32_t *n_of_entry,
                     double *G1, double *G2, double *H1, double *H2, int64_t ld, int64_t stride,
                     float *G1p, float *G2p, float *H1p, float *H2p, int64_t ldp,
                     int64_t planep, int64_t stridep);

int mnpb_bemret_excitation(void *stream, int64_t n, int64_t batch, int64_t nrhs,
                           const double *pots, const double *eps, const double *kvac,
                           const double *nvec, int64_t nvec_stride, double *x_in);

/* Surface charges/currents for nrhs excitations per wavelength.
 * Replaces mnpbem/bem/bem_ret.py:1690-1810 (solve, Eqs. 19-20 of Garcia de
 * Abajo & Howie).  In (device, c128, batch-major): phi (n x nrhs), a (n x 3 x
 * nrhs), alpha (n x 3 x nrhs), De (n x nrhs) -- stored as one block
 * x_in[batch][8][nrhs][n] in the order phi, a_x, a_y, a_z, De, alpha_x..z.
 * Out: x_out[batch][8][nrhs][n] in the order sig1, h1x..z, sig2, h2x..z. */
int mnpb_bemret_solve_f64(void *stream, int64_t n, int64_t batch, int64_t nrhs,
                          const double *G1, const double *G2, const double *S1,
                          const double *S, const double *D, int64_t ld, int64_t stride,
                          const int32_t *piv, const double *eps, const double *kvac,
                          const double *nvec, int64_t nvec_stride, const double *x_in, double *x_out,
                          void *work, int64_t work_bytes);

/* As mnpb_assemble_ret, writing in one pass both the c128 matrices (ld,
 * stride) and planar FP32 copies (ldp, stridep, planep) -- the FP64 operator
 * for refinement and the FP32 input of the mixed-precision factorisation. */
int mnpb_assemble_ret2(void *stream, int64_t n, int64_t batch, const double *pos,
                       const double *nvec, const double *area, int nparts, const int64_t *poff,
                       const double *kblk, const double *sblk, int64_t nref, const int32_t *rows,
                       const int32_t *cols, const double *g, const double *fn, double *G1,
                       double *H1, double *G2, double *H2, int64_t ld, int64_t stride,
                       float *G1p, float *H1p, float *G2p, float *H2p, int64_t ldp,
                       int64_t stridep, int64_t planep);

/* ---------------------------------------------------------------------------
 * Dense retarded solve (BEMRet), mixed precision, batched over wavelengths
 * ------------------------------------------------------------------------- */

/* Workspace bytes of mnpb_bemret_init_mixed. */
int64_t mnpb_bemret_workspace_mixed(int64_t n, int64_t batch);

/* The algebra of mnpb_bemret_init_f64 on planar FP32 matrices (leading
 * dimension ld, a multiple of 4; plane = ld*n; batch stride 2*ld*n) with
 * every LU, triangular solve and GEMM on TF32 tensor cores: G1 -> LU(G1),
 * G2 -> LU(G2), H1 -> Sigma1, H2 -> LU(Sigma), D -> Delta^-1.  Factor
 * values are stored rounded to nearest TF32.  From the second call with the
 * same sizes, buffers and device on, the launch sequence is captured once as
 * a CUDA graph (on a stream of the library's own) and replayed on `stream`;
 * calls made while `stream` is being captured by the caller issue the plain
 * launches.  Replaces mnpbem/bem/bem_ret.py:437-523 in the mixed-precision
 * solver. */
int mnpb_bemret_init_mixed(void *stream, int64_t n, int64_t batch, float *G1, float *G2,
                           float *H1, float *H2, float *D, int64_t ld, const double *eps,
                           const double *kvac, const double *nvec, int64_t nvec_stride, int32_t *piv, int32_t *info,
                           float *dinv, void *work, int64_t work_bytes);

/* Floats of the dinv buffer (inverses of the 32 x 32 diagonal blocks of the
 * G1, G2 and Sigma factors, written by mnpb_bemret_init_mixed and read by
 * mnpb_bemret_solve_refine's one-launch triangular solves). */
int64_t mnpb_bemret_dinv_floats(int64_t n, int64_t batch);

/* Workspace bytes of mnpb_bemret_solve_refine. */
int64_t mnpb_bemret_refine_workspace(int64_t n, int64_t batch, int64_t nrhs);

/* Solve with the mixed factorisation and refine in FP64 against the exact
 * operator of mnpbem/bem/bem_ret_iter.py:1362-1501 (c128 G1, G2, H1, H2 with
 * the same ld): x = M^-1 b, then dx = M^-1 (b - A x), x += dx, per batch
 * entry until |dx| / |x| < tol (a forward-error test) or max_iter
 * corrections (MNPB_ENOCONV then).  b: excitation layout (phi, a, De,
 * alpha), x: solution layout (sig1, h1, sig2, h2), both [batch][8][nrhs][n]
 * c128, nrhs <= 4.  iters (corrections applied) and relres (|b - A x| / |b|
 * of the iterate before the last correction, normally above the final
 * one): host arrays (batch). */
int mnpb_bemret_solve_refine(void *stream, int64_t n, int64_t batch, int64_t nrhs,
                             const float *G1p, const float *G2p, const float *S1p,
                             const float *Sp, const float *Dp, int64_t ld, const int32_t *piv,
                             const float *dinv, const double *G1, const double *G2, const double *H1,
                             const double *H2, const double *eps, const double *kvac,
                             const double *nvec, int64_t nvec_stride, const double *b, double *x, int max_iter,
                             double tol, int32_t *iters, double *relres, void *work,
                             int64_t work_bytes);

/* Batched LU / LU solve of planar FP32 matrices with TF32 tensor-core
 * updates (recursive LU; triangular solves with >= 128 right-hand sides apply
 * the 128 x 128 diagonal blocks through their inverses, also on the tensor
 * cores).  Leading dimensions, planes and strides are multiples of 4 floats
 * and base pointers 16-byte aligned (tensor-core operand rule).
 * work: mnpb_f32_workspace(n, batch) bytes. */
int64_t mnpb_f32_workspace(int64_t n, int64_t batch);
int mnpb_getrf_c32p(void *stream, int64_t n, int64_t batch, float *A, int64_t ld, int64_t plane,
                    int64_t stride, int32_t *piv, int64_t pstride, int32_t *info, void *work,
                    int64_t work_bytes);
/* X = A^-1 from mnpb_getrf_c32p's output (U^-1 L^-1 P^T): the forward solve
 * against the identity skips the identity's zero upper part and takes the
 * leaves from the diagonal-block inverses.  Replaces the Delta^-1 of
 * mnpbem/bem/bem_ret.py:476-479 (lu_solve on the identity).  Same layout
 * rules and workspace as mnpb_getrs_c32p. */
int mnpb_getri_c32p(void *stream, int64_t n, int64_t batch, const float *LU, int64_t ld,
                    int64_t plane, int64_t stride, const int32_t *piv, int64_t pstride, float *X,
                    int64_t ldx, int64_t planeX, int64_t xstride, void *work,
                    int64_t work_bytes);
int mnpb_getrs_c32p(void *stream, int64_t n, int64_t batch, int64_t nrhs, const float *LU,
                    int64_t ld, int64_t plane, int64_t stride, const int32_t *piv,
                    int64_t pstride, float *B, int64_t ldb, int64_t planeB, int64_t bstride,
                    void *work, int64_t work_bytes);

/* ---------------------------------------------------------------------------
 * Dense building blocks (exposed for tests and for the quasistatic solver)
 * ------------------------------------------------------------------------- */

/* Batched complex LU with partial pivoting (FP64, c128).  Replaces
 * scipy.linalg.lu_factor as called from mnpbem/utils/gpu.py:145
 * (lu_factor_dispatch).  piv: 0-based row interchanges, LAPACK order. */
int mnpb_getrf_f64(void *stream, int64_t n, int64_t batch, double *A, int64_t ld,
                   int64_t stride, int32_t *piv, int64_t pstride, int32_t *info);

/* Batched LU solve A X = B for nrhs right-hand sides (c128, in place on B).
 * Replaces scipy.linalg.lu_solve (mnpbem/utils/gpu.py:194). */
int mnpb_getrs_f64(void *stream, int64_t n, int64_t batch, int64_t nrhs, const double *LU,
                   int64_t ld, int64_t stride, const int32_t *piv, int64_t pstride,
                   double *B, int64_t ldb, int64_t bstride);

/* Batched complex GEMM C = alpha A B + beta C (c128, column-major). */
int mnpb_zgemm(void *stream, int64_t m, int64_t n, int64_t k, int64_t batch,
               double alpha_re, double alpha_im, const double *A, int64_t lda, int64_t sA,
               const double *B, int64_t ldb, int64_t sB, double beta_re, double beta_im,
               double *C, int64_t ldc, int64_t sC);

/* Batched complex GEMM on the tensor cores (tcgen05, TF32 inputs rounded to
 * nearest, FP32 accumulation): C = beta C + alpha A B for planar complex FP32
 * column-major matrices (A: m x k, B: k x n).  Base addresses, ld*4 and
 * plane*4, stride*4 must be multiples of 16 bytes.  work: at least
 * mnpb_cgemm_tf32_workspace(m, k, batch) bytes of device memory.  Replaces
 * the complex GEMMs of mnpbem/bem/bem_ret.py:472-495 and the LU trailing
 * updates of scipy.linalg.lu_factor in the mixed-precision solver. */
int64_t mnpb_cgemm_tf32_workspace(int64_t m, int64_t k, int64_t batch);
int mnpb_cgemm_tf32(void *stream, int64_t m, int64_t n, int64_t k, int64_t batch, float alpha,
                    const float *A, int64_t lda, int64_t planeA, int64_t sA, const float *B,
                    int64_t ldb, int64_t planeB, int64_t sB, float beta, float *C, int64_t ldc,
                    int64_t planeC, int64_t sC, void *work, int64_t work_bytes);

/* mnpb_cgemm_tf32 with options (`flags`, an OR of the bits below):
 *   MNPB_GEMM_A_TF32  A already holds TF32 values (the low 13 mantissa bits
 *                     zero): the tensor cores read A in place from the
 *                     column-major matrix (MN-major operand, no pack, `work`
 *                     may be NULL).  A, lda, planeA and sA must be multiples
 *                     of 16 bytes.  This is how the mixed factorisation
 *                     applies its stored (TF32-rounded) factors.
 *   MNPB_GEMM_ROUND_C store C rounded to nearest TF32.
 * Replaces the same cuBLAS zgemm calls as mnpb_cgemm_tf32. */
#define MNPB_GEMM_A_TF32 1
#define MNPB_GEMM_ROUND_C 2
int mnpb_cgemm_tf32_ex(void *stream, int64_t m, int64_t n, int64_t k, int64_t batch, float alpha,
                       const float *A, int64_t lda, int64_t planeA, int64_t sA, const float *B,
                       int64_t ldb, int64_t planeB, int64_t sB, float beta, float *C,
                       int64_t ldc, int64_t planeC, int64_t sC, void *work, int64_t work_bytes,
                       int32_t flags);

/* Launch configuration of the tensor-core GEMMs (process-wide, for the
 * autotuner; no reference counterpart): bn_wide (64 or 128) the tile width for
 * N > 64, persist_tiles_per_sm the tile count per SM from which the persistent
 * kernel is used (0: never), stages the operand-ring depth (0: as many as fit,
 * else 2..4, capped by shared memory).  Defaults 128, 2, 0.  Takes effect for
 * launches issued afterwards; cached factorisation graphs are rebuilt. */
int mnpb_gemm_config(int32_t bn_wide, int32_t persist_tiles_per_sm, int32_t stages);
/* A operand that holds TF32 values (MNPB_GEMM_A_TF32 and the factorisation's
 * stored factors) is packed K-major first instead of being read in place
 * when 64 < N < mn_min_n and a workspace is at hand (exact for TF32 values).
 * Default 0: always in place (over the 2884-face, 81-wavelength sweep the
 * packing costs more than the in-place reads lose). */
int mnpb_gemm_config_mn(int32_t mn_min_n);

/* Same GEMM as mnpb_cgemm_tf32, but it allocates nothing and takes no
 * workspace: the packed TF32 copy of A goes into a fixed 64 MiB array of the
 * library's static device memory (one per device, reserved when the module
 * loads).  No counterpart in the reference, which has no GPU path; it is for
 * callers that cannot provide device memory (a foreign-language host without
 * a device allocator, a pool that owns the whole GPU, a loop that must not
 * synchronise the device through cudaMalloc/cudaFree).
 *   - Limit: mnpb_cgemm_tf32_workspace(m, k, batch) <= 67108864 bytes, else
 *     MNPB_ENOMEM with the sizes in mnpb_last_error() and nothing launched.
 *   - The first call on each device does the setup (address lookup of the
 *     array; the first launch of each kernel on a device also raises its
 *     shared-memory limit there); make it before any stream capture.
 *   - `stream` must belong to the current device (the array used is the
 *     current device's); a stream of another device gives MNPB_EINVAL.
 *   - Nothing has to be zeroed beforehand: every scratch element is written
 *     before it is read.
 *   - Calls that overlap in time on one device (other streams, other host
 *     threads) share the array and race; calls ordered on one stream do not. */
int mnpb_cgemm_tf32_noalloc(void *stream, int64_t m, int64_t n, int64_t k, int64_t batch,
                            float alpha, const float *A, int64_t lda, int64_t planeA, int64_t sA,
                            const float *B, int64_t ldb, int64_t planeB, int64_t sB, float beta,
                            float *C, int64_t ldc, int64_t planeC, int64_t sC);

/* First bounded-wait timeout recorded by a tensor-core kernel since the last
 * call (0 = none); reading clears it. */
int mnpb_tc_error(void *stream, int32_t *code);

/* Failure-path check of the bounded device waits (no reference counterpart:
 * the reference's GPU path catches exceptions and falls back to the CPU,
 * mnpbem/bem/bem_ret.py:321-355).  Launches one thread that waits, with the
 * helper the kernels use, on something nothing completes -- kind 0: an
 * mbarrier (tensor-core GEMM), kind 1: a flag spin (`flag`, one device int,
 * triangular solve), kind 2: an mbarrier (streamed triangular solve) -- for
 * at most limit_ns (<= 2e9).  The wait gives up, records its error word like
 * a kernel would, and returns; the probe then reads and clears the word and
 * returns MNPB_ETIMEOUT with a message.  The device context stays usable. */
int mnpb_wait_probe(void *stream, int32_t kind, int64_t limit_ns, int32_t *flag);

/* Quasistatic matrix for a batch of wavelengths: M_b = -(diag(lambda_b) + F)
 * with lambda = 2 pi (eps1+eps2)/(eps1-eps2) per face (eps12: device,
 * batch x n x 2 complex).  Replaces mnpbem/bem/bem_stat.py:318-330. */
int mnpb_stat_matrix(void *stream, int64_t n, int64_t batch, const double *F, int64_t ldf,
                     const double *eps12, double *M, int64_t ld, int64_t stride);

/* ---------------------------------------------------------------------------
 * Green functions of one region pair, entry by entry, and their products
 * ------------------------------------------------------------------------- */

/* Keys of mnpb_green_eval / mnpb_green_apply (compgreen_ret.py:507-553). */
#define MNPB_KEY_G 0
#define MNPB_KEY_F 1
#define MNPB_KEY_H1 2
#define MNPB_KEY_H2 3
#define MNPB_KEY_GP 4   /* Cartesian derivative, 3 components */
#define MNPB_KEY_H1P 5
#define MNPB_KEY_H2P 6

/* Entries of the region-pair Green function for `key` at one wavelength.
 * Replaces mnpbem/greenfun/compgreen_ret.py:507-738 (eval, eval_block, and
 * eval with `ind`, _eval2 / eval_ind at 859-908, 1770-1857) with the entries
 * of greenret_refined.py:654-867; with kblk = 0 the quasistatic entries of
 * mnpbem/greenfun/compgreen_stat.py:678-990 (CompGreenStat.eval).
 * Tables (device): face data, particle offsets poff (host, nparts+1), kblk
 * (nparts x nparts complex, re/im) and sblk (nparts x nparts; 0 = block not
 * connected) of the region pair, the refined pairs as CSR (rptr n+1, cols
 * ascending within a row) with g (nref x 6), fn (nref x 6), f (nref x 3 x 6).
 * ind == NULL: columns [col_start, col_start + ncol), out row-major complex
 * (n x ncol), or (n x 3 x ncol) for vector keys.  Otherwise the nind entries
 * at row-major linear indices ind (device int64, i * n + j): out (nind) or
 * (nind x 3). */
int mnpb_green_eval(void *stream, int64_t n, const double *pos, const double *nvec,
                    const double *area, int nparts, const int64_t *poff, const double *kblk,
                    const double *sblk, const int64_t *rptr, const int32_t *cols,
                    const double *g, const double *fn, const double *f, int key,
                    int64_t col_start, int64_t ncol, const int64_t *ind, int64_t nind,
                    double *out);

/* Products with the region-pair Green function, entries computed on the fly
 * (no n x n storage), for potentials and fields at the faces.  Replaces the
 * matmul / cross of mnpbem/greenfun/compgreen_ret.py:912-1136 (field,
 * potential).  x, y device, row-major complex:
 *   mode 0, scalar key: y (n x m)     = M x, x (n x m), m <= 12
 *   mode 1, vector key: y (n x 3 x m) = Gp x, x (n x m), m <= 4
 *   mode 2, vector key: y (n x 3 x m) = sum_j Gp_ij cross x_j, x (n x 3 x m),
 *                       m <= 4. */
int mnpb_green_apply(void *stream, int64_t n, const double *pos, const double *nvec,
                     const double *area, int nparts, const int64_t *poff, const double *kblk,
                     const double *sblk, const int64_t *rptr, const int32_t *cols,
                     const double *g, const double *fn, const double *f, int key, int mode,
                     int64_t m, const double *x, double *y);

/* ---------------------------------------------------------------------------
 * Mirror symmetry (FP64): the irreducible part (n faces) of a particle that
 * its nk = 2 or 4 mirror images complete.  An "entry" is one wavelength and
 * one symmetry value, entry e = b * nsym + s; matrices of an entry are
 * `stride` complex elements apart, column-major with leading dimension ld.
 * ------------------------------------------------------------------------- */

/* out(b, s)[i, j] = sum_k tab[s * nk + k] full(b)[i, j + k n] for i, j < n:
 * the Green function of symmetry value s from the full particle's matrix
 * (ldf >= nk n, batch stride sf); tab (nsym x nk) is a host array.
 * Replaces mnpbem/greenfun/compgreen_ret_mirror.py:36-95 (eval). */
int mnpb_mirror_contract(void *stream, int64_t n, int64_t nk, int64_t nsym, int64_t batch,
                         const double *full, int64_t ldf, int64_t sf, const double *tab,
                         double *out, int64_t ld, int64_t stride);

/* Workspace of mnpb_bemret_init_mirror_f64 in bytes. */
int64_t mnpb_bemret_mirror_workspace(int64_t n, int64_t entries);
/* Per entry: LU(G1), LU(G2) in place, H1 <- Sigma1 = H1 G1^-1, H2 <- Sigma2 =
 * H2 G2^-1, Dinv = (Sigma1 - Sigma2)^-1.  piv: 3 x entries x n (G1, G2,
 * Delta), info: 3 x entries.  G2 / H2 directly after G1 / H1 (entries x
 * stride) run as one batch.  Replaces mnpbem/bem/bem_ret_mirror.py:182-328. */
int mnpb_bemret_init_mirror_f64(void *stream, int64_t n, int64_t entries, double *G1,
                                double *G2, double *H1, double *H2, int64_t ld, int64_t stride,
                                double *Dinv, int32_t *piv, int32_t *info, void *work,
                                int64_t work_bytes);
/* For the symmetry-value rows (ix, iy, iz) of an excitation's x, y, z parts:
 * S(b) = eps1 Sigma1_iz - eps2 Sigma2_iz + k^2 (eps1 - eps2)^2
 *        sum_d n_d n_d^T o Dinv_{i_d}, then LU(S) (pivS: batch x n, info:
 * batch).  H1, H2, Dinv as left by mnpb_bemret_init_mirror_f64; eps (batch x
 * 4: eps1, eps2 complex), kvac (batch), nvec (n x 3) of the irreducible part.
 * Replaces bem_ret_mirror.py:568-619 (_init_sigma_lu). */
int mnpb_bemret_sigma_mirror_f64(void *stream, int64_t n, int64_t nsym, int64_t batch,
                                 const double *H1, const double *H2, const double *Dinv,
                                 int64_t ld, int64_t stride, const double *eps,
                                 const double *kvac, const double *nvec, int32_t ix, int32_t iy,
                                 int32_t iz, double *S, int64_t sS, int32_t *pivS, int32_t *info);
/* Workspace of mnpb_bemret_solve_mirror_f64 in bytes. */
int64_t mnpb_bemret_solve_mirror_workspace(int64_t n, int64_t batch, int64_t nrhs);
/* BEMRet solve (layout of mnpb_bemret_solve_f64: x_in from
 * mnpb_bemret_excitation, x_out = [sig1 | h1 | sig2 | h2]) with the matrices
 * of component d (x, y, z) taken at symmetry row i_d and those of the scalar
 * parts at iz; S, pivS from mnpb_bemret_sigma_mirror_f64 for the same rows.
 * Replaces bem_ret_mirror.py:654-760 (solve). */
int mnpb_bemret_solve_mirror_f64(void *stream, int64_t n, int64_t nsym, int64_t batch,
                                 int64_t nrhs, const double *G1, const double *G2,
                                 const double *H1, const double *Dinv, int64_t ld,
                                 int64_t stride, const int32_t *piv, const double *S,
                                 int64_t sS, const int32_t *pivS, int32_t ix, int32_t iy,
                                 int32_t iz, const double *eps, const double *kvac,
                                 const double *nvec, const double *x_in, double *x_out,
                                 void *work, int64_t work_bytes);

/* ---------------------------------------------------------------------------
 * Points off the surface: dipole excitations and point-face Green functions
 *
 * Media are 1-based indices into per-wavelength tables of nmed complex values
 * (eps, k = 2 pi / lambda sqrt(eps), nb = sqrt(eps)), laid out (batch, nmed);
 * face_med (n x 2) holds the inside and outside medium of every face, pt_med
 * the medium of every point (0: not in any medium, contributes nothing).
 * Dipole moments dip are (npt x 3 x ndip); excitation column K index
 * q * ndip + idip, K = npt * ndip.
 * ------------------------------------------------------------------------- */

/* Potentials of the dipoles at the faces, pots (batch x 16 x K x n) in the
 * layout of mnpb_bemret_excitation.  Replaces
 * mnpbem/simulation/dipole_ret.py:319-515 (DipoleRet.potential / _pot). */
int mnpb_dipole_potential(void *stream, int64_t n, int64_t batch, int64_t npt, int64_t ndip,
                          const double *pos, const double *nvec, const int32_t *face_med,
                          const double *ptpos, const int32_t *pt_med, const double *dip,
                          int nmed, const double *eps, const double *k, const double *k0,
                          double *pots);

/* The dipoles' own fields at nobs observation positions in media obs_med:
 * e, h (batch x nobs x 3 x K).  Replaces dipole_ret.py:163-317
 * (DipoleRet.field / _dipolefield, Jackson 9.18). */
int mnpb_dipole_field(void *stream, int64_t nobs, int64_t batch, int64_t npt, int64_t ndip,
                      const double *obs, const int32_t *obs_med, const double *ptpos,
                      const int32_t *pt_med, const double *dip, int nmed, const double *eps,
                      const double *k, const double *nb, double *e, double *h);

/* Quasistatic dipole fields e = (3 x (x.d) - d) / (eps_q r^3) of dipoles
 * dip (npt x 3 x ndip) at positions ptpos screened by eps_pt (npt complex),
 * at nobs positions obs: out = e (nobs x 3 x npt x ndip complex), or with
 * normals nvec (nobs x 3, may be NULL) out = -nvec.e (nobs x npt x ndip
 * complex).  Replaces dipole_stat.py:149-289 (DipoleStat.field /
 * potential). */
int mnpb_dipole_stat_field(void *stream, int64_t nobs, int64_t npt, int64_t ndip,
                           const double *obs, const double *nvec, const double *ptpos,
                           const double *dip, const double *eps_pt, double *out);

/* Adds the far fields of the dipoles whose pt_on flag is set (points in the
 * embedding medium) to e, h (batch x K x ndir x 3, the layout of
 * mnpb_farfield).  emb: per wavelength eps, k, nb of the embedding medium
 * (batch x 3 complex).  Replaces dipole_ret.py:602-672 (DipoleRet.farfield). */
int mnpb_dipole_farfield(void *stream, int64_t ndir, int64_t batch, int64_t npt, int64_t ndip,
                         const double *ptpos, const int8_t *pt_on, const double *dip,
                         const double *dirs, const double *emb, double *e, double *h);

/* Refined Taylor coefficients (order 5, Cartesian derivative) of nref
 * point-face pairs (rows: points, cols: faces; from mnpb_refinematrix with
 * rad1 = NULL), integrated over the faces' quadrature points (qpos, qw, qoff
 * as for mnpb_refine_coefficients): g (nref x 6), f (nref x 3 x 6).
 * Replaces greenfun/greenret_refined.py:287-442 with a point set as p1. */
int mnpb_refine_points(void *stream, int64_t npt, const double *ptpos, int64_t n,
                       const double *pos, int64_t nref, const int32_t *rows, const int32_t *cols,
                       const double *qpos, const double *qw, const int64_t *qoff, double *g,
                       double *f);

/* Fields (mode 0) or potentials (mode 1) at the points from surface charges
 * and currents sol (batch x 8 x K x n, the solver's output layout), entries
 * computed on the fly (far formula, refined pairs from the CSR rptr / cols
 * with columns ascending and coefficients g, f of mnpb_refine_points).
 * k: (batch x nmed) wavenumbers, k0: (batch) 2 pi / lambda.
 *   mode 0: o1 = e, o2 = h (batch x npt x 3 x KC);
 *           e = i k0 sum_j G h_s - Gp sig_s, h = sum_j Gp x h_s
 *   mode 1: o1 = phi (batch x npt x KC), o2 = a (batch x npt x 3 x KC)
 * over faces j and their sides s that border the point's medium.  diag = 0:
 * all K columns (KC = K); diag > 0: point q reads only its own columns
 * [q diag, (q + 1) diag) and KC = diag (what decay rates need).  Replaces
 * greenfun/compgreen_ret.py:912-1036 (CompGreenRet(points, particle).field /
 * potential). */
int mnpb_point_green(void *stream, int64_t npt, const double *ptpos, const int32_t *pt_med,
                     int64_t n, const double *pos, const double *area, const int32_t *face_med,
                     int nmed, const double *k, const int64_t *rptr, const int32_t *cols,
                     const double *g, const double *f, int mode, int64_t batch, int64_t K,
                     int64_t diag, const double *k0, const double *sol, double *o1, double *o2);

/* Entries of the point-face region pair (points, side `side` of the faces)
 * for one wavelength: G (vec = 0, out npt x ncol) or Gp = H1p = H2p (vec = 1,
 * out npt x 3 x ncol) for face columns [col_start, col_start + ncol).
 * Replaces compgreen_ret.py:507-553 eval with a point set as p1. */
int mnpb_point_green_eval(void *stream, int64_t npt, const double *ptpos, const int32_t *pt_med,
                          int64_t n, const double *pos, const double *area,
                          const int32_t *face_med, int nmed, const double *k,
                          const int64_t *rptr, const int32_t *cols, const double *g,
                          const double *f, int side, int vec, int64_t col_start, int64_t ncol,
                          double *out);

/* ---------------------------------------------------------------------------
 * Electron beams (EELS, retarded)
 *
 * Beams run along z through impact parameters impact (nimp x 2) with width
 * `width` (> 0) and velocity vel (units of c, 0 < vel < 1).  Faces with
 * indquad[i * nimp + j] set are integrated over their quadrature points
 * (qpos, qw, qoff as for mnpb_refine_coefficients, weights divided by the
 * face area), the others take their centroid.  K0 and K1 of complex argument
 * are evaluated for |arg z| <= 1.2 (the caller checks 1/gamma).
 * ------------------------------------------------------------------------- */

/* BEM excitation pots (batch x 16 x nimp x n): face side s with medium m gets
 * the infinite-beam potential of medium m (1/gamma_m = igam, eps_m) for every
 * impact with beam_in[(m - 1) * nimp + j] set, if med_on[m - 1]:
 * phi / eps, phi' / eps and vel z^ phi, vel z^ phi'.  q: (batch) 2 pi /
 * (lambda vel); eps, igam: (batch x nmed) complex.  Replaces
 * mnpbem/simulation/eels_ret.py:149-294 with eels_base.py:315-416. */
int mnpb_eels_potential(void *stream, int64_t n, int64_t batch, int64_t nimp, const double *pos,
                        const double *nvec, const double *area, const int32_t *face_med,
                        int nmed, const int8_t *med_on, const int8_t *beam_in,
                        const double *impact, const int8_t *indquad, const double *qpos,
                        const double *qw, const int64_t *qoff, double width, double vel,
                        const double *q, const double *eps, const double *igam, double *pots);

/* Infinite-beam potentials phi, phip (nimp x n complex) of one medium
 * (1/gamma = igam) at faces with face_on set, 0 elsewhere
 * (eels_base.py:315-416, potinfty). */
int mnpb_eels_infty(void *stream, int64_t n, int64_t nimp, const double *pos, const double *nvec,
                    const double *area, const int8_t *face_on, const double *impact,
                    const int8_t *indquad, const double *qpos, const double *qw,
                    const int64_t *qoff, double width, double vel, double q, double igam_re,
                    double igam_im, double *phi, double *phip);

/* Potentials phi (nseg x n complex) of beam segments [seg[2c], seg[2c+1]] of
 * impact seg_imp[c] inside particles, -1/vel times the charged-wire integral
 * with wavenumbers q (beam) and k (medium) on the 11 Legendre-Gauss-Lobatto
 * nodes lgl_x / weights lgl_w (host arrays) (eels_base.py:418-523 and
 * 713-783, potinside / potwire); with phip non-null also their surface
 * derivatives along nvec (nseg x n complex). */
int mnpb_eels_wire(void *stream, int64_t n, int64_t nimp, const double *pos, const double *nvec,
                   const double *area, const int8_t *face_on, const double *impact,
                   const int8_t *indquad, const double *qpos, const double *qw,
                   const int64_t *qoff, double width, double vel, int64_t nseg,
                   const double *seg, const int32_t *seg_imp, double q, double k_re, double k_im,
                   const double *lgl_x, const double *lgl_w, double *phi, double *phip);

/* Fields of the beams at nobs positions in media obs_med: e, h (nobs x 3 x
 * nimp complex); mtab (nmed x 3 complex): eps, q = k / (vel sqrt(eps)) and
 * 1/gamma of every medium (eels_ret.py:506-637). */
int mnpb_eels_field(void *stream, int64_t nobs, int64_t nimp, const double *obs,
                    const int32_t *obs_med, int nmed, const int8_t *beam_in,
                    const double *impact, double width, double vel, const double *mtab,
                    double *e, double *h);

/* ---------------------------------------------------------------------------
 * Plane-wave excitation and cross sections (batched over wavelengths)
 * ------------------------------------------------------------------------- */

/* Plane-wave potentials for a batch of wavelengths, written in the pots
 * layout of mnpb_bemret_excitation.  Replaces
 * mnpbem/simulation/planewave_ret.py:257-361 (potential).  pol, dirs: npol x 3
 * (host-independent device arrays); kmed (batch complex), k0 (batch). */
int mnpb_planewave_potential(void *stream, int64_t n, int64_t batch, int64_t npol,
                             const double *pos, const double *nvec, const int8_t *side_in,
                             const int8_t *side_out, const double *pol, const double *dirs,
                             const double *kmed, const double *k0, double *pots);

/* Far field e (ndir x 3 x npol per wavelength) of the solution for the
 * directions dirs (ndir x 3).  Replaces mnpbem/spectrum/spectrum_ret.py:231
 * (farfield).  side_in/side_out (device int8, n): 1 if the face's inside /
 * outside medium is the embedding medium.  kmed: batch complex wavenumbers
 * in the medium; k0: batch vacuum wavenumbers.  sol as written by
 * mnpb_bemret_solve_f64.  e_out, h_out: device c128 [batch][npol][ndir][3]. */
int mnpb_farfield(void *stream, int64_t n, int64_t batch, int64_t npol, int64_t ndir,
                  const double *pos, const double *area, const int8_t *side_in,
                  const int8_t *side_out, const double *dirs, const double *kmed,
                  const double *k0, const double *sol, double *e_out, double *h_out);

/* ---------------------------------------------------------------------------
 * H-matrices and GMRES (iterative retarded solver, BEMRetIter)
 *
 * Block rectangles are int32 quadruples (row start, rows, col start, cols) in
 * cluster positions; c2p (int32, n) maps a cluster position to a face.  Dense
 * matrices are complex128, column-major, face order.
 * ------------------------------------------------------------------------- */

/* Partially-pivoted ACA of nblk low-rank blocks of A, one CTA per block, in
 * FP64.  UV: FP64 complex scratch; block b writes U (rows x cap) at
 * UV + 2*offU[b] doubles and V (cols x cap) at UV + 2*offV[b], cap =
 * min(rows, cols, kmax); rank[b] receives the rank.  max_mn: largest
 * rows + cols.  kmax <= 128.  Replaces HMatrix.aca/_aca_block
 * (mnpbem/greenfun/hmatrix.py:159-336) over ACACompGreenRet._eval_elements
 * (mnpbem/greenfun/aca_compgreen_ret.py:196-208). */
int mnpb_hmat_aca(void *stream, int64_t n, const double *A, int64_t lda, const int32_t *c2p,
                  int64_t nblk, const int32_t *blocks, const int64_t *offU, const int64_t *offV,
                  int64_t max_mn, int64_t kmax, double htol, double *UV, int32_t *rank);

/* Dense (leaf x leaf) blocks of A as complex64, block b at out + 2*offD[b]
 * floats, column-major.  Replaces the dense-block fill of HMatrix.aca
 * (mnpbem/greenfun/hmatrix.py:173-181). */
int mnpb_hmat_gather_dense(void *stream, const double *A, int64_t lda, const int32_t *c2p,
                           int64_t nblk, const int32_t *blocks, const int64_t *offD, float *out);

/* ACA factors from the FP64 scratch of mnpb_hmat_aca to complex64 storage:
 * U of block b (rows x rank, column-major) at U + 2*outU[b]; V stored
 * transposed (element (j, q) at q + j*rank) at V + 2*outV[b]. */
int mnpb_hmat_compact(void *stream, int64_t nblk, const int32_t *blocks, const int32_t *rank,
                      const int64_t *offU, const int64_t *offV, const double *UV,
                      const int64_t *outU, const int64_t *outV, float *U, float *V);

/* Y_i = H_i X_i for nmat (<= 4) H-matrices of one block partition; descs
 * points to nmat host records of 13 pointers each: D, U, V, rank, offT, X,
 * Y, T, Xc, offTP, TP, rent, vent.  X, Y: complex128 n x nc, column stride
 * n, face order; T: FP64 scratch of 2 * min(nc, 4) * sum(rank) doubles
 * (t_b = V_b^T x of block b at T + 2 * min(nc, 4) * offT[b]); Xc: FP64
 * scratch of 2 * n * min(nc, 4) doubles for X in cluster order; offTP
 * (int64 per low-rank block) and TP (FP64 scratch, 8 doubles per entry)
 * hold the per-segment partials of V^T x (block b's segments start at TP +
 * 8 * offTP[b], rank entries per segment).
 * rent: one 32-byte record per entry of the leaves' contribution lists
 * {int64 a, int64 xo, int32 lda, int32 cnt, int32 kind, int32 pad}: the
 * leaf's rows of a dense block (kind 0: a = float2 offset in D of (leaf's
 * first row, column 0), lda = block rows, cnt = block columns, xo = first
 * column in cluster order) or of a low-rank factor U (kind 1: a in U, cnt =
 * rank, xo = offT[b]).  vent: one 32-byte record per V^T x item {int64 v,
 * int64 out, int32 xo, int32 cnt, int32 r, int32 pad}: a segment of <= 64
 * columns of one low-rank block, V(j, q) at V + 2 * (v + (j - j0) * r + q),
 * x columns from xo (cluster order), partial to TP + 8 * out; vptr (nlr + 1)
 * the items of each block, in segment order.  leaf_rows: int32 (start,
 * rows) per leaf cluster; chunks: nchunk int32 pairs (leaf, first row)
 * covering every leaf in 32-row pieces; items: nitem int32 quadruples
 * (chunk, first entry, end entry, first row in the leaf << 6 | rows) with
 * at most 32 entries each, cptr (nchunk + 1) the items of each chunk;
 * partial: FP64 scratch of nmat * nitem * 256 doubles.
 * Replaces HMatrix.mtimes_vec (mnpbem/greenfun/hmatrix.py:450-541). */
int mnpb_hmat_matvec(void *stream, int64_t n, int64_t nc, int64_t nmat, const void *descs,
                     const int32_t *c2p, int64_t nlr, int64_t nchunk, const int32_t *chunks,
                     const int32_t *leaf_rows, int64_t nitem, const int32_t *items,
                     const int32_t *cptr, double *partial, int64_t nvitem,
                     const int32_t *vptr);

/* y = A x of the packed retarded operator from the four products P1 = G1 v1,
 * P2 = G2 v2, Q1 = H1 v1, Q2 = H2 v2 (n x 4*nrhs each, columns sig then h
 * x, y, z), scalar eps1/eps2, vacuum wavenumber k; y in the excitation layout
 * of mnpb_bemret_excitation.  Replaces BEMRetIter._afun
 * (mnpbem/bem/bem_ret_iter.py:1362-1501). */
int mnpb_bem_afun(void *stream, int64_t n, int64_t nrhs, const double *P1, const double *P2,
                  const double *Q1, const double *Q2, double *y, double e1_re, double e1_im,
                  double e2_re, double e2_im, double k, const double *nvec);

/* GMRES steps in FP64 (the Krylov solver of scipy.sparse.linalg.gmres as
 * called by mnpbem/bem/bem_iter.py:79-89).  Vectors complex128 of length L;
 * basis V column-major (column stride ldv); Hessenberg H column-major.
 * arnoldi: CGS2 orthogonalisation of w against V[:, 0..j], H column j
 * (Hcol, j + 2 entries) and V[:, j+1] = w / |w|; nrm (device) = |w|.
 * givens: rotations on column j, new rotation j, g update; out (device) =
 * |g[j+1]|.  update: y = R^{-1} g (m x m), x += V[:, 0..m-1] y. */
int64_t mnpb_gmres_workspace(int64_t L, int64_t jmax);
int mnpb_gmres_arnoldi(void *stream, int64_t L, int64_t j, double *V, int64_t ldv, double *w,
                       double *Hcol, double *nrm, void *work, int64_t work_bytes);
int mnpb_gmres_givens(void *stream, int64_t j, double *H, int64_t ldh, double *cs, double *sn,
                      double *g, double *out);
int mnpb_gmres_update(void *stream, int64_t L, int64_t m, const double *H, int64_t ldh,
                      const double *g, const double *V, int64_t ldv, double *y, double *x);

/* out[v] = |x_v| (FP64, device) for nvec complex128 vectors of length L at
 * x + 2*v*ldx doubles; partial: nvec * ceil(L / 2048) doubles of scratch.
 * Replaces the np.linalg.norm calls of mnpbem/bem/bem_iter.py:88. */
int mnpb_vec_norms(void *stream, int64_t L, int64_t nvec, const double *x, int64_t ldx,
                   double *partial, double *out);

/* ---------------------------------------------------------------------------
 * Warm-start network (per-face MLP predicting the next wavelength's
 * solution; no counterpart in the reference, which has no learned part).
 * Activations row-major FP32, weights [out][in] bf16 + FP32 master copy.
 * ------------------------------------------------------------------------- */

/* C (M x N) = A B with element strides (A(m,k) = A[m*sam + k*sak], B(k,n) =
 * B[k*sbk + n*sbn], C(m,n) = C[m*scm + n*scn]); b_bf16 != 0: B holds bf16.
 * mode 0: plain product (nsplit > 1 splits K; work holds nsplit*M*N floats
 * and C must be row-major dense); mode 1: C = SiLU(AB + bias), Z = AB +
 * bias; mode 2: C = Z = AB + bias (Z may be NULL). */
int mnpb_mlp_gemm(void *stream, int64_t M, int64_t N, int64_t K, const float *A, int64_t sam,
                  int64_t sak, const void *B, int64_t sbk, int64_t sbn, int32_t b_bf16, float *C,
                  int64_t scm, int64_t scn, const float *bias, int32_t mode, float *Z,
                  int64_t nsplit, float *work);
/* dZ = dY * SiLU'(Z) element-wise. */
int mnpb_mlp_silu_back(void *stream, int64_t len, const float *dY, const float *Z, float *dZ);
/* out[c] = sum over rows of X[r*ld + c]. */
int mnpb_mlp_colsum(void *stream, int64_t rows, int64_t cols, const float *X, int64_t ld,
                    float *out);
/* dY = 2 (Y - T) / len; part[ceil(len/256)] partial sums of (Y - T)^2. */
int mnpb_mlp_mse(void *stream, int64_t len, const float *Y, const float *T, float *dY,
                 float *part);
/* Adam step (bias correction in the step size) on FP32 w with gradient g,
 * moments m, v; wb (bf16, may be NULL) receives the rounded weights. */
int mnpb_mlp_adam(void *stream, int64_t len, float *w, void *wb, const float *g, float *m,
                  float *v, double lr, double b1, double b2, double eps, int64_t step);
/* wb = bf16(w), round to nearest even. */
int mnpb_mlp_to_bf16(void *stream, int64_t len, const float *w, void *wb);

#ifdef __cplusplus
}
#endif
#endif /* MNPBEM_B200_H */
