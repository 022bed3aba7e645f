/*
 * pssfss_b200 -- C ABI of the B200 (sm_100a) periodic method-of-moments fill-and-solve
 * library.  Plain pointers and sizes only; every entry point returns 0 on success or a
 * negative code (message via pss_last_error()).  No entry point aborts or traps.
 *
 * Conventions (chosen so a Julia caller passes its arrays unchanged):
 *   - index arrays are int64 with 1-based values, laid out column-major exactly like the
 *     reference's Julia arrays (fv/fe are 3 x nface, bff 2 x nbf, ufpm nface x nface);
 *   - complex numbers are interleaved (re, im) doubles;
 *   - lengths in sheet units unless stated; wavenumbers in 1/m.
 *
 * Reference interfaces replaced (PSSFSS.jl v0.1.4):
 *   pss_sheet_create   <- RWGSheet + RWGData fields used by the fill (src/Sheets.jl:19-58,
 *                          src/RWG.jl:27-76); the J/K cache of Sheets.jl:35-47 lives on the
 *                          device inside the sheet object, keyed as in FillZY.jl:97-99.
 *   pss_partial_gsms   <- the hot body of calculate_jtype_gsm / calculate_mtype_gsm
 *                          (src/PSSFSS.jl:391-457, 516-584): fillz/filly (src/FillZY.jl:50,273),
 *                          lu! (PSSFSS.jl:401,526), rwgbfft! (src/RWG.jl:428), ldiv!
 *                          (PSSFSS.jl:439,566) and the modal projection (Eqs. 6.18/6.37),
 *                          batched over all frequency / steering points of a sweep.
 *   pss_fill_matrix    <- fillz / filly alone (src/FillZY.jl:50-245, 273-457).
 *   pss_modal_tables   <- electric_/magnetic_modal_sum_funcs tables (src/PGF.jl:196, 478).
 *   pss_face_integrals <- filljk! (src/Zint.jl:54-179).
 *   pss_lu_solve       <- lu! followed by ldiv! on a caller matrix (LinearAlgebra).
 */
#ifndef PSSFSS_B200_H
#define PSSFSS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pss_ctx pss_ctx;
typedef struct pss_sheet pss_sheet;

/* precision of the dense solve */
#define PSS_FP64 0        /* complex128 LU and solves */
#define PSS_FP32_REFINE 1 /* complex64 LU, FP64 residuals and iterative refinement */

/* per-point status bits */
#define PSS_STATUS_TABLE_NOCONV 1   /* modal tables reached mmax = 2048 (PGF.jl:300 warning) */
#define PSS_STATUS_JK_NOCONV 2      /* a spatial lattice sum reached 65 rings (PGF.jl:104) */
#define PSS_STATUS_SINGULAR 4       /* exactly zero pivot */
#define PSS_STATUS_REFINE_NOCONV 8  /* refinement stopped before its tolerance */
#define PSS_STATUS_NONFINITE 16     /* NaN or Inf in the solution */
#define PSS_STATUS_FP64_FALLBACK 32 /* PSS_FP32_REFINE only: refinement stalled (cond(Z) too
                                       large for FP32 factors), point recomputed in FP64 */
#define PSS_STATUS_DEVICE_TIMEOUT 64 /* a bounded wait inside a kernel gave up (a pipeline or
                                        solve-chain stall); the point's results are invalid */

const char *pss_last_error(void);
int pss_version(void);
/* Total number of CUDA kernels this library has launched in the process so far. */
int64_t pss_kernel_launches(void);

/* One context per device; nworkers CUDA streams process frequency points concurrently. */
int pss_ctx_create(int device, int nworkers, pss_ctx **out);
int pss_ctx_destroy(pss_ctx *ctx);
/* The device a context runs on. */
int pss_ctx_device(const pss_ctx *ctx, int *device);

/* Upload a triangulated sheet and its basis-function topology.
 * cls: 'J' (conductor, fillz) or 'M' (aperture, filly).  s1, s2, beta1, beta2 in sheet
 * units (and 1/sheet units); rho: 2 x nnode; fv, fe: 3 x nface (fe[k] opposite fv[k]);
 * fr: nface sheet resistances (ohm/sq); bff: 2 x nbf plus/minus faces; ebf, eci: nedge;
 * ufpm: nface x nface unique-face-pair class numbers (match index fastest);
 * ufp_rep: nufp column-major face-pair index of each class's first member. */
int pss_sheet_create(pss_ctx *ctx, char cls, double units_per_meter, const double *s1, const double *s2,
                     const double *beta1, const double *beta2, int64_t nnode, const double *rho,
                     int64_t nface, const int64_t *fv, const int64_t *fe, const double *fr, int64_t nedge,
                     int64_t nbf, const int64_t *bff, const int64_t *ebf, const int64_t *eci, int64_t nufp,
                     const int64_t *ufpm, const int64_t *ufp_rep, pss_sheet **out);
int pss_sheet_destroy(pss_sheet *sheet);
/* Drop the sheet's cached face-pair integrals (the RWGSheet J/K fields, Sheets.jl:35-47), so
 * the next call recomputes them as the reference does when its cache key changes
 * (FillZY.jl:97-99); for a caller that edits geometry in place, or times whole sweeps. */
int pss_sheet_clear_cache(pss_sheet *sheet);

/* Scattered part of the sheet's partial GSM at npts points.
 * Region layers: nl layers, eps/mu complex (2*nl doubles), width in metres; s = 1-based
 * interface of the sheet; u = smoothing parameter (1/m).
 * Per point i: k0[i] (1/m), psi[2i], psi[2i+1] (rad).  Per point and mode j
 * (nmodes, region-1 modes first): kvec[(i*nmodes+j)*2 + 0..1] (1/m), src (2 complex),
 * tobs (2 real), wobs (1 complex) such that
 *     rhs[n, j] = conj(F_j[n]) . src_j,   Z x = rhs,
 *     dS[i][a + b*nmodes] = wobs_a * sum_n (tobs_a . F_a[n]) x[n, b],
 * where F_j is the basis-function transform at kvec_j (RWG.jl:428).  dS: npts *
 * nmodes^2 complex (column-major per point); status: npts (PSS_STATUS_* bits). */
int pss_partial_gsms(pss_sheet *sheet, int nl, const double *eps, const double *mu, const double *width,
                     int s, double u, int npts, const double *k0, const double *psi, int nmodes,
                     const double *kvec, const double *src, const double *tobs, const double *wobs,
                     int precision, double *dS, int *status);

/* One problem of pss_partial_gsms_multi: the arguments of pss_partial_gsms for one sheet,
 * plus the batch size (points factored together; 0: the context's default, PSS_BATCH) and
 * the FP32 LU tile shape (panel_w 8, 16 or 32 columns per cluster panel, outer_nb 64 or 128
 * columns per outer block = the tensor-core update's depth; 0: 32 and 128), as an
 * autotuner picks them per unknown count. */
typedef struct pss_problem {
  pss_sheet *sheet;
  int nl;
  const double *eps, *mu, *width;
  int s;
  double u;
  int npts;
  const double *k0, *psi;
  int nmodes;
  const double *kvec, *src, *tobs, *wobs;
  int batch, panel_w, outer_nb;
  double *dS;
  int *status;
} pss_problem;

/* Many sweeps in one call - problems on sheets of different unknown counts (and layers,
 * steering, modes), all of one context.  The scattered partial GSMs of every point of every
 * problem, as pss_partial_gsms gives them, computed from one shared work list: every point's
 * modal tables first, then batches of points with the same unknown and mode counts (from one
 * problem, or from several whose sheets have the same N; the largest matrices first) taken
 * by the context's worker streams, so no stream idles between problems.
 * Replaces the loop of _analyze over sheets and steering (src/PSSFSS.jl:230-329) when many
 * problems are swept together. */
int pss_partial_gsms_multi(int nprob, const pss_problem *problems, int precision);

/* Linearised partial GSMs for gradients with one factorisation per point (no counterpart in
 * the reference, which has no gradients).  The unperturbed inputs are those of
 * pss_partial_gsms.  For each of npert perturbed input sets k (a sheet psheets[k] of the same
 * context, class and basis count - the same sheet for a layer parameter - layers
 * peps/pmu/pwidth + k*nl, smoothing parameter pu[k], per point ppsi[(k*npts+i)*2 ..] and per
 * point and mode pkvec, psrc, ptobs, pwobs laid out like kvec .. wobs with index
 * (k*npts+i)*nmodes + j) it returns
 *     dSp[k][i] = wobs_k o (P_k Z^-1 R_k + P Z^-1 (R - Z_k X)),   X = Z^-1 R,
 * the first-order value of the perturbed partial GSM from the factors of the unperturbed Z
 * (P, R: projection and right-hand sides as in pss_partial_gsms), so central differences
 * of dSp over +/- steps give dS/dp to O(h^2).  dS: as pss_partial_gsms; dSp: npert * npts *
 * nmodes^2 complex.  Points run one at a time on the context's first stream; calls on one
 * context must not overlap. */
int pss_partial_gsms_lin(pss_sheet *sheet, int nl, const double *eps, const double *mu, const double *width,
                         int s, double u, int npts, const double *k0, const double *psi, int nmodes,
                         const double *kvec, const double *src, const double *tobs, const double *wobs,
                         int npert, pss_sheet *const *psheets, const double *peps, const double *pmu,
                         const double *pwidth, const double *pu, const double *ppsi, const double *pkvec,
                         const double *psrc, const double *ptobs, const double *pwobs, int precision,
                         double *dS, double *dSp, int *status);

/* Adjoint form of pss_partial_gsms_lin (no counterpart in the reference, which has no
 * gradients): the same arguments and output layout, with
 *     dSp[k][i] = wobs_k o (P_k X + Lam^T (R_k - Z_k X)),   X = Z^-1 R,   Lam = Z^-T P^T,
 * the first-order value of the perturbed partial GSM (central differences of dSp over
 * +/- steps give dS/dp to O(h^2)).  Per point: one factorisation, the forward solves of R
 * and the adjoint (transposed) solves of P^T on the same factors; each perturbed set then
 * recomputes its pair terms (the Green's-function values of its sheet and layers) and
 * contracts Lam^T Z_k X while assembling Z_k entry by entry - no perturbed matrix is stored
 * and no further solve is taken.  The points are swept as pss_partial_gsms sweeps them
 * (batched fills and factorisations on the context's worker streams); calls on one context
 * must not overlap.  nmodes <= 1024, npert <= 64. */
int pss_partial_gsms_adj(pss_sheet *sheet, int nl, const double *eps, const double *mu, const double *width,
                         int s, double u, int npts, const double *k0, const double *psi, int nmodes,
                         const double *kvec, const double *src, const double *tobs, const double *wobs,
                         int npert, pss_sheet *const *psheets, const double *peps, const double *pmu,
                         const double *pwidth, const double *pu, const double *ppsi, const double *pkvec,
                         const double *psrc, const double *ptobs, const double *pwobs, int precision,
                         double *dS, double *dSp, int *status);

/* GSM cascade of npts frequency points on the device: the Gblock walk of _analyze
 * (src/PSSFSS.jl:256-305) - cascade (the star product of Eq. 3.35, src/GSMs.jl:125-141) and
 * cascade! (propagation through a layer, src/GSMs.jl:154-176) - for every point at once.
 * Per point the chain starts from the identity GSM of region 0 propagated through layer 0,
 * then for each Gblock k = 0..nblk-1: A <- cascade(A, B_k), and A's region-2 ports are
 * propagated through the layer behind the block.  dims: nblk + 1 mode counts (block k joins
 * region k, dims[k] modes, to region k + 1), each 1..64, the same for every point.
 * gsm: per point, per block: s11 (dims[k]^2), s12 (dims[k] x dims[k+1]), s21, s22, each
 * column-major complex, in that order.  prop: per point, exp(-gamma d) of every mode of
 * layer 0 (dims[0] values), then of the layer behind each block (dims[k+1]); 1 where the
 * width is zero.  out: per point s11 (d0 x d0), s12 (d0 x dK), s21 (dK x d0), s22 (dK x dK).
 * status: npts, PSS_STATUS_SINGULAR where a star-product system had a zero pivot. */
int pss_cascade(pss_ctx *ctx, int npts, int nblk, const int *dims, const double *gsm, const double *prop,
                double *out, int *status);

/* Unique face-pair classes of a sheet on the device (the O(nface^2) classing of setup_rwg,
 * src/RWG.jl:287-319): pair (match m, source n) is keyed by the source face's shape class
 * shape[n] (0-based ids, < 2^31) and the offset of match centroid cen[m] from the source's first
 * vertex r1[n], quantised on the grid g (round half to even; offsets within 2^31 grid steps);
 * equal keys share a class.  Classes are numbered from 1 in the order of their first member in
 * column-major (match fastest) order.  cen, r1: nface x 2 interleaved (sheet units).
 * ufpm: nface x nface int32 out, column-major; rep: rep_cap int64 out, the 1-based column-major
 * pair index of each class's first member; nufp_out: the number of classes (also when it
 * exceeds rep_cap, which returns -5).  nface <= 16384. */
int pss_face_pair_classes(pss_ctx *ctx, int64_t nface, const double *cen, const double *r1, const int64_t *shape,
                          double g, int32_t *ufpm, int64_t *rep, int64_t rep_cap, int64_t *nufp_out);

/* The MoM matrix of one point: Z (nbf x nbf complex, column-major like zorymat). */
int pss_fill_matrix(pss_sheet *sheet, int nl, const double *eps, const double *mu, const double *width, int s,
                    double u, double k0, double psi1, double psi2, double *Z, int *mmax_out);

/* Padded modal tables (capacity cap entries each, (mmax+2)^2 used, column-major). */
int pss_modal_tables(pss_ctx *ctx, int magnetic, int nl, const double *eps, const double *mu,
                     const double *width, int s, double k0, double u, double psi1, double psi2,
                     const double *b1, const double *b2, double convtest, int64_t cap, double *t1,
                     double *t2, int *mmax_out, int *status);

/* Frequency-independent face-pair integrals of every unique pair (ulocal in 1/sheet units).
 * Outputs (nufp entries each): J, Jxi, Jeta, K, Kxi, Keta complex; rho_r 2*nufp; rinv. */
int pss_face_integrals(pss_sheet *sheet, double ulocal, double psi1, double psi2, double *J, double *Jxi,
                       double *Jeta, double *K, double *Kxi, double *Keta, double *rho_r, double *rinv,
                       int *nonconv);

/* Basis-function transforms at nmodes transform variables: F (nmodes x nbf x 2 complex). */
int pss_basis_transforms(pss_sheet *sheet, int nmodes, const double *kvec, double psi1, double psi2, double *F);

/* Solve Z X = B with Z n x n complex column-major, B/X n x nrhs column-major. */
int pss_lu_solve(pss_ctx *ctx, int n, const double *Z, int nrhs, const double *B, int precision, double *X,
                 int *status);

/* FP32 factorisation of the FP32 + refinement form on its own (no counterpart; the reference's
 * zgetrf is FP64): Z n x n complex column-major in, rounded to complex64; LU out, the packed
 * unit-lower L and upper U, n x n complex64 column-major; ipiv out 1-based, LAPACK's
 * interchange convention (row j swapped with row ipiv[j]); info out, the first zero pivot. */
int pss_lu32_factor(pss_ctx *ctx, int n, const double *Z, float *LU, int *ipiv, int *info);

/* Device milliseconds of the last pss_partial_gsms call, summed over worker 0's batches:
 * [tables, face_integrals (0: folded into fill), fill, transforms+rhs, 0, factor+solve+refine,
 *  projection, total span of the call over all workers]. */
int pss_last_timings(pss_ctx *ctx, double *ms8);

/* Per-launch CUDA-event timing (on each launch's own stream) of the factorisation's main
 * kernels during pss_partial_gsms calls while enabled.  out receives 3 doubles per kind -
 * launches, summed milliseconds, summed algorithmic work - for the last call:
 *   PSS_PROF_TC_UPDATE   tensor-core Schur update, work = 8*M*N*K flops per complex update
 *   PSS_PROF_PANEL       cluster panel factorisation, work = bytes of the panel read + written
 *   PSS_PROF_SIMT_UPDATE SIMT Schur update (FP64, and FP32 updates below the tensor-core size),
 *                        work = 8*M*N*K flops */
#define PSS_PROF_TC_UPDATE 0
#define PSS_PROF_PANEL 1
#define PSS_PROF_SIMT_UPDATE 2
#define PSS_PROF_KINDS 3
int pss_profile(pss_ctx *ctx, int enable);
int pss_profile_result(pss_ctx *ctx, double *out);

/* Schur-complement update C -= L * U in complex FP32 on the tensor cores (tcgen05, 3xTF32
 * products: FP32-level accuracy), the kernel the PSS_FP32_REFINE factorisation uses for its
 * trailing updates.  Host arrays, row-major, real and imaginary parts separate: L m x k,
 * U k x n, C m x n (updated in place).  status: 0, or PSS_STATUS_DEVICE_TIMEOUT.
 * No counterpart in the reference, whose LU is LAPACK zgetrf behind lu! (src/PSSFSS.jl:401,
 * 526); exposed so the kernel can be checked on its own. */
int pss_schur_update(pss_ctx *ctx, int m, int n, int k, const float *Lr, const float *Li, const float *Ur,
                     const float *Ui, float *Cr, float *Ci, int *status);

/* Poll limit of the bounded hand-off waits inside the tensor-core update (TMA producer, MMA
 * issuer and epilogue waiting on each other); 0 restores the default of 2^24 polls.  A wait
 * that runs out marks the update's matrices with PSS_STATUS_DEVICE_TIMEOUT, and the kernel
 * waits (at the default limit) for its copies and MMAs in flight, frees its tensor memory
 * and returns, leaving the context usable.  A test hook: a limit of a few polls makes the
 * waits run out.  No counterpart in the reference.  Applies to launches made after the call. */
int pss_set_wait_limit(int64_t iterations);

/* FP64 complex LU factorisation, in place, on caller-owned device memory, allocating no
 * device memory at all (no cudaMalloc, cudaFree or allocating library routine).  It has
 * no counterpart in the reference.  It serves callers that cannot let a library allocate
 * per call - a host whose device memory is held by its own pool (Julia CUDA.jl, PyTorch),
 * or a latency-sensitive loop in which cudaFree's device-wide synchronisation would stall
 * every other stream.
 *   A     device, n x n interleaved complex128, ROW-major, leading dimension ld >= n
 *         (elements), 16-byte aligned; overwritten by U (upper) and the unit-lower L.
 *   ipiv  device, n ints, 0-based: row k was interchanged with row ipiv[k], k = 0..n-1
 *         applied in order (LAPACK's convention minus one).
 *   info  device int: set to 0 by this call (on `stream`, before the first kernel), then
 *         to j+1 if column j held the first exactly-zero pivot.
 *   stream  a cudaStream_t of the current device (NULL: the legacy default stream).
 * Runs on the current device and is asynchronous with respect to the host.
 * Limit: n <= 8192; larger n returns -1 with a message in pss_last_error().  Its scratch
 * is a fixed 1 KB file-scope device array (the panels' interchange list), one per device:
 * nothing in it has to start at zero, but calls that overlap in time on the same device
 * race on it - serialise them.  The first call on each device resolves that array's
 * address (cudaGetSymbolAddress); make that first call before any stream capture on the
 * device.  The address is cached with the CUDA context it belongs to and looked up again
 * when another context is current (after cudaDeviceReset, for instance). */
int pss_lu_factor_noalloc(int n, double *A, int64_t ld, int *ipiv, int *info, void *stream);

#ifdef __cplusplus
}
#endif
#endif
