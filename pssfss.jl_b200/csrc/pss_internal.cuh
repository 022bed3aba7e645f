// Internal declarations shared by the library's translation units.
#pragma once
#include <atomic>
#include <mutex>

#include "pss_common.cuh"
#include "pssfss_b200.h"

// Per-device one-time set-up (kernel attributes and the like), safe to reach from several
// host threads: f() runs once for each device it is first called on (that device current).
struct DeviceOnce {
  std::atomic<unsigned long long> done{0};
  std::mutex mu;
};
template <class F>
int device_once(DeviceOnce &o, F &&f) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    pss_set_error("no usable current device (%d) for kernel set-up", dev);
    return -3;
  }
  const unsigned long long bit = 1ull << dev;
  if (o.done.load(std::memory_order_acquire) & bit) return 0;
  std::lock_guard<std::mutex> lk(o.mu);
  if (o.done.load(std::memory_order_relaxed) & bit) return 0;
  const int rc = f();
  if (!rc) o.done.fetch_or(bit, std::memory_order_release);
  return rc;
}

// Layer stack of one Gblock region (same for every frequency point of a batch).
struct StackParams {
  int nl, s;  // number of layers, 1-based interface index of the sheet
  cd eps[PSS_MAXLAYERS], mu[PSS_MAXLAYERS];
  double width[PSS_MAXLAYERS];  // metres
};

// Per frequency-point scalars (computed on the host, read by the kernels).
struct PointParams {
  double k0, u, psi1, psi2, omega;
  double b1[2], b2[2], b00[2];  // reciprocal lattice (1/m) and principal Floquet vector
  double area;                  // 4π²/|β1×β2|  (m²)
  double k0sq, b2min;
  cd mutilde, epsbar, c3, d3;       // electric (PGF.jl:205-210, FillZY.jl:60-61)
  cd f1, f3, p1, p3;                // magnetic summand factors (PGF.jl:496-499)
  cd I1fact, KFfact, I2fact, KPfact;  // filly factors (FillZY.jl:319-322)
  cd ff[5];                         // Floquet factors by edge code (FillZY.jl:72-77)
  int magnetic;
};

// Device-resident sheet topology (0-based indices).
struct SheetDev {
  int nface, nbf, nufp, nnode;
  double upm;  // sheet units per metre
  const double *rho;     // 2*nnode, sheet units
  const int *fv;         // 3*nface
  const int *ufpm;       // nface*nface, 0-based class of (match fa, source fb) at fa + fb*nface
  const int *ufp_rep;    // nufp, 0-based column-major face pair of the class representative
  // pair terms zb (pss_fill_pairs): 9 planes of nufp complex, term 3*isl + iml of class iu at
  // zb[(3*isl + iml)*nufp + iu]
  const double *fr;      // nface
  const double *face_ls; // 3*nface edge lengths (m): |r3-r2|, |r1-r3|, |r1-r2|
  const double *face_a48;// nface: 48*|area| (m²)
  const int *inc_cnt;    // nbf
  const int *inc_face;   // 4*nbf
  const int *inc_loc;    // 4*nbf local edge slot 0..2
  const int *inc_sgn;    // 4*nbf +1 plus / -1 minus
  const int *inc_eci;    // 4*nbf edge boundary code 0..4
};

// J/K cache (Zint.jl:54-179), SoA over unique face pairs.
struct JKDev {
  cd *J, *Jxi, *Jeta, *K, *Kxi, *Keta;
  double *rho_r;  // 2*nufp
  double *rinv;   // nufp
};

// Face-pair integrals of up to kJKGroup phasings (psi1, psi2) of one sheet in one launch: the
// phasing-free part of every lattice summand is shared, each phasing keeps its own sums.
constexpr int kJKGroup = 4;
struct PsiGroup {
  double psi1[kJKGroup], psi2[kJKGroup];
  int n;
};
struct JKGroup {
  JKDev s[kJKGroup];
};

// Modal tables of one point: padded (mmax+2)^2 column-major, index (m,n) in -1..mmax.
struct TableDev {
  cd *t1, *t2;
  int mmax;
};

// Six-point interpolation of a padded table (PGF.jl:396-441).
__device__ __forceinline__ cd sigma_interp(const cd *__restrict__ T, int mmax, const PointParams &P,
                                           double rx, double ry) {
  double x1o = (P.b1[0] * rx + P.b1[1] * ry) / PSS_TWOPI;
  if (fabs(x1o) < 1e-8) x1o = 0.0;
  double x2o = (P.b2[0] * rx + P.b2[1] * ry) / PSS_TWOPI;
  if (fabs(x2o) < 1e-8) x2o = 0.0;
  // Julia's mod(x, 1) in [0, 1]: x - floor(x) rounds once, exactly as fmod(x, 1) (exact)
  // followed by + 1 for negative x, so the result is bit-identical and avoids fmod
  const double x1 = x1o - floor(x1o), x2 = x2o - floor(x2o);
  double ms = rint(x1o - x1), ns = rint(x2o - x2);
  int m = (int)trunc(mmax * x1);
  double p = mmax * x1 - m;
  int n = (int)trunc(mmax * x2);
  double q = mmax * x2 - n;
  // x < 1 always, but mmax*x can round up to mmax; the stencil then must stay inside
  // the padded table (same point, one cell to the left).
  if (m >= mmax) { m = mmax - 1; p = mmax * x1 - m; }
  if (n >= mmax) { n = mmax - 1; q = mmax * x2 - n; }
  double p2 = p * p, q2 = q * q, pq = p * q;
  const int L = mmax + 2;
#define TX(a, b) T[(size_t)((a) + 1) + (size_t)((b) + 1) * L]
  cd s = (0.5 * (q2 - q)) * TX(m, n - 1);
  s = s + (0.5 * (p2 - p)) * TX(m - 1, n);
  s = s + (((1.0 + pq) - p2) - q2) * TX(m, n);
  s = s + (0.5 * ((p2 - 2.0 * pq) + p)) * TX(m + 1, n);
  s = s + (0.5 * ((q2 - 2.0 * pq) + q)) * TX(m, n + 1);
  s = s + pq * TX(m + 1, n + 1);
#undef TX
  if (ms != 0.0 || ns != 0.0) s = s * cisd(-(ms * P.psi1 + ns * P.psi2));
  return s;
}

// The device a context runs on (0, or -1 for a null context with a message).
extern "C" int pss_ctx_device(const pss_ctx *c, int *dev);

// Counts every kernel the library launches (reported by pss_kernel_launches()).
void pss_count_launch();
// Optional CUDA-event timing of the Schur-complement GEMM launches (pss_profile): returns
// a token (-1 when profiling is off) to pass to pss_prof_end with the launch's flops.
int pss_prof_begin(cudaStream_t st);
void pss_prof_end(int token, cudaStream_t st, int kind, double work);

// ---- host launchers (return 0 or a negative error code; errors via pss_set_error) ----
// Modal tables (pss_tables.cu)
void pss_tables_ring_fill(const StackParams &S, const PointParams *dP, int npts, int R, cd *dense,
                          size_t point_stride, cudaStream_t st);
void pss_tables_ring_sums(const PointParams *dP, int npts, int R, const cd *dense, size_t point_stride,
                          double convtest, unsigned char *conv, cudaStream_t st);
void pss_tables_find_mmax(int npts, int R, const unsigned char *conv, int *mmax, int *flag, cudaStream_t st);
int pss_tables_finish(const cd *dense, int R, int mmax, const PointParams *dP1, cd *stage, cd *t1, cd *t2,
                      cudaStream_t st);
size_t pss_table_cap(int mmax);  // (mmax+2)^2 entries per padded table

// Face-pair integrals and matrix fill (pss_fill.cu)
void pss_filljk(const SheetDev &G, double ulocal, double psi1, double psi2, const double s1[2],
                const double s2[2], JKDev jk, int *nonconv, cudaStream_t st);
// np <= kJKGroup phasings at once into jk[0..np), non-convergence counts into nonconv[0..np)
void pss_filljk_group(const SheetDev &G, double ulocal, int np, const double *psi1, const double *psi2,
                      const double s1[2], const double s2[2], const JKDev *jk, int *nonconv, cudaStream_t st);
void pss_fill_pairs(const SheetDev &G, const PointParams *dP1, const JKDev &jk, const cd *t1, const cd *t2,
                    int mmax, cd *zb, cudaStream_t st);
// Assemble Z (row-major): z64 with leading dimension ld, the FP32 planes (zr, zi) with ldf.
// z64 and/or (zr, zi) may be null.
void pss_fill_assemble(const SheetDev &G, const PointParams *dP1, const cd *zb, cd *z64, float *zr, float *zi,
                       long long ld, long long ldf, cudaStream_t st);

// Basis-function transforms, right-hand sides, projection (pss_bfft.cu)
void pss_bfft(const SheetDev &G, int nmodes, const double *kvec, double psi1, double psi2, cd *bf,
              cudaStream_t st);
void pss_rhs(int nbf, int nmodes, const cd *bf, const cd *src, cd *rhs, cudaStream_t st);
void pss_project(int nbf, int nmodes, const cd *bf, const double *tobs, const cd *wobs, const cd *X, cd *dS,
                 cudaStream_t st);
// PT (nbf x nmodes, column-major): row i of the projection, t_i · F_i[n], for the adjoint solve.
void pss_proj_rows(int nbf, int nmodes, const cd *bf, const double *tobs, cd *PT, cudaStream_t st);
// Adjoint contraction of a perturbed set from its pair terms zb (no matrix stored):
//   Gout[a + b*nm] = sum_m Lam[m, a] (R[m, b] - sum_n Z[m, n] X[n, b]);
// part: scratch of pss_adj_part_bytes(nbf, nm).
size_t pss_adj_part_bytes(int nbf, int nm);
void pss_adj_contract(const SheetDev &G, const PointParams *dP1, const cd *zb, const cd *X, const cd *R,
                      const cd *Lam, int nm, cd *part, cd *Gout, cudaStream_t st);

// Dense complex LU and solves (pss_lu.cu); matrices row-major with leading dimension ld.
// Batched forms factor nb matrices of order n at A + b*ms (elements), pivots at ipiv + b*n,
// info words at info + b; all matrices advance together, one launch per step.
int pss_lu64(int n, cd *A, long long ld, int *ipiv, int *info, void *ws, size_t ws_bytes, cudaStream_t st);
int pss_lu32(int n, float *Ar, float *Ai, long long ld, int *ipiv, int *info, void *ws, size_t ws_bytes,
             cudaStream_t st);
int pss_lu64_batched(int n, int nb, cd *A, long long ld, long long ms, int *ipiv, int *info, void *ws,
                     size_t ws_bytes, cudaStream_t st);
// FP32 tile shape: panel_w in {8, 16, 32} columns per cluster panel, outer_nb in {64, 128}
// columns per outer block (the tensor-core update's K); 0 picks 32 / 128.
int pss_lu32_batched(int n, int nb, float *Ar, float *Ai, long long ld, long long ms, int *ipiv, int *info,
                     void *ws, size_t ws_bytes, cudaStream_t st, int panel_w = 0, int outer_nb = 0);
size_t pss_lu_ws_bytes(int n, int precision, int nb = 1);

// Tensor-core (tcgen05, 3xTF32) complex Schur update on FP32 planes (pss_gemm_tc.cu), for
// each of nb matrices A_b = A + b*ms (elements):
//   A_b[m0:m0+M, n0:n0+N] -= A_b[m0:m0+M, k0:k0+K] * A_b[k0:k0+K, n0:n0+N],
// row-major, leading dimension ld; ws holds the split operands
// (pss_tc_ws_bytes(M, N, K rounded up to 16, nb)).  A bounded pipeline wait that gives up
// writes -1 to err[b].
size_t pss_tc_ws_bytes(int Mmax, int Nmax, int KP, int nb = 1);
int pss_cgemm_tc(float *Ar, float *Ai, long long ld, long long ms, int nb, int m0, int M, int n0, int N, int k0,
                 int K, void *ws, size_t ws_bytes, int *err, cudaStream_t st);

// Triangular solves and refinement (pss_trsv.cu).  The factor is either FP64 (LU64) or
// FP32 planes (Lr, Li); pass the other as null.
struct SolveWS {
  int n = 0, nblk = 0, nb = 0, epoch = 0;
  long long dstride = 0;   // elements between the matrices' diagonal-block inverses
  int cstride = 0;         // ints between the matrices' control words
  cd *Dinv = nullptr;      // inverses of the 64x64 diagonal blocks (L and U), per matrix
  int *perm = nullptr;     // pivot permutations
  int *ctrl = nullptr;     // per matrix: ticket, error flag, converged flag, per-block epoch flags
  double *norms = nullptr; // refinement norms, per matrix
  void bind(void *base, int n_, int nb_ = 1);
};
// Batched over nb matrices: factors at LU64 (or Lr/Li) + b*ms, ipiv + b*n, right-hand sides
// and solutions (n x nrhs column-major) at B/X + b*vs, status[b].
size_t pss_solve_ws_bytes(int n, int nb = 1);
int pss_solve_prepare(SolveWS &ws, int nb, const cd *LU64, const float *Lr, const float *Li, long long ld,
                      long long ms, const int *ipiv, cudaStream_t st);
int pss_solve_lu(SolveWS &ws, int nb, const cd *LU64, const float *Lr, const float *Li, long long ld, long long ms,
                 int nrhs, const cd *B, cd *X, long long vs, int use_done, cudaStream_t st);
int pss_refine(SolveWS &ws, int nb, const cd *A, long long ld, long long ms, const float *Lr, const float *Li,
               long long ldf, long long msf, int nrhs, const cd *B, cd *X, cd *R, cd *D, long long vs, int maxit, int *status, cudaStream_t st);
void pss_solve_status(SolveWS &ws, int nb, int *status, cudaStream_t st);
// Adjoint (transposed) solves on the same factors: Y = Z^-T B (W: scratch like B), and their
// FP64 refinement against A (FP32 factors) with a scratch of pss_refine_trans_ws_bytes.
int pss_solve_lu_trans(SolveWS &ws, int nb, const cd *LU64, const float *Lr, const float *Li, long long ld,
                       long long ms, int nrhs, const cd *B, cd *Y, cd *W, long long vs, int use_done,
                       cudaStream_t st);
size_t pss_refine_trans_ws_bytes(int n, int nrhs, int nb);
int pss_refine_trans(SolveWS &ws, int nb, const cd *A, long long ld, long long ms, const float *Lr, const float *Li,
                     long long ldf, long long msf, int nrhs, const cd *B, cd *Y, cd *R, cd *D, cd *W, void *scratch, size_t scratch_bytes,
                     long long vs, int maxit, int *status, cudaStream_t st);
