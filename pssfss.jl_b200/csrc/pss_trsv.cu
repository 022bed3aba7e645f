// K5: triangular solves with the LU factors, FP64 residuals and iterative refinement.
//
// Replaces LAPACK zgetrs (ldiv!, PSSFSS.jl:439,566) for the small right-hand-side sets
// of a sweep point (n_rhs = number of incident modes, 4 at normal incidence).
//
// Chained block substitution: the factor is cut into 64-row blocks; CTA tickets are
// taken in start order (atomicAdd), CTA b solves block b and only waits (bounded spin on
// a per-block epoch flag) for blocks that started before it, so it never waits on a CTA
// that is not resident.  Every CTA streams its share of the triangle (the bulk of the
// bytes) concurrently; the serial chain per block is one 64x64 product with the
// precomputed inverse of the diagonal block.  FP64 arithmetic for FP32 or FP64 factors.
//
// Refinement (LAPACK zcgesv's scheme): r = b - A x with the FP64 matrix, stop when
// max|r_j| <= max|x_j| * ||A||_inf * eps * sqrt(n) for every rhs j (cabs1 norms).
#include <cuda/atomic>
#include "pss_internal.cuh"

namespace {

constexpr int BS = 64;        // block rows
constexpr int kMaxRhs = 8;    // right-hand sides per pass
constexpr int kMaxRefRhs = 1024;          // right-hand sides of one refinement
constexpr int kNX = kMaxRefRhs;           // norms layout: [max|r_j|] [max|x_j|] [||A||]
constexpr int kNA = 2 * kMaxRefRhs;
constexpr int kNormCount = 2 * kMaxRefRhs + 1;
constexpr long long kSpinCap = 1LL << 24;

struct Fac {  // row-major factor access: FP64 interleaved or FP32 planes
  const cd *a64;
  const float *ar, *ai;
  long long ld;
  long long ms;  // elements between the factors of a batch
  __device__ __forceinline__ cd at(long long r, long long c) const {
    if (a64) return a64[r * ld + c];
    return mkcd((double)ar[r * ld + c], (double)ai[r * ld + c]);
  }
  __device__ __forceinline__ Fac of(int b) const {  // factor b of the batch
    return Fac{a64 ? a64 + b * ms : nullptr, ar ? ar + b * ms : nullptr, ai ? ai + b * ms : nullptr, ld, ms};
  }
};

// Per-matrix control words of a batch: [0] ticket, [1] error, [2] converged, [8..] flags.
struct Ctrl {
  int *base;
  int stride;
  __device__ __forceinline__ int *of(int b) const { return base + (long long)b * stride; }
};

__device__ __forceinline__ double cabs1(cd z) { return fabs(z.x) + fabs(z.y); }

// L2-only (L1-bypassing) access to blocks of X that other CTAs produce or consume.
__device__ __forceinline__ cd ldcg(const cd *p) {
  const double2 v = __ldcg(reinterpret_cast<const double2 *>(p));
  return mkcd(v.x, v.y);
}
__device__ __forceinline__ void stcg(cd *p, cd v) { __stcg(reinterpret_cast<double2 *>(p), make_double2(v.x, v.y)); }

// Spin until flags[c] >= epoch (acquire).  Returns false (and records an error) at the cap.
__device__ __forceinline__ bool wait_flag(int *flags, int c, int epoch, int *err) {
  cuda::atomic_ref<int, cuda::thread_scope_device> f(flags[c]);
  long long it = 0;
  while (f.load(cuda::memory_order_acquire) < epoch) {
    if (++it > kSpinCap) {
      atomicExch(err, 1);
      return false;
    }
    if (it > 512) __nanosleep(64);  // hot spin first: the chain's step time is a few microseconds
  }
  return true;
}

__device__ __forceinline__ void post_flag(int *flags, int b, int epoch) {
  cuda::atomic_ref<int, cuda::thread_scope_device> f(flags[b]);
  f.store(epoch, cuda::memory_order_release);
}

// Inverses of the 64x64 diagonal blocks: Dinv[(2*blk + 0)] = L_bb^{-1} (unit lower),
// Dinv[(2*blk + 1)] = U_bb^{-1}; each 64x64 row-major FP64.
__global__ void __launch_bounds__(64) k_diag_inv(Fac F0, int n, cd *Dinv0, long long dstride) {
  const int blk = blockIdx.x, upper = blockIdx.y;
  const Fac F = F0.of(blockIdx.z);
  cd *Dinv = Dinv0 + blockIdx.z * dstride;
  const int r0 = blk * BS, nb = min(BS, n - r0);
  extern __shared__ cd sm[];
  cd *T = sm;            // 64 x 64 block
  cd *X = sm + BS * BS;  // 64 x 64 inverse, column k owned by thread k
  const int k = threadIdx.x;
  for (int i = 0; i < BS; ++i) T[i * BS + k] = (i < nb && k < nb) ? F.at(r0 + i, r0 + k) : mkcd(i == k, 0);
  __syncthreads();
  if (!upper) {
    for (int i = 0; i < BS; ++i) {
      cd v = mkcd(i == k, 0);
      for (int t = k; t < i; ++t) v = v - T[i * BS + t] * X[t * BS + k];
      X[i * BS + k] = (i < k) ? mkcd(0, 0) : v;
    }
  } else {
    for (int i = BS - 1; i >= 0; --i) {
      cd v = mkcd(i == k, 0);
      for (int t = i + 1; t <= k; ++t) v = v - T[i * BS + t] * X[t * BS + k];
      X[i * BS + k] = (i > k) ? mkcd(0, 0) : v / T[i * BS + i];
    }
  }
  __syncthreads();
  cd *D = Dinv + (size_t)(2 * blk + upper) * BS * BS;
  for (int i = 0; i < BS; ++i) D[i * BS + k] = X[i * BS + k];
}

// perm[i] = original row that ends in position i after the LAPACK swap sequence ipiv.
__global__ void __launch_bounds__(1024) k_ipiv_to_perm(int n, const int *ipiv0, int *perm0) {
  extern __shared__ int sp[];
  const int *ipiv = ipiv0 + (long long)blockIdx.x * n;
  int *perm = perm0 + (long long)blockIdx.x * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) sp[i] = i;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < n; ++k) {
      int p = ipiv[k];
      int t = sp[k]; sp[k] = sp[p]; sp[p] = t;
    }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = sp[i];
}

// Arithmetic of a chained pass: FP64 for FP64 factors; FP32 for FP32 factors, as LAPACK
// zcgesv solves its corrections in single precision (cgetrs) before the FP64 update.
template <bool F32>
struct SolveT;
template <>
struct SolveT<false> {
  using C = cd;
  __device__ static C fac(const Fac &F, long long r, long long c) { return F.a64[r * F.ld + c]; }
  __device__ static C from(cd v) { return v; }
  __device__ static cd to(C v) { return v; }
};
template <>
struct SolveT<true> {
  using C = cf;
  __device__ static C fac(const Fac &F, long long r, long long c) { return cf{F.ar[r * F.ld + c], F.ai[r * F.ld + c]}; }
  __device__ static C from(cd v) { return cf{(float)v.x, (float)v.y}; }
  __device__ static cd to(C v) { return mkcd(v.x, v.y); }
};
__device__ __forceinline__ cf operator+(cf a, cf b) { return cf{a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cf operator-(cf a, cf b) { return cf{a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ cf operator*(cf a, cf b) { return cf{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
template <class C>
__device__ __forceinline__ C czero() { return C{0, 0}; }

// One chained substitution pass over right-hand sides j0 .. j0+nj-1 (nj <= NJ):
//   lower: X[rows_b] = Linv_b (B[perm[rows_b]] - sum_{c<b} L[b,c] X[c])
//   upper: X[rows_b] = Uinv_b (X[rows_b] - sum_{c>b} U[b,c] X[c])   (in place)
// TRANS (the adjoint system Z^T y = b, Z = P^T L U, so U^T L^T (P y) = b): the lower pass
// runs with U^T (block (b, c) read as the transpose of block (c, b) of the factor, the
// diagonal inverse transposed) on B unpermuted, the upper pass with L^T in place; the
// caller applies P^T to the result (pss_solve_lu_trans).
// One CTA per 64-row block b (ticket order), 256 threads: row i = tid/4 of the block,
// quarter p = tid%4 covers 16 columns of each 64-column tile.  Each tile of the factor is
// loaded into registers BEFORE the wait for the CTA that produces x_c, so the wait hides
// the load; Dinv_b (dynamic shared memory) and the block's right-hand side are staged at
// the start.  Blocks of X written by other CTAs are read with L1-bypassing loads.
template <bool LOWER, bool F32, int NJ, bool TRANS = false>
__global__ void __launch_bounds__(256, F32 ? 2 : 1) k_trsv(Fac F0, int n, const int *__restrict__ perm0, const cd *__restrict__ B0,
                                              cd *__restrict__ X0, long long vs, int nrhs, int j0,
                                              const cd *__restrict__ Dinv0, long long dstride, Ctrl ctrl, int epoch,
                                              int use_done) {
  using T = SolveT<F32>;
  using C = typename T::C;
  // matrix of the batch: the grid runs matrix-fastest, so the CTAs start block row by block
  // row across all matrices and every matrix's chain advances in the same waves
  const int bm = blockIdx.x;
  int *cw = ctrl.of(bm);
  if (use_done && cw[2]) return;
  const Fac F = F0.of(bm);
  const int *perm = perm0 + (long long)bm * n;
  const cd *B = B0 + bm * vs;
  cd *X = X0 + bm * vs;
  const cd *Dinv = Dinv0 + bm * dstride;
  int *ticket = cw, *err = cw + 1, *flags = cw + 8;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *Ds = (C *)smraw;  // BS x BS, row-major
  __shared__ C y[BS][NJ];
  __shared__ C xs[BS][NJ];
  __shared__ int s_b;
  const int tid = threadIdx.x;
  const int i = tid >> 2, p = tid & 3;
  const int nblk = (n + BS - 1) / BS;
  const int nj = min(NJ, nrhs - j0);
  if (tid == 0) s_b = atomicAdd(ticket, 1);
  __syncthreads();
  const int tk = s_b;
  const int b = LOWER ? tk : nblk - 1 - tk;
  const int r0 = b * BS, nr = min(BS, n - r0);
  // diagonal block: L_bb^-1 (lower pass) or U_bb^-1 (upper pass); transposed, U_bb^-T for the
  // lower pass of the adjoint system and L_bb^-T for its upper pass
  const cd *D = Dinv + (size_t)(2 * b + ((LOWER != TRANS) ? 0 : 1)) * BS * BS;
  for (int e = tid; e < BS * BS; e += 256) Ds[e] = T::from(TRANS ? D[(e % BS) * BS + e / BS] : D[e]);
  for (int e = tid; e < BS * NJ; e += 256) {
    const int r = e / NJ, j = e % NJ;
    cd v = mkcd(0, 0);
    if (r < nr && j < nj)
      v = LOWER ? B[(size_t)(j0 + j) * n + (TRANS ? r0 + r : perm[r0 + r])] : ldcg(&X[(size_t)(j0 + j) * n + r0 + r]);
    y[r][j] = T::from(v);
  }
  const int c_lo = LOWER ? 0 : b + 1, c_hi = LOWER ? b : nblk;
  if constexpr (F32 && !TRANS && NJ == 4) {
    // Coalesced form for the FP32 factors of the sweep: warp w owns rows 8w .. 8w+7 of the
    // block, lane l columns l and l + 32 of every 64-column tile, so each load instruction of
    // a warp reads one contiguous 128-byte row segment; the lane's partial sums run over all
    // tiles and are reduced across the warp once at the end.  Each warp waits for x_c on its
    // own (lane 0 polls the flag), so no block barrier sits in the tile loop.
    const int warp = tid >> 5, lane = tid & 31;
    C a8[8][NJ];
#pragma unroll
    for (int rr = 0; rr < 8; ++rr)
#pragma unroll
      for (int j = 0; j < NJ; ++j) a8[rr][j] = czero<C>();
    for (int cc = c_lo; cc < c_hi; ++cc) {
      const int c = LOWER ? cc : c_hi - 1 - (cc - c_lo);
      const int t0 = c * BS, nt = min(BS, n - t0);
      C lv[8][2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int col = lane + 32 * h;
#pragma unroll
        for (int rr = 0; rr < 8; ++rr) {
          const int row = warp * 8 + rr;
          lv[rr][h] = (row < nr && col < nt) ? T::fac(F, r0 + row, t0 + col) : czero<C>();
        }
      }
      if (lane == 0) {
        wait_flag(flags, c, epoch, err);
        __threadfence();
      }
      __syncwarp();
      C xv[2][NJ];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int col = lane + 32 * h;
#pragma unroll
        for (int j = 0; j < NJ; ++j)
          xv[h][j] = (col < nt && j < nj) ? T::from(ldcg(&X[(size_t)(j0 + j) * n + t0 + col])) : czero<C>();
      }
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int rr = 0; rr < 8; ++rr)
#pragma unroll
          for (int j = 0; j < NJ; ++j) a8[rr][j] = a8[rr][j] + lv[rr][h] * xv[h][j];
    }
#pragma unroll
    for (int rr = 0; rr < 8; ++rr)
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        for (int o = 16; o > 0; o >>= 1) {
          a8[rr][j].x += __shfl_xor_sync(0xffffffff, a8[rr][j].x, o);
          a8[rr][j].y += __shfl_xor_sync(0xffffffff, a8[rr][j].y, o);
        }
        if (lane == 0) xs[warp * 8 + rr][j] = a8[rr][j];
      }
    __syncthreads();
    for (int e = tid; e < BS * NJ; e += 256) {
      const int r = e / NJ, j = e % NJ;
      if (r < nr && j < nj) y[r][j] = y[r][j] - xs[r][j];
    }
    __syncthreads();
  } else {
  C acc[NJ];
#pragma unroll
  for (int j = 0; j < NJ; ++j) acc[j] = czero<C>();
  for (int cc = c_lo; cc < c_hi; ++cc) {
    const int c = LOWER ? cc : c_hi - 1 - (cc - c_lo);  // upper: the last block is ready first
    const int t0 = c * BS, nt = min(BS, n - t0);
    C lv[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int t = p * 16 + q;
      lv[q] = (i < nr && t < nt) ? (TRANS ? T::fac(F, t0 + t, r0 + i) : T::fac(F, r0 + i, t0 + t)) : czero<C>();
    }
    if (tid == 0) {
      wait_flag(flags, c, epoch, err);
      __threadfence();
    }
    __syncthreads();
    for (int e = tid; e < BS * NJ; e += 256) {
      const int t = e / NJ, j = e % NJ;
      xs[t][j] = (t < nt && j < nj) ? T::from(ldcg(&X[(size_t)(j0 + j) * n + t0 + t])) : czero<C>();
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 16; ++q) {
#pragma unroll
      for (int j = 0; j < NJ; ++j) acc[j] = acc[j] + lv[q] * xs[p * 16 + q][j];
    }
  }
#pragma unroll
  for (int j = 0; j < NJ; ++j)
    for (int o = 1; o < 4; o <<= 1) {
      acc[j].x += __shfl_xor_sync(0xffffffff, acc[j].x, o);
      acc[j].y += __shfl_xor_sync(0xffffffff, acc[j].y, o);
    }
  __syncthreads();
  if (p == 0 && i < nr) {
#pragma unroll
    for (int j = 0; j < NJ; ++j) y[i][j] = y[i][j] - acc[j];
  }
  __syncthreads();
  }
  // X[rows] = Dinv_b * y: 4 threads per output, 16 terms each, combined by shuffles
  for (int e0 = 0; e0 < nr * nj; e0 += 64) {
    const int e = e0 + (tid >> 2), part = tid & 3;
    const int r = e / nj, j = e % nj;
    C s = czero<C>();
    if (e < nr * nj) {
#pragma unroll 4
      for (int k = part * 16; k < part * 16 + 16; ++k)
        if (k < nr) s = s + Ds[r * BS + k] * y[k][j];
    }
    for (int o = 1; o < 4; o <<= 1) {
      s.x += __shfl_xor_sync(0xffffffff, s.x, o);
      s.y += __shfl_xor_sync(0xffffffff, s.y, o);
    }
    if (part == 0 && e < nr * nj) stcg(&X[(size_t)(j0 + j) * n + r0 + r], T::to(s));
  }
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    post_flag(flags, b, epoch);
  }
}

// R = B - A X with max|r_j| (norms[j]), max|x_j| (norms[kNX + j]) and ||A||_inf (norms[kNA]).
__global__ void __launch_bounds__(256) k_resid(int n, const cd *__restrict__ A0, long long ld, long long ms, int nrhs,
                                               const cd *__restrict__ X0, const cd *__restrict__ B0,
                                               cd *__restrict__ R0, long long vs, double *norms0, Ctrl ctrl) {
  const int bm = blockIdx.y;
  if (ctrl.of(bm)[2]) return;
  const cd *A = A0 + bm * ms, *X = X0 + bm * vs, *B = B0 + bm * vs;
  cd *R = R0 + bm * vs;
  double *norms = norms0 + (long long)bm * kNormCount;
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (row < n) {
    const cd *a = A + (long long)row * ld;
    for (int j0 = 0; j0 < nrhs; j0 += kMaxRhs) {
      const int nj = min(kMaxRhs, nrhs - j0);
      cd acc[kMaxRhs];
      for (int j = 0; j < kMaxRhs; ++j) acc[j] = mkcd(0, 0);
      double rs = 0;
      for (int t = lane; t < n; t += 32) {
        cd av = a[t];
        if (j0 == 0) rs += cabs1(av);
        for (int j = 0; j < nj; ++j) acc[j] = acc[j] + av * X[(size_t)(j0 + j) * n + t];
      }
      for (int j = 0; j < nj; ++j)
        for (int o = 16; o > 0; o >>= 1) {
          acc[j].x += __shfl_xor_sync(0xffffffff, acc[j].x, o);
          acc[j].y += __shfl_xor_sync(0xffffffff, acc[j].y, o);
        }
      if (j0 == 0) {
        for (int o = 16; o > 0; o >>= 1) rs += __shfl_xor_sync(0xffffffff, rs, o);
        if (lane == 0) atomicMax((unsigned long long *)&norms[kNA], (unsigned long long)__double_as_longlong(rs));
      }
#pragma unroll
      for (int j = 0; j < kMaxRhs; ++j) {
        if (j < nj && lane == j) {
          cd r = B[(size_t)(j0 + j) * n + row] - acc[j];
          R[(size_t)(j0 + j) * n + row] = r;
          atomicMax((unsigned long long *)&norms[j0 + j], (unsigned long long)__double_as_longlong(cabs1(r)));
          double xv = cabs1(X[(size_t)(j0 + j) * n + row]);
          atomicMax((unsigned long long *)&norms[kNX + j0 + j], (unsigned long long)__double_as_longlong(xv));
        }
      }
    }
  }
}

// Residual for up to 4 right-hand sides (the sweep's usual case): a CTA of 8 warps takes 16
// rows, each warp 2 of them; the columns go in chunks whose X block (4 x 1024) is staged in
// shared memory and reused by the rows of every warp, so the matrix rows are the only HBM
// stream (each read once, streaming loads).  The column loop has no early exit (the ragged
// last chunk is predicated), so the loads of several steps are in flight per lane; rows past
// n are clamped to row n-1 for their loads and dropped at the end.
constexpr int kResRows = 2, kResChunk = 1024;
constexpr int kResSmem = 4 * kResChunk * (int)sizeof(cd);  // 64 KB
__device__ __forceinline__ cd ldcs(const cd *p) {
  const double2 v = __ldcs(reinterpret_cast<const double2 *>(p));
  return cd{v.x, v.y};
}
__global__ void __launch_bounds__(256) k_resid4(int n, const cd *__restrict__ A0, long long ld, long long ms, int nrhs,
                                                const cd *__restrict__ X0, const cd *__restrict__ B0,
                                                cd *__restrict__ R0, long long vs, double *norms0, Ctrl ctrl) {
  const int bm = blockIdx.y;
  if (ctrl.of(bm)[2]) return;
  const cd *A = A0 + bm * ms, *X = X0 + bm * vs, *B = B0 + bm * vs;
  cd *R = R0 + bm * vs;
  double *norms = norms0 + (long long)bm * kNormCount;
  extern __shared__ __align__(16) unsigned char res_smem[];
  cd(*xs)[kResChunk] = reinterpret_cast<cd(*)[kResChunk]>(res_smem);  // [4][kResChunk]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r0 = blockIdx.x * (8 * kResRows) + warp * kResRows;
  const cd *arow[kResRows];
  cd acc[kResRows][4];
  double rs[kResRows];
#pragma unroll
  for (int i = 0; i < kResRows; ++i) {
    arow[i] = A + (long long)min(r0 + i, n - 1) * ld;
    rs[i] = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = mkcd(0, 0);
  }
  for (int t0 = 0; t0 < n; t0 += kResChunk) {
    const int len = min(kResChunk, n - t0);
    __syncthreads();
    for (int e = threadIdx.x; e < 4 * kResChunk; e += blockDim.x) {
      const int j = e / kResChunk, t = e % kResChunk;
      xs[j][t] = (j < nrhs && t < len) ? X[(size_t)j * n + t0 + t] : mkcd(0, 0);
    }
    __syncthreads();
    const int qn = (len + 31) >> 5;
#pragma unroll 4
    for (int q = 0; q < qn; ++q) {
      const int t = q * 32 + lane;
      const bool ok = t < len;
      cd av[kResRows];
#pragma unroll
      for (int i = 0; i < kResRows; ++i) av[i] = ok ? ldcs(arow[i] + t0 + t) : mkcd(0, 0);
      cd xv[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) xv[j] = xs[j][t];
#pragma unroll
      for (int i = 0; i < kResRows; ++i) {
        rs[i] += cabs1(av[i]);
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = acc[i][j] + av[i] * xv[j];
      }
    }
  }
#pragma unroll
  for (int i = 0; i < kResRows; ++i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      rs[i] += __shfl_xor_sync(0xffffffff, rs[i], o);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        acc[i][j].x += __shfl_xor_sync(0xffffffff, acc[i][j].x, o);
        acc[i][j].y += __shfl_xor_sync(0xffffffff, acc[i][j].y, o);
      }
    }
    const int row = r0 + i;
    if (row >= n) continue;
    if (lane == 0) atomicMax((unsigned long long *)&norms[kNA], (unsigned long long)__double_as_longlong(rs[i]));
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (j < nrhs && lane == j) {
        const cd r = B[(size_t)j * n + row] - acc[i][j];
        R[(size_t)j * n + row] = r;
        atomicMax((unsigned long long *)&norms[j], (unsigned long long)__double_as_longlong(cabs1(r)));
        const double xv = cabs1(X[(size_t)j * n + row]);
        atomicMax((unsigned long long *)&norms[kNX + j], (unsigned long long)__double_as_longlong(xv));
      }
    }
  }
}

__global__ void k_ir_check(int n, int nrhs, double *norms0, Ctrl ctrl, int *status0, int last) {
  int *cw = ctrl.of(blockIdx.x);
  int *done = cw + 2, *err = cw + 1, *status = status0 + blockIdx.x;
  double *norms = norms0 + (long long)blockIdx.x * kNormCount;
  if (*done) return;
  const double cte = 1.1102230246251565e-16 * sqrt((double)n) * norms[kNA];
  int ok = 1, bad = 0;
  for (int j = 0; j < nrhs; ++j) {
    double rn = norms[j], xn = norms[kNX + j];
    if (!(isfinite(rn) && isfinite(xn))) bad = 1;
    else if (rn > xn * cte) ok = 0;
  }
  if (*err) { bad = 1; *status |= PSS_ST_DEVICE_TIMEOUT; }
  if (bad) { *status |= PSS_ST_NONFINITE; *done = 1; }
  else if (ok) *done = 1;
  else if (last) { *status |= PSS_ST_REFINE_NOCONV; *done = 1; }
  for (int j = 0; j < nrhs; ++j) norms[j] = norms[kNX + j] = 0.0;
  norms[kNA] = 0.0;
}

__global__ void k_err_status(Ctrl ctrl, int *status0) {
  int *err = ctrl.of(blockIdx.x) + 1;
  if (*err) status0[blockIdx.x] |= PSS_ST_DEVICE_TIMEOUT;
  *err = 0;
}

__global__ void k_axpy(long long total, cd *X0, const cd *D0, long long vs, Ctrl ctrl) {
  const int bm = blockIdx.y;
  if (ctrl.of(bm)[2]) return;
  cd *X = X0 + bm * vs;
  const cd *D = D0 + bm * vs;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < total) X[i] = X[i] + D[i];
}

// y[perm[r]] = w[r] for every right-hand side: applies P^T after the adjoint passes.
__global__ void k_unpermute(int n, int nrhs, const int *__restrict__ perm0, const cd *__restrict__ W0,
                            cd *__restrict__ Y0, long long vs, Ctrl ctrl, int use_done) {
  const int bm = blockIdx.y;
  if (use_done && ctrl.of(bm)[2]) return;
  const int *perm = perm0 + (long long)bm * n;
  const cd *W = W0 + bm * vs;
  cd *Y = Y0 + bm * vs;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)n * nrhs) return;
  const int r = (int)(e % n), j = (int)(e / n);
  Y[(size_t)j * n + perm[r]] = W[e];
}

// Adjoint residual R = B - A^T Y, first stage: CTA (column block cb of 128, row chunk q of
// kTrRows) sums its rows for each column j and right-hand side, and the column's |a| sums
// (the infinity norm of A^T is the largest column sum of A), into part[q] (fixed order, no
// atomics; the second stage adds the chunks in order).  A thread owns a column, so every row
// of the chunk is read coalesced across the CTA.
constexpr int kTrRows = 256, kTrCols = 128;
__global__ void __launch_bounds__(kTrCols) k_resid_t1(int n, const cd *__restrict__ A0, long long ld, long long ms,
                                                      int nrhs, const cd *__restrict__ Y0, long long vs,
                                                      cd *__restrict__ part0, double *__restrict__ cabs0,
                                                      long long pstride, Ctrl ctrl) {
  const int bm = blockIdx.z;
  if (ctrl.of(bm)[2]) return;
  const cd *A = A0 + bm * ms, *Y = Y0 + bm * vs;
  const int j = blockIdx.x * kTrCols + threadIdx.x, q = blockIdx.y;
  const int i0 = q * kTrRows, i1 = min(n, i0 + kTrRows);
  const int nch = (int)gridDim.y;
  cd *part = part0 + (long long)bm * pstride;
  double *cabs = cabs0 + (long long)bm * nch * n;
  if (j >= n) return;
  for (int j0 = 0; j0 < nrhs; j0 += kMaxRhs) {
    const int nj = min(kMaxRhs, nrhs - j0);
    cd acc[kMaxRhs];
#pragma unroll
    for (int t = 0; t < kMaxRhs; ++t) acc[t] = mkcd(0, 0);
    double cs = 0.0;
    for (int i = i0; i < i1; ++i) {
      const cd a = A[(long long)i * ld + j];
      if (j0 == 0) cs += cabs1(a);
#pragma unroll
      for (int t = 0; t < kMaxRhs; ++t)
        if (t < nj) acc[t] = acc[t] + a * Y[(size_t)(j0 + t) * n + i];
    }
    if (j0 == 0) cabs[(long long)q * n + j] = cs;
#pragma unroll
    for (int t = 0; t < kMaxRhs; ++t)
      if (t < nj) part[((long long)q * nrhs + j0 + t) * n + j] = acc[t];
  }
}

// Second stage: R = B - sum of the chunks (in chunk order), with the refinement norms of
// k_resid: max|r_j| (norms[j]), max|y_j| (norms[kNX + j]) and ||A^T||_inf (norms[kNA]).
__global__ void k_resid_t2(int n, int nch, int nrhs, const cd *__restrict__ part0, const double *__restrict__ cabs0,
                           long long pstride, const cd *__restrict__ Y0, const cd *__restrict__ B0, cd *__restrict__ R0,
                           long long vs, double *norms0, Ctrl ctrl) {
  const int bm = blockIdx.y;
  if (ctrl.of(bm)[2]) return;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const cd *part = part0 + (long long)bm * pstride;
  const double *cabs = cabs0 + (long long)bm * nch * n;
  const cd *Y = Y0 + bm * vs, *B = B0 + bm * vs;
  cd *R = R0 + bm * vs;
  double *norms = norms0 + (long long)bm * kNormCount;
  double cs = 0.0;
  for (int q = 0; q < nch; ++q) cs += cabs[(long long)q * n + j];
  atomicMax((unsigned long long *)&norms[kNA], (unsigned long long)__double_as_longlong(cs));
  for (int t = 0; t < nrhs; ++t) {
    cd s = mkcd(0, 0);
    for (int q = 0; q < nch; ++q) s = s + part[((long long)q * nrhs + t) * n + j];
    const cd r = B[(size_t)t * n + j] - s;
    R[(size_t)t * n + j] = r;
    atomicMax((unsigned long long *)&norms[t], (unsigned long long)__double_as_longlong(cabs1(r)));
    atomicMax((unsigned long long *)&norms[kNX + t],
              (unsigned long long)__double_as_longlong(cabs1(Y[(size_t)t * n + j])));
  }
}

template <bool LOWER>
cudaError_t set_trsv_smem() {
  const int s64 = BS * BS * (int)sizeof(cd);
  cudaError_t e = cudaFuncSetAttribute(k_trsv<LOWER, false, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_trsv<LOWER, false, kMaxRhs>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_trsv<LOWER, false, 4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_trsv<LOWER, false, kMaxRhs, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64);
  return e;  // the FP32 forms stage 32 KB, under the default limit
}

}  // namespace

// ------------------------------- host side -------------------------------

size_t pss_solve_ws_bytes(int n, int nb) {
  int nblk = (n + BS - 1) / BS;
  return (size_t)nb * ((size_t)nblk * 2 * BS * BS * sizeof(cd) + (size_t)n * sizeof(int) +
                       (size_t)(nblk + 64) * sizeof(int) + kNormCount * sizeof(double)) + 512;
}

void SolveWS::bind(void *base, int n_, int nb_) {
  n = n_;
  nb = nb_;
  nblk = (n + BS - 1) / BS;
  dstride = (long long)nblk * 2 * BS * BS;
  cstride = nblk + 64;
  char *p = (char *)base;
  Dinv = (cd *)p;
  p += (size_t)nb * dstride * sizeof(cd);
  perm = (int *)p;
  p += (size_t)nb * n * sizeof(int);
  ctrl = (int *)p;  // per matrix: [0] ticket, [1] error, [2] converged, [8..8+nblk) flags
  p += (size_t)nb * cstride * sizeof(int);
  p = (char *)(((uintptr_t)p + 15) & ~(uintptr_t)15);
  norms = (double *)p;
}

// After the LU of nb matrices: pivot permutations and diagonal-block inverses; control
// words and norms cleared, epoch reset.
int pss_solve_prepare(SolveWS &ws, int nb, const cd *LU64, const float *Lr, const float *Li, long long ld,
                      long long ms, const int *ipiv, cudaStream_t st) {
  if (nb > ws.nb) { pss_set_error("solve workspace holds %d matrices, %d asked", ws.nb, nb); return -4; }
  Fac F{LU64, Lr, Li, ld, ms};
  pss_count_launch();
  k_ipiv_to_perm<<<nb, 1024, ws.n * sizeof(int), st>>>(ws.n, ipiv, ws.perm);
  static DeviceOnce once;
  if (int rc = device_once(once, [] {
        PSS_CUDA_TRY(
            cudaFuncSetAttribute(k_diag_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * BS * BS * (int)sizeof(cd)));
        return 0;
      }))
    return rc;
  pss_count_launch();
  k_diag_inv<<<dim3(ws.nblk, 2, nb), BS, 2 * BS * BS * sizeof(cd), st>>>(F, ws.n, ws.Dinv, ws.dstride);
  PSS_CUDA_TRY(cudaMemsetAsync(ws.ctrl, 0, (size_t)nb * ws.cstride * sizeof(int), st));
  PSS_CUDA_TRY(cudaMemsetAsync(ws.norms, 0, (size_t)nb * kNormCount * sizeof(double), st));
  ws.epoch = 0;
  return 0;
}

// X = (LU)^{-1} P B for each of nb matrices (B and X distinct, n x nrhs column-major, vs
// elements apart).  use_done: skip matrices whose refinement has converged.
int pss_solve_lu(SolveWS &ws, int nb, const cd *LU64, const float *Lr, const float *Li, long long ld, long long ms,
                 int nrhs, const cd *B, cd *X, long long vs, int use_done, cudaStream_t st) {
  Fac F{LU64, Lr, Li, ld, ms};
  const Ctrl ctrl{ws.ctrl, ws.cstride};
  static DeviceOnce once;
  if (int rc = device_once(once, [] {
        PSS_CUDA_TRY(set_trsv_smem<true>());
        PSS_CUDA_TRY(set_trsv_smem<false>());
        return 0;
      }))
    return rc;
  const bool f32 = LU64 == nullptr;
  for (int pass = 0; pass < 2; ++pass)
    for (int j0 = 0; j0 < nrhs; j0 += kMaxRhs) {
      ++ws.epoch;
      // tickets of every matrix back to zero (the flags keep their epochs)
      PSS_CUDA_TRY(cudaMemset2DAsync(ws.ctrl, ws.cstride * sizeof(int), 0, sizeof(int), nb, st));
      pss_count_launch();
      const bool small = nrhs - j0 <= 4;
      const dim3 grid(nb, ws.nblk);
      auto go = [&](auto kern, size_t smem) {
        kern<<<grid, 256, smem, st>>>(F, ws.n, ws.perm, B, X, vs, nrhs, j0, ws.Dinv, ws.dstride, ctrl, ws.epoch,
                                      use_done);
      };
      const size_t s64 = BS * BS * sizeof(cd), s32 = BS * BS * sizeof(cf);
      if (pass == 0) {
        if (f32) small ? go(k_trsv<true, true, 4>, s32) : go(k_trsv<true, true, kMaxRhs>, s32);
        else small ? go(k_trsv<true, false, 4>, s64) : go(k_trsv<true, false, kMaxRhs>, s64);
      } else {
        if (f32) small ? go(k_trsv<false, true, 4>, s32) : go(k_trsv<false, true, kMaxRhs>, s32);
        else small ? go(k_trsv<false, false, 4>, s64) : go(k_trsv<false, false, kMaxRhs>, s64);
      }
    }
  PSS_CUDA_TRY(cudaGetLastError());
  return 0;
}

// A timed-out wait in a solve (never expected) marks the point (status[b]).
void pss_solve_status(SolveWS &ws, int nb, int *status, cudaStream_t st) {
  pss_count_launch();
  k_err_status<<<nb, 1, 0, st>>>(Ctrl{ws.ctrl, ws.cstride}, status);
}

// Iterative refinement of each X_b against its FP64 matrix A_b (FP32 factors), up to
// maxit steps; matrices that converge drop out (their converged word).
int pss_refine(SolveWS &ws, int nb, const cd *A, long long ld, long long ms, const float *Lr, const float *Li,
               long long ldf, long long msf, int nrhs, const cd *B, cd *X, cd *R, cd *D, long long vs, int maxit, int *status, cudaStream_t st) {
  if (nrhs > kMaxRefRhs) { pss_set_error("refinement supports at most %d right-hand sides", kMaxRefRhs); return -1; }
  const Ctrl ctrl{ws.ctrl, ws.cstride};
  static DeviceOnce once;
  if (int rc = device_once(once, [] {
        PSS_CUDA_TRY(cudaFuncSetAttribute(k_resid4, cudaFuncAttributeMaxDynamicSharedMemorySize, kResSmem));
        return 0;
      }))
    return rc;
  // converged words of every matrix cleared
  PSS_CUDA_TRY(cudaMemset2DAsync(ws.ctrl + 2, ws.cstride * sizeof(int), 0, sizeof(int), nb, st));
  const long long total = (long long)ws.n * nrhs;
  for (int it = 0; it <= maxit; ++it) {
    pss_count_launch();
    if (nrhs <= 4)
      k_resid4<<<dim3(cdiv_u(ws.n, 8 * kResRows), nb), 256, kResSmem, st>>>(ws.n, A, ld, ms, nrhs, X, B, R, vs,
                                                                            ws.norms, ctrl);
    else
      k_resid<<<dim3(cdiv_u(ws.n, 8), nb), 256, 0, st>>>(ws.n, A, ld, ms, nrhs, X, B, R, vs, ws.norms, ctrl);
    pss_count_launch();
    k_ir_check<<<nb, 1, 0, st>>>(ws.n, nrhs, ws.norms, ctrl, status, it == maxit);
    if (it == maxit) break;
    int rc = pss_solve_lu(ws, nb, nullptr, Lr, Li, ldf, msf, nrhs, R, D, vs, 1, st);
    if (rc) return rc;
    pss_count_launch();
    k_axpy<<<dim3(cdiv_u(total, 256), nb), 256, 0, st>>>(total, X, D, vs, ctrl);
  }
  PSS_CUDA_TRY(cudaGetLastError());
  return 0;
}

// Adjoint solves Y = Z^-T B with the factors of P Z = L U (the same factors as pss_solve_lu,
// after pss_solve_prepare): U^T V = B, L^T W = V (both chained passes into W), Y = P^T W.
// W: scratch of the size of B.  use_done: skip matrices whose refinement has converged.
int pss_solve_lu_trans(SolveWS &ws, int nb, const cd *LU64, const float *Lr, const float *Li, long long ld,
                       long long ms, int nrhs, const cd *B, cd *Y, cd *W, long long vs, int use_done,
                       cudaStream_t st) {
  Fac F{LU64, Lr, Li, ld, ms};
  const Ctrl ctrl{ws.ctrl, ws.cstride};
  static DeviceOnce once;
  if (int rc = device_once(once, [] {
        PSS_CUDA_TRY(set_trsv_smem<true>());
        PSS_CUDA_TRY(set_trsv_smem<false>());
        return 0;
      }))
    return rc;
  const bool f32 = LU64 == nullptr;
  for (int pass = 0; pass < 2; ++pass)
    for (int j0 = 0; j0 < nrhs; j0 += kMaxRhs) {
      ++ws.epoch;
      PSS_CUDA_TRY(cudaMemset2DAsync(ws.ctrl, ws.cstride * sizeof(int), 0, sizeof(int), nb, st));
      pss_count_launch();
      const bool small = nrhs - j0 <= 4;
      const dim3 grid(nb, ws.nblk);
      auto go = [&](auto kern, size_t smem) {
        kern<<<grid, 256, smem, st>>>(F, ws.n, ws.perm, B, W, vs, nrhs, j0, ws.Dinv, ws.dstride, ctrl, ws.epoch,
                                      use_done);
      };
      const size_t s64 = BS * BS * sizeof(cd), s32 = BS * BS * sizeof(cf);
      if (pass == 0) {
        if (f32) small ? go(k_trsv<true, true, 4, true>, s32) : go(k_trsv<true, true, kMaxRhs, true>, s32);
        else small ? go(k_trsv<true, false, 4, true>, s64) : go(k_trsv<true, false, kMaxRhs, true>, s64);
      } else {
        if (f32) small ? go(k_trsv<false, true, 4, true>, s32) : go(k_trsv<false, true, kMaxRhs, true>, s32);
        else small ? go(k_trsv<false, false, 4, true>, s64) : go(k_trsv<false, false, kMaxRhs, true>, s64);
      }
    }
  pss_count_launch();
  k_unpermute<<<dim3(cdiv_u((long long)ws.n * nrhs, 256), nb), 256, 0, st>>>(ws.n, nrhs, ws.perm, W, Y, vs, ctrl,
                                                                          use_done);
  PSS_CUDA_TRY(cudaGetLastError());
  return 0;
}

// Scratch of the adjoint residual for nb matrices and nrhs right-hand sides (row-chunk partial
// sums and column sums).
size_t pss_refine_trans_ws_bytes(int n, int nrhs, int nb) {
  const size_t nch = (size_t)(n + kTrRows - 1) / kTrRows;
  return (size_t)nb * nch * ((size_t)nrhs * n * sizeof(cd) + (size_t)n * sizeof(double)) + 256;
}

// Iterative refinement of the adjoint solutions Y_b (Z_b^T Y_b = B_b) against the FP64
// matrices, as pss_refine: r = B - Z^T Y in FP64 (two-stage, fixed order), correction from the
// FP32 factors (pss_solve_lu_trans), the same stopping rule with ||Z^T||_inf.
int pss_refine_trans(SolveWS &ws, int nb, const cd *A, long long ld, long long ms, const float *Lr, const float *Li,
                     long long ldf, long long msf, int nrhs, const cd *B, cd *Y, cd *R, cd *D, cd *W, void *scratch, size_t scratch_bytes,
                     long long vs, int maxit, int *status, cudaStream_t st) {
  if (nrhs > kMaxRefRhs) { pss_set_error("refinement supports at most %d right-hand sides", kMaxRefRhs); return -1; }
  if (scratch_bytes < pss_refine_trans_ws_bytes(ws.n, nrhs, nb)) {
    pss_set_error("adjoint refinement scratch too small");
    return -4;
  }
  const Ctrl ctrl{ws.ctrl, ws.cstride};
  const int nch = (ws.n + kTrRows - 1) / kTrRows;
  const long long pstride = (long long)nch * nrhs * ws.n;
  cd *part = (cd *)scratch;
  double *cabs = (double *)(part + (size_t)nb * pstride);
  PSS_CUDA_TRY(cudaMemset2DAsync(ws.ctrl + 2, ws.cstride * sizeof(int), 0, sizeof(int), nb, st));
  const long long total = (long long)ws.n * nrhs;
  for (int it = 0; it <= maxit; ++it) {
    pss_count_launch();
    k_resid_t1<<<dim3(cdiv_u(ws.n, kTrCols), nch, nb), kTrCols, 0, st>>>(ws.n, A, ld, ms, nrhs, Y, vs, part, cabs,
                                                                        pstride, ctrl);
    pss_count_launch();
    k_resid_t2<<<dim3(cdiv_u(ws.n, 256), nb), 256, 0, st>>>(ws.n, nch, nrhs, part, cabs, pstride, Y, B, R, vs,
                                                            ws.norms, ctrl);
    pss_count_launch();
    k_ir_check<<<nb, 1, 0, st>>>(ws.n, nrhs, ws.norms, ctrl, status, it == maxit);
    if (it == maxit) break;
    int rc = pss_solve_lu_trans(ws, nb, nullptr, Lr, Li, ldf, msf, nrhs, R, D, W, vs, 1, st);
    if (rc) return rc;
    pss_count_launch();
    k_axpy<<<dim3(cdiv_u(total, 256), nb), 256, 0, st>>>(total, Y, D, vs, ctrl);
  }
  PSS_CUDA_TRY(cudaGetLastError());
  return 0;
}
