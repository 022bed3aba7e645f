// K4/K5: dense complex LU with partial pivoting and the multi-RHS solves.
//
// Replaces LAPACK zgetrf / zgetrs (LinearAlgebra.lu! / ldiv!, PSSFSS.jl:401,439).
// Matrices are row-major (row swaps are contiguous).  Blocked right-looking LU with a
// two-level panel:
//   * the narrow panel (W columns) is factored by one thread-block cluster: its rows are
//     spread over the CTAs' shared memory, each column's pivot is found by a CTA-local
//     argmax plus an exchange of candidates through distributed shared memory, and the
//     pivot row is broadcast the same way (two cluster barriers per column);
//   * pivots follow LAPACK izamax: largest |re|+|im|, first index on ties;
//   * row interchanges, the unit-lower TRSM of the block row and the Schur-complement
//     GEMM run as separate kernels.  In FP32 mode the matrix is two float planes
//     (real, imaginary) and the Schur update is the complex product written as real
//     products C_r -= L_r U_r - L_i U_i, C_i -= L_r U_i + L_i U_r.
// Solves: one CTA per right-hand-side set (latency-bound; batches of frequency points
// run concurrently on other SMs), FP64 arithmetic even with FP32 factors, so iterative
// refinement against the FP64 matrix recovers FP64 accuracy.
#include <cooperative_groups.h>
#include "pss_internal.cuh"

namespace cg = cooperative_groups;

namespace {

template <bool F32>
struct Prec;
template <>
struct Prec<false> {
  using R = double;
  struct E { double x, y; };
};
template <>
struct Prec<true> {
  using R = float;
  struct E { float x, y; };
};

template <class E>
__device__ __forceinline__ E cmulE(E a, E b) { return E{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
template <class E>
__device__ __forceinline__ E csubE(E a, E b) { return E{a.x - b.x, a.y - b.y}; }

// Matrix accessor: FP64 interleaved (A), FP32 planes (Ar, Ai).
template <bool F32>
struct Mat {
  void *a;
  float *ai;
  long long ld;
  __device__ __forceinline__ typename Prec<F32>::E get(long long r, long long c) const {
    if constexpr (F32) return {((float *)a)[r * ld + c], ai[r * ld + c]};
    else { cd v = ((cd *)a)[r * ld + c]; return {v.x, v.y}; }
  }
  __device__ __forceinline__ void put(long long r, long long c, typename Prec<F32>::E v) const {
    if constexpr (F32) { ((float *)a)[r * ld + c] = v.x; ai[r * ld + c] = v.y; }
    else ((cd *)a)[r * ld + c] = cd{v.x, v.y};
  }
};

constexpr int kPanelThreads = 512;

template <bool F32>
__global__ void __launch_bounds__(kPanelThreads) k_panel(Mat<F32> M, int row0, int nrows, int col0, int w,
                                                         int *ipiv, int *info) {
  using E = typename Prec<F32>::E;
  using Rl = typename Prec<F32>::R;
  cg::cluster_group cluster = cg::this_cluster();
  const int cs = (int)cluster.num_blocks();
  const int crank = (int)cluster.block_rank();
  const int tid = threadIdx.x, nth = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nth >> 5;
  const int rpc = (nrows + cs - 1) / cs;
  const int ws = w + 1;  // padded row stride in shared memory
  const int my0 = crank * rpc;
  const int myn = max(0, min(rpc, nrows - my0));
  extern __shared__ __align__(16) unsigned char smraw[];
  E *tile = (E *)smraw;
  E *prow = tile + (size_t)rpc * ws;
  E *oldj = prow + 32;
  double *candv = (double *)(oldj + 32);
  int *candi = (int *)(candv + 2);
  int *pivs = candi + 2;       // 32
  double *redv = (double *)(pivs + 32);
  int *redi = (int *)(redv + 32);
  int *bcast = redi + 32;      // [0] = p, [1] = singular

  for (int r = warp; r < myn; r += nwarp)
    for (int c = lane; c < w; c += 32) tile[r * ws + c] = M.get(row0 + my0 + r, col0 + c);
  __syncthreads();

  for (int j = 0; j < w; ++j) {
    // CTA-local argmax of |re|+|im| over panel rows >= j
    double best = -1.0;
    int bidx = 0x7fffffff;
    for (int r = tid; r < myn; r += nth) {
      int pr = my0 + r;
      if (pr < j) continue;
      E v = tile[r * ws + j];
      double a = fabs((double)v.x) + fabs((double)v.y);
      if (a > best || (a == best && pr < bidx)) { best = a; bidx = pr; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      double ob = __shfl_xor_sync(0xffffffff, best, o);
      int oi = __shfl_xor_sync(0xffffffff, bidx, o);
      if (ob > best || (ob == best && oi < bidx)) { best = ob; bidx = oi; }
    }
    if (lane == 0) { redv[warp] = best; redi[warp] = bidx; }
    __syncthreads();
    if (tid == 0) {
      for (int k = 1; k < nwarp; ++k)
        if (redv[k] > best || (redv[k] == best && redi[k] < bidx)) { best = redv[k]; bidx = redi[k]; }
      candv[j & 1] = best;
      candi[j & 1] = bidx;
    }
    cluster.sync();  // candidates visible cluster-wide
    if (tid == 0) {
      double gb = -1.0;
      int gi = 0x7fffffff;
      for (int c = 0; c < cs; ++c) {
        double *rv = cluster.map_shared_rank(candv, c);
        int *ri = cluster.map_shared_rank(candi, c);
        double v = rv[j & 1];
        int i = ri[j & 1];
        if (v > gb || (v == gb && i < gi)) { gb = v; gi = i; }
      }
      int sing = !(gb > 0.0);
      bcast[0] = sing ? j : gi;
      bcast[1] = sing;
      if (crank == 0) pivs[j] = bcast[0];
    }
    __syncthreads();
    const int p = bcast[0];
    const int sing = bcast[1];
    const int op = p / rpc, rp = p % rpc, oj = j / rpc, rj = j % rpc;
    {
      E *tp = cluster.map_shared_rank(tile, op);
      for (int c = tid; c < w; c += nth) prow[c] = tp[rp * ws + c];
      if (crank == op && p != j) {
        E *tj = cluster.map_shared_rank(tile, oj);
        for (int c = tid; c < w; c += nth) oldj[c] = tj[rj * ws + c];
      }
    }
    cluster.sync();  // all remote reads of rows j and p done
    if (p != j) {
      if (crank == oj)
        for (int c = tid; c < w; c += nth) tile[rj * ws + c] = prow[c];
      if (crank == op)
        for (int c = tid; c < w; c += nth) tile[rp * ws + c] = oldj[c];
    }
    __syncthreads();
    if (!sing) {
      E piv = prow[j];
      Rl den = piv.x * piv.x + piv.y * piv.y;
      // reciprocal of the pivot (LAPACK zgetf2 scales by 1/pivot)
      E inv;
      if (fabs((double)piv.y) <= fabs((double)piv.x)) {
        Rl rr = piv.y / piv.x, d = piv.x + piv.y * rr;
        inv = E{(Rl)1 / d, -rr / d};
      } else {
        Rl rr = piv.x / piv.y, d = piv.y + piv.x * rr;
        inv = E{rr / d, (Rl)-1 / d};
      }
      (void)den;
      for (int r = warp; r < myn; r += nwarp) {
        int pr = my0 + r;
        if (pr <= j) continue;
        E l = cmulE(tile[r * ws + j], inv);
        for (int c = j + 1 + lane; c < w; c += 32) tile[r * ws + c] = csubE(tile[r * ws + c], cmulE(l, prow[c]));
        if (lane == 0) tile[r * ws + j] = l;
      }
    }
    if (sing && tid == 0 && crank == 0) atomicCAS(info, 0, col0 + j + 1);
    __syncthreads();
  }
  for (int r = warp; r < myn; r += nwarp)
    for (int c = lane; c < w; c += 32) M.put(row0 + my0 + r, col0 + c, tile[r * ws + c]);
  if (crank == 0)
    for (int j = tid; j < w; j += nth) ipiv[col0 + j] = row0 + pivs[j];
}

// Apply swaps k = k0..k0+cnt-1 (row k <-> ipiv[k]) to columns [c0, c1).
template <bool F32>
__global__ void k_laswp(Mat<F32> M, int k0, int cnt, const int *ipiv, int c0, int c1) {
  int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= c1) return;
  for (int k = k0; k < k0 + cnt; ++k) {
    int p = ipiv[k];
    if (p != k) {
      auto a = M.get(k, c), b = M.get(p, c);
      M.put(k, c, b);
      M.put(p, c, a);
    }
  }
}

// Rows k0..k0+kb-1, columns [c0, c1): X = L11^{-1} X with L11 unit lower (in A).
template <bool F32>
__global__ void __launch_bounds__(32) k_trsm(Mat<F32> M, int k0, int kb, int c0, int c1) {
  using E = typename Prec<F32>::E;
  extern __shared__ __align__(16) unsigned char smraw[];
  E *xs = (E *)smraw;  // kb x 32
  int c = c0 + blockIdx.x * 32 + threadIdx.x;
  bool ok = c < c1;
  for (int i = 0; i < kb; ++i) {
    E v = ok ? M.get(k0 + i, c) : E{0, 0};
    for (int t = 0; t < i; ++t) v = csubE(v, cmulE(M.get(k0 + i, k0 + t), xs[t * 32 + threadIdx.x]));
    xs[i * 32 + threadIdx.x] = v;
    if (ok) M.put(k0 + i, c, v);
  }
}

// C[r0:r1, c0:c1] -= A[r0:r1, k0:k0+kb] * A[k0:k0+kb, c0:c1]  (FP64 complex, SIMT, 64x64 tiles)
__global__ void __launch_bounds__(256) k_gemm64(cd *A, long long ld, int r0, int r1, int c0, int c1, int k0, int kb) {
  __shared__ cd As[16][64 + 1];
  __shared__ cd Bs[16][64 + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int rb = r0 + blockIdx.y * 64, cb = c0 + blockIdx.x * 64;
  cd acc[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) acc[i][j] = mkcd(0, 0);
  for (int kk = 0; kk < kb; kk += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      int i = e / 16, t = e % 16;  // A tile: row i, k t
      int r = rb + i, k = k0 + kk + t;
      As[t][i] = (r < r1 && kk + t < kb) ? A[(long long)r * ld + k] : mkcd(0, 0);
      int t2 = e / 64, j = e % 64;  // B tile: k t2, col j
      int cc = cb + j, k2 = k0 + kk + t2;
      Bs[t2][j] = (cc < c1 && kk + t2 < kb) ? A[(long long)k2 * ld + cc] : mkcd(0, 0);
    }
    __syncthreads();
#pragma unroll 4
    for (int t = 0; t < 16; ++t) {
      cd a[4], b[4];
      for (int i = 0; i < 4; ++i) a[i] = As[t][ty + 16 * i];
      for (int j = 0; j < 4; ++j) b[j] = Bs[t][tx + 16 * j];
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x = fma(a[i].x, b[j].x, fma(-a[i].y, b[j].y, acc[i][j].x));
          acc[i][j].y = fma(a[i].x, b[j].y, fma(a[i].y, b[j].x, acc[i][j].y));
        }
    }
    __syncthreads();
  }
  for (int i = 0; i < 4; ++i) {
    int r = rb + ty + 16 * i;
    if (r >= r1) continue;
    for (int j = 0; j < 4; ++j) {
      int cc = cb + tx + 16 * j;
      if (cc >= c1) continue;
      cd &z = A[(long long)r * ld + cc];
      z = z - acc[i][j];
    }
  }
}

// FP32 planes variant (SIMT).
__global__ void __launch_bounds__(256) k_gemm32(float *Ar, float *Ai, long long ld, int r0, int r1, int c0, int c1,
                                                int k0, int kb) {
  __shared__ float Asr[16][128 + 4], Asi[16][128 + 4];
  __shared__ float Bsr[16][128 + 4], Bsi[16][128 + 4];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int rb = r0 + blockIdx.y * 128, cb = c0 + blockIdx.x * 128;
  float cr[8][8], ci[8][8];
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) cr[i][j] = ci[i][j] = 0.f;
  for (int kk = 0; kk < kb; kk += 16) {
    for (int e = threadIdx.x; e < 16 * 128; e += 256) {
      int i = e / 16, t = e % 16;
      int r = rb + i, k = k0 + kk + t;
      bool v = r < r1 && kk + t < kb;
      Asr[t][i] = v ? Ar[(long long)r * ld + k] : 0.f;
      Asi[t][i] = v ? Ai[(long long)r * ld + k] : 0.f;
      int t2 = e / 128, j = e % 128;
      int cc = cb + j, k2 = k0 + kk + t2;
      bool v2 = cc < c1 && kk + t2 < kb;
      Bsr[t2][j] = v2 ? Ar[(long long)k2 * ld + cc] : 0.f;
      Bsi[t2][j] = v2 ? Ai[(long long)k2 * ld + cc] : 0.f;
    }
    __syncthreads();
#pragma unroll 2
    for (int t = 0; t < 16; ++t) {
      float ar[8], ai[8], br[8], bi[8];
      for (int i = 0; i < 8; ++i) { ar[i] = Asr[t][ty + 16 * i]; ai[i] = Asi[t][ty + 16 * i]; }
      for (int j = 0; j < 8; ++j) { br[j] = Bsr[t][tx + 16 * j]; bi[j] = Bsi[t][tx + 16 * j]; }
      for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) {
          cr[i][j] = fmaf(ar[i], br[j], fmaf(-ai[i], bi[j], cr[i][j]));
          ci[i][j] = fmaf(ar[i], bi[j], fmaf(ai[i], br[j], ci[i][j]));
        }
    }
    __syncthreads();
  }
  for (int i = 0; i < 8; ++i) {
    int r = rb + ty + 16 * i;
    if (r >= r1) continue;
    for (int j = 0; j < 8; ++j) {
      int cc = cb + tx + 16 * j;
      if (cc >= c1) continue;
      long long o = (long long)r * ld + cc;
      Ar[o] -= cr[i][j];
      Ai[o] -= ci[i][j];
    }
  }
}

// ---- solves (one CTA of 1024 threads per call) ----
template <bool F32>
__device__ __forceinline__ cd lu_at(const Mat<F32> &M, long long r, long long c) {
  auto v = M.get(r, c);
  return mkcd((double)v.x, (double)v.y);
}

template <bool F32>
__global__ void __launch_bounds__(1024) k_solve(Mat<F32> M, int n, const int *ipiv, int nrhs, cd *B,
                                                const int *done) {
  if (done && *done) return;
  __shared__ cd part[32][8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // row interchanges (sequential, one thread per rhs)
  if (tid < nrhs) {
    cd *b = B + (size_t)tid * n;
    for (int k = 0; k < n; ++k) {
      int p = ipiv[k];
      if (p != k) { cd t = b[k]; b[k] = b[p]; b[p] = t; }
    }
  }
  __syncthreads();
  for (int j0 = 0; j0 < nrhs; j0 += 8) {
    const int nj = min(8, nrhs - j0);
    // forward: unit lower
    for (int blk = 0; blk < n; blk += 32) {
      const int nr = min(32, n - blk);
      if (warp < nr) {
        const int row = blk + warp;
        cd acc[8];
        for (int j = 0; j < 8; ++j) acc[j] = mkcd(0, 0);
        for (int t = lane; t < blk; t += 32) {
          cd l = lu_at<F32>(M, row, t);
          for (int j = 0; j < nj; ++j) acc[j] = acc[j] + l * B[(size_t)(j0 + j) * n + t];
        }
        for (int j = 0; j < nj; ++j)
          for (int o = 16; o > 0; o >>= 1) {
            acc[j].x += __shfl_xor_sync(0xffffffff, acc[j].x, o);
            acc[j].y += __shfl_xor_sync(0xffffffff, acc[j].y, o);
          }
        if (lane == 0)
          for (int j = 0; j < nj; ++j) part[warp][j] = B[(size_t)(j0 + j) * n + row] - acc[j];
      }
      __syncthreads();
      if (warp == 0 && lane < nj) {
        cd *b = B + (size_t)(j0 + lane) * n;
        for (int i = 0; i < nr; ++i) {
          cd v = part[i][lane];
          for (int t = 0; t < i; ++t) v = v - lu_at<F32>(M, blk + i, blk + t) * b[blk + t];
          b[blk + i] = v;
        }
      }
      __syncthreads();
    }
    // backward: upper with diagonal
    for (int top = n; top > 0; top -= 32) {
      const int blk = max(0, top - 32);
      const int nr = top - blk;
      if (warp < nr) {
        const int row = blk + warp;
        cd acc[8];
        for (int j = 0; j < 8; ++j) acc[j] = mkcd(0, 0);
        for (int t = top + lane; t < n; t += 32) {
          cd u = lu_at<F32>(M, row, t);
          for (int j = 0; j < nj; ++j) acc[j] = acc[j] + u * B[(size_t)(j0 + j) * n + t];
        }
        for (int j = 0; j < nj; ++j)
          for (int o = 16; o > 0; o >>= 1) {
            acc[j].x += __shfl_xor_sync(0xffffffff, acc[j].x, o);
            acc[j].y += __shfl_xor_sync(0xffffffff, acc[j].y, o);
          }
        if (lane == 0)
          for (int j = 0; j < nj; ++j) part[warp][j] = B[(size_t)(j0 + j) * n + row] - acc[j];
      }
      __syncthreads();
      if (warp == 0 && lane < nj) {
        cd *b = B + (size_t)(j0 + lane) * n;
        for (int i = nr - 1; i >= 0; --i) {
          cd v = part[i][lane];
          for (int t = i + 1; t < nr; ++t) v = v - lu_at<F32>(M, blk + i, blk + t) * b[blk + t];
          b[blk + i] = v / lu_at<F32>(M, blk + i, blk + i);
        }
      }
      __syncthreads();
    }
  }
}

// R = B - A X  (A row-major FP64), one warp per row.
__global__ void __launch_bounds__(256) k_residual(int n, const cd *A, long long ld, int nrhs, const cd *X,
                                                  const cd *B, cd *Rr, const int *done) {
  if (done && *done) return;
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (row >= n) return;
  for (int j0 = 0; j0 < nrhs; j0 += 8) {
    const int nj = min(8, nrhs - j0);
    cd acc[8];
    for (int j = 0; j < 8; ++j) acc[j] = mkcd(0, 0);
    const cd *a = A + (long long)row * ld;
    for (int t = lane; t < n; t += 32) {
      cd av = a[t];
      for (int j = 0; j < nj; ++j) acc[j] = acc[j] + av * X[(size_t)(j0 + j) * n + t];
    }
    for (int j = 0; j < nj; ++j)
      for (int o = 16; o > 0; o >>= 1) {
        acc[j].x += __shfl_xor_sync(0xffffffff, acc[j].x, o);
        acc[j].y += __shfl_xor_sync(0xffffffff, acc[j].y, o);
      }
    if (lane == 0)
      for (int j = 0; j < nj; ++j) Rr[(size_t)(j0 + j) * n + row] = B[(size_t)(j0 + j) * n + row] - acc[j];
  }
}

__device__ __forceinline__ void atomic_max_pos(double *addr, double v) {
  atomicMax((unsigned long long *)addr, (unsigned long long)__double_as_longlong(v));
}

// X += D; norms[0] = max|D|, norms[1] = max|X| (over all entries).
__global__ void k_axpy_norms(long long total, cd *X, const cd *D, double *norms, const int *done) {
  if (done && *done) return;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double md = 0, mx = 0;
  if (i < total) {
    cd x = X[i] + D[i];
    X[i] = x;
    md = fmax(fabs(D[i].x), fabs(D[i].y));
    mx = fmax(fabs(x.x), fabs(x.y));
  }
  for (int o = 16; o > 0; o >>= 1) {
    md = fmax(md, __shfl_xor_sync(0xffffffff, md, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffff, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(&norms[0], md);
    atomic_max_pos(&norms[1], mx);
  }
}

}  // namespace

// ------------------------------- host side -------------------------------

namespace {
constexpr int kClusterCTAs = 8;
constexpr size_t kPanelSmemCap = 220 * 1024;

template <bool F32>
size_t panel_smem(int nrows, int w) {
  using E = typename Prec<F32>::E;
  int rpc = (nrows + kClusterCTAs - 1) / kClusterCTAs;
  return (size_t)rpc * (w + 1) * sizeof(E) + 64 * sizeof(E) + 2 * sizeof(double) + 2 * sizeof(int) +
         32 * sizeof(int) + 32 * sizeof(double) + 32 * sizeof(int) + 2 * sizeof(int) + 64;
}

template <bool F32>
int launch_panel(Mat<F32> M, int row0, int nrows, int col0, int w, int *ipiv, int *info, cudaStream_t st) {
  size_t smem = panel_smem<F32>(nrows, w);
  if (smem > kPanelSmemCap) {
    pss_set_error("panel %d x %d does not fit a %d-CTA cluster", nrows, w, kClusterCTAs);
    return -6;
  }
  static bool attr[2] = {false, false};
  if (!attr[F32]) {
    cudaFuncSetAttribute(k_panel<F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelSmemCap);
    attr[F32] = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kClusterCTAs);
  cfg.blockDim = dim3(kPanelThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = kClusterCTAs;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  pss_count_launch();
  PSS_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_panel<F32>, M, row0, nrows, col0, w, ipiv, info));
  return 0;
}

template <bool F32>
void launch_laswp(Mat<F32> M, int k0, int cnt, const int *ipiv, int c0, int c1, cudaStream_t st) {
  if (c1 <= c0) return;
  pss_count_launch();
  k_laswp<F32><<<cdiv_u(c1 - c0, 256), 256, 0, st>>>(M, k0, cnt, ipiv, c0, c1);
}

template <bool F32>
void launch_trsm(Mat<F32> M, int k0, int kb, int c0, int c1, cudaStream_t st) {
  if (c1 <= c0) return;
  size_t smem = (size_t)kb * 32 * sizeof(typename Prec<F32>::E);
  static bool attr[2] = {false, false};
  if (!attr[F32]) {
    cudaFuncSetAttribute(k_trsm<F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr[F32] = true;
  }
  pss_count_launch();
  k_trsm<F32><<<cdiv_u(c1 - c0, 32), 32, smem, st>>>(M, k0, kb, c0, c1);
}

void launch_gemm(Mat<false> M, int r0, int r1, int c0, int c1, int k0, int kb, cudaStream_t st) {
  if (r1 <= r0 || c1 <= c0) return;
  pss_count_launch();
  k_gemm64<<<dim3(cdiv_u(c1 - c0, 64), cdiv_u(r1 - r0, 64)), 256, 0, st>>>((cd *)M.a, M.ld, r0, r1, c0, c1, k0, kb);
}
void launch_gemm(Mat<true> M, int r0, int r1, int c0, int c1, int k0, int kb, cudaStream_t st) {
  if (r1 <= r0 || c1 <= c0) return;
  pss_count_launch();
  k_gemm32<<<dim3(cdiv_u(c1 - c0, 128), cdiv_u(r1 - r0, 128)), 256, 0, st>>>((float *)M.a, M.ai, M.ld, r0, r1, c0,
                                                                             c1, k0, kb);
}

template <bool F32>
int lu_blocked(int n, Mat<F32> M, int *ipiv, int *info, int NB, int W, cudaStream_t st) {
  for (int K0 = 0; K0 < n; K0 += NB) {
    const int JB = min(NB, n - K0);
    for (int k0 = K0; k0 < K0 + JB; k0 += W) {
      const int w = min(W, K0 + JB - k0);
      int rc = launch_panel<F32>(M, k0, n - k0, k0, w, ipiv, info, st);
      if (rc) return rc;
      launch_laswp<F32>(M, k0, w, ipiv, K0, k0, st);
      launch_laswp<F32>(M, k0, w, ipiv, k0 + w, K0 + JB, st);
      if (k0 + w < K0 + JB) {
        launch_trsm<F32>(M, k0, w, k0 + w, K0 + JB, st);
        launch_gemm(M, k0 + w, n, k0 + w, K0 + JB, k0, w, st);
      }
    }
    launch_laswp<F32>(M, K0, JB, ipiv, 0, K0, st);
    launch_laswp<F32>(M, K0, JB, ipiv, K0 + JB, n, st);
    if (K0 + JB < n) {
      launch_trsm<F32>(M, K0, JB, K0 + JB, n, st);
      launch_gemm(M, K0 + JB, n, K0 + JB, n, K0, JB, st);
    }
  }
  PSS_CUDA_TRY(cudaGetLastError());
  return 0;
}

template <bool F32>
int pick_panel_width(int n, int want) {
  int w = want;
  while (w > 4 && panel_smem<F32>(n, w) > kPanelSmemCap) w /= 2;
  if (panel_smem<F32>(n, w) > kPanelSmemCap) return -1;
  return w;
}
}  // namespace

size_t pss_lu_ws_bytes(int n, int precision) { (void)n; (void)precision; return 0; }

int pss_lu64(int n, cd *A, long long ld, int *ipiv, int *info, void *ws, size_t ws_bytes, cudaStream_t st) {
  (void)ws; (void)ws_bytes;
  Mat<false> M{A, nullptr, ld};
  int W = pick_panel_width<false>(n, 16);
  if (W < 0) { pss_set_error("matrix order %d too large for the cluster panel", n); return -6; }
  return lu_blocked<false>(n, M, ipiv, info, 64, W, st);
}

int pss_lu32(int n, float *Ar, float *Ai, long long ld, int *ipiv, int *info, void *ws, size_t ws_bytes,
             cudaStream_t st) {
  (void)ws; (void)ws_bytes;
  Mat<true> M{Ar, Ai, ld};
  int W = pick_panel_width<true>(n, 32);
  if (W < 0) { pss_set_error("matrix order %d too large for the cluster panel", n); return -6; }
  return lu_blocked<true>(n, M, ipiv, info, 128, W, st);
}

void pss_solve64(int n, const cd *LU, long long ld, const int *ipiv, int nrhs, cd *B, const int *done,
                 cudaStream_t st) {
  Mat<false> M{(void *)LU, nullptr, ld};
  pss_count_launch();
  k_solve<false><<<1, 1024, 0, st>>>(M, n, ipiv, nrhs, B, done);
}

void pss_solve32(int n, const float *Lr, const float *Li, long long ld, const int *ipiv, int nrhs, cd *B,
                 const int *done, cudaStream_t st) {
  Mat<true> M{(void *)Lr, (float *)Li, ld};
  pss_count_launch();
  k_solve<true><<<1, 1024, 0, st>>>(M, n, ipiv, nrhs, B, done);
}

void pss_residual64(int n, const cd *A, long long ld, int nrhs, const cd *X, const cd *B, cd *Rout,
                    const int *done, cudaStream_t st) {
  pss_count_launch();
  k_residual<<<cdiv_u(n, 8), 256, 0, st>>>(n, A, ld, nrhs, X, B, Rout, done);
}

void pss_axpy_norms(int n, int nrhs, cd *X, const cd *D, double *norms, const int *done, cudaStream_t st) {
  long long total = (long long)n * nrhs;
  pss_count_launch();
  k_axpy_norms<<<cdiv_u(total, 256), 256, 0, st>>>(total, X, D, norms, done);
}

namespace {
// After a refinement step: converged when max|dx| <= tol * max|x|.  Resets the norm
// accumulators for the next step; on the last step records non-convergence.
__global__ void k_refine_check(double *norms, double tol, int *done, int *status, int last) {
  if (*done) return;
  double dn = norms[0], xn = norms[1];
  bool finite = isfinite(dn) && isfinite(xn);
  if (!finite) { *status |= PSS_ST_NONFINITE; *done = 1; }
  else if (dn <= tol * xn) *done = 1;
  else if (last) *status |= PSS_ST_REFINE_NOCONV;
  norms[0] = 0.0;
  norms[1] = 0.0;
}
}  // namespace

void pss_refine_check(double *norms, double tol, int *done, int *status, int last, cudaStream_t st) {
  pss_count_launch();
  k_refine_check<<<1, 1, 0, st>>>(norms, tol, done, status, last);
}
