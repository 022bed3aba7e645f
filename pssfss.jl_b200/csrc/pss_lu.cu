// K4: dense complex LU with partial pivoting (replaces LAPACK zgetrf behind lu!,
// PSSFSS.jl:401, 526).
//
// Matrices are row-major (row interchanges are contiguous).  Blocked right-looking LU in
// LAPACK zgetrf order, two-level: an outer block of NB columns is factored as panels of W.
//   * k_panel: a thread-block cluster of ceil(rows / 512) CTAs (<= 16) owns a W-column
//     panel, 512 rows per CTA in shared memory.  For each column every CTA reduces its
//     pivot candidates (|re|+|im| as LAPACK izamax, lowest row on ties) with redux.sync,
//     pushes its candidate (key, row index, entries) into every CTA's shared memory, one
//     cluster barrier makes them visible, and every CTA picks the same winner and updates
//     its own rows.  At the end every CTA replays the interchange sequence in shared memory
//     (a sparse map of the <= 2W moved positions), CTA 0 writes ipiv and a compact
//     interchange list, and the rows are copied to their final positions.
//   * k_laswp applies that list to all other columns in one launch.
//   * k_trsm_small: the W-row block-row solve L11^{-1} X, one column per thread.
//   * the Schur complement A22 -= L21 U12: k_gemm64 (FP64, SIMT), and in FP32 mode
//     k_gemm32 for the skinny updates inside an outer block and the tcgen05 3xTF32 kernel
//     (pss_gemm_tc.cu) for the trailing update of each outer block.
// In FP32 mode the matrix is two float planes (real, imaginary).
#include <cooperative_groups.h>
#include <type_traits>

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
template <class E>
__device__ __forceinline__ E caddE(E a, E b) { return E{a.x + b.x, a.y + b.y}; }

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
  // matrix b of a batch whose matrices are ms elements apart
  __host__ __device__ __forceinline__ Mat at(int b, long long ms) const {
    if constexpr (F32) return Mat{(float *)a + b * ms, ai + b * ms, ld};
    else return Mat{(cd *)a + b * ms, nullptr, ld};
  }
};

// A batch of independent factorisations of the same order: matrix b at M.at(b, ms), its
// pivots at ipiv + b*n, its info word at info + b, its panel interchange list at
// xlist + b*kListInts.  Every kernel below takes the matrix index from its grid.
struct LuBatch {
  long long ms;
  int n;
  int *ipiv, *info, *xlist;
};

#ifndef PSS_PANEL_ROWS
#define PSS_PANEL_ROWS 512
#endif
#ifndef PSS_PANEL_RPT
#define PSS_PANEL_RPT 2
#endif
constexpr int kPanelRows = PSS_PANEL_ROWS;  // panel rows per CTA
constexpr int kPanelRpt = PSS_PANEL_RPT;  // panel rows per thread
constexpr int kMaxCluster = 16;
constexpr int kMaxW = 32;
constexpr int kMaxMov = 2 * kMaxW;  // rows one panel's interchanges can move
constexpr int kSwpThreads = 64;
constexpr int kListInts = 1 + 2 * kMaxMov;  // interchange list: count, destinations, sources
constexpr int kTcMinRows = 64, kTcMinCols = 32;  // smallest FP32 update sent to the tensor cores
static_assert(kPanelRows / kPanelRpt / 32 <= 32 && kMaxCluster <= 32, "panel reductions run over one warp's lanes");

// Pivot keys: LAPACK's izamax order (largest |re|+|im|, then the lowest row) as one 64-bit
// unsigned key per candidate, 0 = no candidate, 1 = an exactly zero candidate.  The bits
// of a non-negative float or double are monotonic, so the largest key is the largest
// value; among equal keys the lowest lane wins, and lanes, warps and cluster ranks are in
// row order.  A warp reduces with redux.sync (one instruction per 32-bit half).
template <bool F32>
__device__ __forceinline__ unsigned long long piv_key(typename Prec<F32>::E v, bool act) {
  if (!act) return 0ull;
  if constexpr (F32) return (unsigned long long)__float_as_uint(fabsf(v.x) + fabsf(v.y)) + 1ull;
  else return (unsigned long long)__double_as_longlong(fabs(v.x) + fabs(v.y)) + 1ull;
}
// Warp-wide maximum key and, among the lanes holding it, the lowest row (all lanes get both):
// exactly izamax's choice whatever the lane order of the rows.
template <bool F32>
__device__ __forceinline__ unsigned long long warp_max_key(unsigned long long k, int r, int &win_row) {
  const unsigned lo = (unsigned)k;
  unsigned long long m;
  bool mine;
  if constexpr (F32) {  // keys fit in 32 bits
    const unsigned ml = __reduce_max_sync(0xffffffffu, lo);
    m = ml;
    mine = lo == ml;
  } else {
    const unsigned hi = (unsigned)(k >> 32);
    const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
    const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? lo : 0u);
    m = ((unsigned long long)mh << 32) | ml;
    mine = hi == mh && lo == ml;
  }
  win_row = (int)__reduce_min_sync(0xffffffffu, mine ? (unsigned)r : 0x7fffffffu);
  return m;
}

// Panel of W columns (w <= W used), rows row0..row0+nrows-1, factored by a cluster of
// cs = gridDim.x CTAs of 256 threads; CTA q owns panel rows q*512 .. q*512+511, held in its
// shared memory column by column (R[c][local row], conflict-free for a warp), and thread t
// works on local rows t and 256 + t.  Per column: the two rows' pivot keys are reduced per
// warp (redux.sync), one CTA barrier, per CTA; warp 0 pushes the CTA's candidate (key, row
// index and its entries j..w-1, read from shared memory) into every CTA's shared memory;
// one cluster barrier; every CTA picks the same winner and updates its active rows over
// the live columns only.  Multipliers overwrite the rows in place, pivot rows keep their U
// entries, so the final write-back is a coalesced copy to the permuted positions.
template <bool F32, int W, int RPT>
__global__ void __launch_bounds__(kPanelRows / RPT) k_panel(Mat<F32> M0, LuBatch bt, int row0, int nrows, int col0,
                                                            int w) {
  using E = typename Prec<F32>::E;
  using Rl = typename Prec<F32>::R;
  constexpr int T = kPanelRows / RPT;  // threads; thread t works on local rows t + k*T, k < RPT
  cg::cluster_group cluster = cg::this_cluster();
  const int cs = (int)cluster.num_blocks();
  const int crank = (int)cluster.block_rank();
  const int bidx = blockIdx.x / cs;  // one cluster per matrix of the batch
  const Mat<F32> M = M0.at(bidx, bt.ms);
  int *ipiv = bt.ipiv + (long long)bidx * bt.n, *info = bt.info + bidx, *xlist = bt.xlist + bidx * kListInts;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = T / 32;
  extern __shared__ __align__(16) unsigned char panel_smem[];
  E *R = (E *)panel_smem;                      // [W][kPanelRows] the CTA's panel rows
  __shared__ E srow[2][kMaxCluster][W];        // candidate rows pushed by every CTA (double-buffered)
  __shared__ unsigned long long skey[2][kMaxCluster];
  __shared__ int sidx[2][kMaxCluster];         // their panel rows
  __shared__ unsigned long long wkey[NW];      // per-warp winners
  __shared__ int wrow[NW];
  __shared__ int chosen[kMaxW];
  __shared__ int sdst[kPanelRows];             // final panel position of each local row
  const int base = crank * kPanelRows;
  const int nloc = max(0, min(kPanelRows, nrows - base));  // rows this CTA owns
  // coalesced load: one row per warp step, one column per lane, LB rows of a warp in flight
  constexpr int LB = F32 ? 16 : 8;
  static_assert(kPanelRows % (NW * LB) == 0, "panel rows split evenly into load batches");
  for (int r0 = warp; r0 < kPanelRows; r0 += NW * LB) {
    E t[LB];
#pragma unroll
    for (int u = 0; u < LB; ++u) {
      const int r = r0 + u * NW;
      t[u] = (r < nloc && lane < w) ? M.get(row0 + base + r, col0 + lane) : E{0, 0};
    }
    if (lane < W) {
#pragma unroll
      for (int u = 0; u < LB; ++u) R[lane * kPanelRows + r0 + u * NW] = t[u];
    }
  }
  bool act[RPT];
#pragma unroll
  for (int k = 0; k < RPT; ++k) act[k] = tid + k * T < nloc;
  __syncthreads();

  for (int j = 0; j < w; ++j) {
    const int par = j & 1;
    E v[RPT];
    unsigned long long k = 0ull;
    int r = base + tid;
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      v[q] = R[j * kPanelRows + tid + q * T];
      const unsigned long long kq = piv_key<F32>(v[q], act[q]);
      if (kq > k) { k = kq; r = base + tid + q * T; }  // equal keys keep the lower row
    }
    int wr;
    k = warp_max_key<F32>(k, r, wr);
    if (lane == 0) { wkey[warp] = k; wrow[warp] = wr; }
    __syncthreads();
    if (warp == 0) {  // the CTA's candidate, pushed to slot [par][crank] of every CTA
      int cr;
      const unsigned long long kc =
          warp_max_key<F32>(lane < NW ? wkey[lane] : 0ull, lane < NW ? wrow[lane] : 0x7fffffff, cr);
      const int lr = kc ? cr - base : 0;
      const E pv = (lane < W && j + lane < w) ? R[(j + lane) * kPanelRows + lr] : E{0, 0};
      if (lane < W && j + lane < w)
        for (int dst = 0; dst < cs; ++dst)
          cluster.map_shared_rank(&srow[0][0][0], dst)[(par * kMaxCluster + crank) * W + j + lane] = pv;
      if (lane < cs) {
        cluster.map_shared_rank(&skey[0][0], lane)[par * kMaxCluster + crank] = kc;
        cluster.map_shared_rank(&sidx[0][0], lane)[par * kMaxCluster + crank] = cr;
      }
    }
    cluster.sync();
    int grow;
    const unsigned long long kg =
        warp_max_key<F32>(lane < cs ? skey[par][lane] : 0ull, lane < cs ? sidx[par][lane] : 0x7fffffff, grow);
    const bool sing = kg <= 1ull;  // no candidate, or an exactly zero one
    if (tid == 0) chosen[j] = sing ? -1 : grow;
    if (sing) {  // zero column: nothing to eliminate (LAPACK skips the scaling)
      if (tid == 0 && crank == 0) atomicCAS(info, 0, col0 + j + 1);
      continue;
    }
    bool any = false;
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      if (base + tid + q * T == grow) act[q] = false;  // the pivot row keeps its entries (row of U)
      any = any || act[q];
    }
    if (!any) continue;
    const E *prow = srow[par][grow / kPanelRows];
    const E piv = prow[j];
    E inv;  // 1/pivot (LAPACK zgetf2 scales the column by the reciprocal)
    if (fabs((double)piv.y) <= fabs((double)piv.x)) {
      const Rl rr = piv.y / piv.x, id = (Rl)1 / (piv.x + piv.y * rr);
      inv = E{id, -rr * id};
    } else {
      const Rl rr = piv.x / piv.y, id = (Rl)1 / (piv.y + piv.x * rr);
      inv = E{rr * id, -id};
    }
    E l[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      l[q] = cmulE(v[q], inv);
      if (act[q]) R[j * kPanelRows + tid + q * T] = l[q];
    }
#pragma unroll 4
    for (int c = j + 1; c < w; ++c) {
      const E p = prow[c];
#pragma unroll
      for (int q = 0; q < RPT; ++q)
        if (act[q]) R[c * kPanelRows + tid + q * T] = csubE(R[c * kPanelRows + tid + q * T], cmulE(l[q], p));
    }
  }
#pragma unroll
  for (int q = 0; q < RPT; ++q) sdst[tid + q * T] = base + tid + q * T;
  __syncthreads();
  // Replay the interchanges (LAPACK semantics) by warp 0 of every CTA (each holds the same
  // chosen[]).  Only the w top rows can be displaced before they are chosen (a row leaves
  // position j only when step j swaps it out), and a chosen row stays at its pivot
  // position, so lane r < w keeps the position of original top row r and the original row
  // now at top position r; one step is two shuffles.
  if (warp == 0) {
    constexpr unsigned full = 0xffffffffu;
    int pos_top = lane, row_at = lane;
    const int ch = lane < w ? chosen[lane] : -1;
    for (int j = 0; j < w; ++j) {
      const int c = __shfl_sync(full, ch, j);  // original row chosen at step j, -1 = zero column
      const int pc = __shfl_sync(full, pos_top, c & 31);
      const int x = __shfl_sync(full, row_at, j);  // original row at position j (a top row)
      const int p = c < 0 ? j : (c < w ? pc : c);   // current position of row c
      if (c >= 0 && p != j) {  // row c -> position j, row x -> position p
        if (lane == j) row_at = c;
        if (lane == c) pos_top = j;
        if (lane == p) row_at = x;
        if (lane == x) pos_top = p;
      }
      if (crank == 0 && lane == 0) ipiv[col0 + j] = row0 + p;
    }
    // final positions of this CTA's moved rows: top rows and chosen rows below them
    if (lane < w && lane >= base && lane < base + nloc) sdst[lane - base] = pos_top;
    if (ch >= w && ch >= base && ch < base + nloc) sdst[ch - base] = lane;
    // interchange list for the other columns: dst = row0 + position, src = row0 + original row
    if (crank == 0) {
      const unsigned lt = (1u << lane) - 1u;
      const bool m1 = lane < w && row_at != lane;  // top position holding another row
      const bool m2 = lane < w && pos_top >= w;    // top row moved below the top rows
      const unsigned b1 = __ballot_sync(full, m1), b2 = __ballot_sync(full, m2);
      const int n1 = __popc(b1);
      if (m1) {
        const int i = __popc(b1 & lt);
        xlist[1 + i] = row0 + lane;
        xlist[1 + kMaxMov + i] = row0 + row_at;
      }
      if (m2) {
        const int i = n1 + __popc(b2 & lt);
        xlist[1 + i] = row0 + pos_top;
        xlist[1 + kMaxMov + i] = row0 + lane;
      }
      if (lane == 0) xlist[0] = n1 + __popc(b2);
    }
  }
  __syncthreads();
  // coalesced write-back: one row per warp step, one column per lane, to its final position
  for (int r0 = warp; r0 < nloc; r0 += NW * 8) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int r = r0 + u * NW;
      if (r < nloc && lane < w) M.put(row0 + sdst[r], col0 + lane, R[lane * kPanelRows + r]);
    }
  }
}

// Apply a panel's interchanges (its list: xlist[0] = m moves, dst rows xlist[1..m], source
// rows xlist[1+kMaxMov..]) to columns [0, ncol) except the panel's own [skip0, skip0 + w):
// every thread gathers its column's moved entries first and scatters them after.
template <bool F32>
__global__ void __launch_bounds__(kSwpThreads) k_laswp(Mat<F32> M0, long long ms, const int *__restrict__ xlist0,
                                                       int ncol, int skip0, int w) {
  using E = typename Prec<F32>::E;
  const Mat<F32> M = M0.at(blockIdx.y, ms);
  const int *xlist = xlist0 + blockIdx.y * kListInts;
  constexpr int MOV = F32 ? 2 * 32 : 2 * 16;  // 2 x panel width
  __shared__ int dst[MOV], src[MOV];
  __shared__ E stage[MOV][kSwpThreads];
  __shared__ int nm;
  if (threadIdx.x == 0) nm = min(xlist[0], MOV);
  for (int q = threadIdx.x; q < MOV; q += blockDim.x) {
    dst[q] = xlist[1 + q];
    src[q] = xlist[1 + kMaxMov + q];
  }
  __syncthreads();
  const int m = nm;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ncol - w) return;
  const int c = t < skip0 ? t : t + w;
  for (int q = 0; q < m; ++q) stage[q][threadIdx.x] = M.get(src[q], c);
  for (int q = 0; q < m; ++q) M.put(dst[q], c, stage[q][threadIdx.x]);
}

// Rows k0..k0+w-1 of columns [c0, c1): X = L11^{-1} X, L11 the w x w unit-lower block at
// (k0, k0) in shared memory; one column per thread, its w entries in shared memory too.
// Runtime loops keep the code small: each instruction of a fully unrolled triangle would
// run once per launch and miss the instruction cache.
template <bool F32, int W>
__global__ void __launch_bounds__(128) k_trsm_small(Mat<F32> M0, long long ms, int k0, int w, int c0, int c1) {
  using E = typename Prec<F32>::E;
  const Mat<F32> M = M0.at(blockIdx.y, ms);
  __shared__ E L[W][W];
  __shared__ E xs[W][128];
  for (int e = threadIdx.x; e < W * W; e += blockDim.x) {
    const int i = e / W, t = e % W;
    L[i][t] = (i < w && t < i) ? M.get(k0 + i, k0 + t) : E{0, 0};
  }
  const int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = c < c1;
  const int tx = threadIdx.x;
#pragma unroll 8
  for (int i = 0; i < w; ++i) xs[i][tx] = ok ? M.get(k0 + i, c) : E{0, 0};
  __syncthreads();
  for (int i = 1; i < w; ++i) {
    E v0 = xs[i][tx], v1{0, 0};  // two partial sums halve the dependency chain
    int t = 0;
    for (; t + 1 < i; t += 2) {
      v0 = csubE(v0, cmulE(L[i][t], xs[t][tx]));
      v1 = caddE(v1, cmulE(L[i][t + 1], xs[t + 1][tx]));
    }
    if (t < i) v0 = csubE(v0, cmulE(L[i][t], xs[t][tx]));
    xs[i][tx] = csubE(v0, v1);
  }
  if (ok) {
#pragma unroll 8
    for (int i = 0; i < w; ++i) M.put(k0 + i, c, xs[i][tx]);
  }
}

// C[r0:r1, c0:c1] -= A[r0:r1, k0:k0+kb] * A[k0:k0+kb, c0:c1]  (FP64 complex, SIMT, 64x64 tiles)
__global__ void __launch_bounds__(256) k_gemm64(cd *A0, long long ms, long long ld, int r0, int r1, int c0, int c1,
                                                int k0, int kb) {
  cd *A = A0 + blockIdx.z * ms;
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
__global__ void __launch_bounds__(256) k_gemm32(float *Ar0, float *Ai0, long long ms, long long ld, int r0, int r1,
                                                int c0, int c1, int k0, int kb) {
  float *Ar = Ar0 + blockIdx.z * ms, *Ai = Ai0 + blockIdx.z * ms;
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

// ------------------------------- host side -------------------------------
// Every launcher runs one step for all nb matrices of a batch (grid dimension = matrix).
template <bool F32>
int launch_panel(Mat<F32> M, const LuBatch &bt, int nb, int row0, int nrows, int col0, int w, cudaStream_t st) {
  const int cs = (nrows + kPanelRows - 1) / kPanelRows;
  const int Wt = F32 ? 32 : 16;
  if (cs > kMaxCluster || w > Wt) {
    pss_set_error("panel %d x %d exceeds a %d-CTA cluster", nrows, w, kMaxCluster);
    return -6;
  }
  auto kern = k_panel<F32, (F32 ? 32 : 16), kPanelRpt>;
  constexpr int smem = kPanelRows * (F32 ? 32 : 16) * (int)sizeof(typename Prec<F32>::E);  // the panel rows
  static DeviceOnce once;
  if (int rc = device_once(once, [&] {
        PSS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        PSS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        return 0;
      }))
    return rc;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cs * nb);  // one cluster of cs CTAs per matrix
  cfg.blockDim = dim3(kPanelRows / kPanelRpt);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cs;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  pss_count_launch();
  const int tok = pss_prof_begin(st);
  PSS_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, M, bt, row0, nrows, col0, w));
  // algorithmic bytes: every panel read once and written once
  pss_prof_end(tok, st, PSS_PROF_PANEL, 2.0 * nb * nrows * w * (F32 ? 8.0 : 16.0));
  return 0;
}

template <bool F32>
void launch_laswp(Mat<F32> M, const LuBatch &bt, int nb, int n, int k0, int w, cudaStream_t st) {
  if (n - w <= 0) return;
  pss_count_launch();
  k_laswp<F32><<<dim3(cdiv_u(n - w, kSwpThreads), nb), kSwpThreads, 0, st>>>(M, bt.ms, bt.xlist, n, k0, w);
}

template <bool F32>
void launch_trsm(Mat<F32> M, long long ms, int nb, int k0, int w, int c0, int c1, cudaStream_t st) {
  if (c1 <= c0) return;
  pss_count_launch();
  const dim3 grid(cdiv_u(c1 - c0, 128), nb);
  if constexpr (F32) {
    if (w <= 16) k_trsm_small<true, 16><<<grid, 128, 0, st>>>(M, ms, k0, w, c0, c1);
    else k_trsm_small<true, 32><<<grid, 128, 0, st>>>(M, ms, k0, w, c0, c1);
  } else {  // FP64 panels are at most 16 wide
    k_trsm_small<false, 16><<<grid, 128, 0, st>>>(M, ms, k0, w, c0, c1);
  }
}

void launch_gemm(Mat<false> M, long long ms, int nb, int r0, int r1, int c0, int c1, int k0, int kb,
                 cudaStream_t st) {
  if (r1 <= r0 || c1 <= c0) return;
  int tok = pss_prof_begin(st);
  pss_count_launch();
  k_gemm64<<<dim3(cdiv_u(c1 - c0, 64), cdiv_u(r1 - r0, 64), nb), 256, 0, st>>>((cd *)M.a, ms, M.ld, r0, r1, c0, c1,
                                                                              k0, kb);
  pss_prof_end(tok, st, PSS_PROF_SIMT_UPDATE, 8.0 * nb * (r1 - r0) * (double)(c1 - c0) * kb);
}
void launch_gemm(Mat<true> M, long long ms, int nb, int r0, int r1, int c0, int c1, int k0, int kb,
                 cudaStream_t st) {
  if (r1 <= r0 || c1 <= c0) return;
  int tok = pss_prof_begin(st);
  pss_count_launch();
  k_gemm32<<<dim3(cdiv_u(c1 - c0, 128), cdiv_u(r1 - r0, 128), nb), 256, 0, st>>>((float *)M.a, M.ai, ms, M.ld, r0,
                                                                                r1, c0, c1, k0, kb);
  pss_prof_end(tok, st, PSS_PROF_SIMT_UPDATE, 8.0 * nb * (r1 - r0) * (double)(c1 - c0) * kb);
}

// Tensor-core workspace of an FP32 factorisation (split operand planes); pipeline errors
// go to the matrices' info words (-1).
struct TcWs {
  void *ws = nullptr;
  size_t bytes = 0;
};

int launch_update(Mat<false> M, const LuBatch &bt, int nb, int r0, int r1, int c0, int c1, int k0, int kb,
                  const TcWs &, cudaStream_t st) {
  launch_gemm(M, bt.ms, nb, r0, r1, c0, c1, k0, kb, st);
  return 0;
}
// FP32: updates of at least kTcMinRows x kTcMinCols go to the tcgen05 kernel, smaller ones SIMT.
int launch_update(Mat<true> M, const LuBatch &bt, int nb, int r0, int r1, int c0, int c1, int k0, int kb,
                  const TcWs &tc, cudaStream_t st) {
  if (r1 - r0 >= kTcMinRows && c1 - c0 >= kTcMinCols && tc.ws)
    return pss_cgemm_tc((float *)M.a, M.ai, M.ld, bt.ms, nb, r0, r1 - r0, c0, c1 - c0, k0, kb, tc.ws, tc.bytes,
                        bt.info, st);
  launch_gemm(M, bt.ms, nb, r0, r1, c0, c1, k0, kb, st);
  return 0;
}

// Outer blocks of NB columns, inner panels of W columns (LAPACK dgetrf order):
//   1. each inner panel: factor, its interchanges on every other column, the W-row
//      triangular solve and Schur update restricted to the outer block's own columns;
//   2. once all interchanges of the outer block are applied, the block row of the
//      trailing columns, U12 = L11^{-1} A12, as W-row solves plus block-row updates;
//   3. the trailing matrix A22 -= L21 U12, one GEMM with K = NB.
// All nb matrices of the batch advance together, one launch per step.
template <bool F32>
int lu_blocked(int n, int nb, Mat<F32> M, const LuBatch &bt, int NB, int W, const TcWs &tc, cudaStream_t st) {
  int rc = 0;
  for (int K0 = 0; K0 < n; K0 += NB) {
    const int JB = min(NB, n - K0);
    const int E = K0 + JB;
    for (int k0 = K0; k0 < E; k0 += W) {
      const int w = min(W, E - k0);
      if ((rc = launch_panel<F32>(M, bt, nb, k0, n - k0, k0, w, st))) return rc;
      launch_laswp<F32>(M, bt, nb, n, k0, w, st);
      if (k0 + w < E) {
        launch_trsm<F32>(M, bt.ms, nb, k0, w, k0 + w, E, st);
        if ((rc = launch_update(M, bt, nb, k0 + w, n, k0 + w, E, k0, w, tc, st))) return rc;
      }
    }
    if (E < n) {
      for (int k0 = K0; k0 < E; k0 += W) {
        const int w = min(W, E - k0);
        launch_trsm<F32>(M, bt.ms, nb, k0, w, E, n, st);
        if (k0 + w < E && (rc = launch_update(M, bt, nb, k0 + w, E, E, n, k0, w, tc, st))) return rc;
      }
      if ((rc = launch_update(M, bt, nb, E, n, E, n, K0, JB, tc, st))) return rc;
    }
  }
  PSS_CUDA_TRY(cudaGetLastError());
  return 0;
}

template <bool F32>
int pick_panel_width(int n, int want) {
  if ((n + kPanelRows - 1) / kPanelRows > kMaxCluster) return -1;
  return want;
}

constexpr int kNB64 = 64, kNB32 = 128;
size_t list_bytes(int nb) { return ((size_t)nb * kListInts * sizeof(int) + 255) & ~(size_t)255; }
}  // namespace

// Workspace of a batch of nb factorisations: the panels' interchange lists (kListInts ints
// per matrix), then for the FP32 factorisation the split operand planes of one batched
// tensor-core update.
size_t pss_lu_ws_bytes(int n, int precision, int nb) {
  return list_bytes(nb) + (precision == 0 ? 0 : pss_tc_ws_bytes(n, n, kNB32, nb));
}

int pss_lu64_batched(int n, int nb, cd *A, long long ld, long long ms, int *ipiv, int *info, void *ws,
                     size_t ws_bytes, cudaStream_t st) {
  if (nb <= 0) return 0;
  if (ws_bytes < pss_lu_ws_bytes(n, 0, nb)) { pss_set_error("LU workspace too small"); return -4; }
  Mat<false> M{A, nullptr, ld};
  int W = pick_panel_width<false>(n, 16);
  if (W < 0) { pss_set_error("matrix order %d too large for the cluster panel", n); return -6; }
  const LuBatch bt{ms, n, ipiv, info, (int *)ws};
  return lu_blocked<false>(n, nb, M, bt, kNB64, W, TcWs{}, st);
}

int pss_lu32_batched(int n, int nb, float *Ar, float *Ai, long long ld, long long ms, int *ipiv, int *info,
                     void *ws, size_t ws_bytes, cudaStream_t st, int panel_w, int outer_nb) {
  if (nb <= 0) return 0;
  if (ws_bytes < pss_lu_ws_bytes(n, 1, nb)) { pss_set_error("LU workspace too small"); return -4; }
  if (panel_w == 0) panel_w = 32;
  if (outer_nb == 0) outer_nb = kNB32;
  if ((panel_w != 8 && panel_w != 16 && panel_w != 32) || (outer_nb != 64 && outer_nb != 128) ||
      outer_nb % panel_w) {
    pss_set_error("FP32 LU tile shape (panel %d, outer block %d) not one of panel 8/16/32, outer 64/128",
                  panel_w, outer_nb);
    return -1;
  }
  Mat<true> M{Ar, Ai, ld};
  int W = pick_panel_width<true>(n, panel_w);
  if (W < 0) { pss_set_error("matrix order %d too large for the cluster panel", n); return -6; }
  const size_t lb = list_bytes(nb);
  const LuBatch bt{ms, n, ipiv, info, (int *)ws};
  return lu_blocked<true>(n, nb, M, bt, outer_nb, W, TcWs{(char *)ws + lb, ws_bytes - lb}, st);
}

int pss_lu64(int n, cd *A, long long ld, int *ipiv, int *info, void *ws, size_t ws_bytes, cudaStream_t st) {
  return pss_lu64_batched(n, 1, A, ld, 0, ipiv, info, ws, ws_bytes, st);
}

int pss_lu32(int n, float *Ar, float *Ai, long long ld, int *ipiv, int *info, void *ws, size_t ws_bytes,
             cudaStream_t st) {
  return pss_lu32_batched(n, 1, Ar, Ai, ld, 0, ipiv, info, ws, ws_bytes, st, 0, 0);
}
