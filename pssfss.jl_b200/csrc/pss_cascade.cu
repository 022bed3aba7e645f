// GSM cascade of many frequency points on the device: the Gblock walk of _analyze
// (src/PSSFSS.jl:256-305) with cascade (the Redheffer star product of Eq. 3.35,
// src/GSMs.jl:125-141) and cascade! (propagation through a layer, src/GSMs.jl:154-176).
//
// One CTA per point.  The running GSM A and the new one live in a per-point global scratch
// (L2-resident: at most 64 modes per region, 64 x 64 complex blocks); the two linear systems
// of each star product, (I - A22 B11) G1 = A21 and (I - B11 A22) G2 = B12, are solved in
// shared memory by Gauss-Jordan elimination with partial pivoting (the largest |re| + |im| in
// the column, the first one on ties, as LAPACK's zgesv chooses); the small products run one
// output entry per thread with the sum in a fixed order.
#include <vector>

#include "pss_internal.cuh"

namespace {

constexpr int kCascadeMaxModes = 64;
constexpr int kCascadeThreads = 256;

__device__ __forceinline__ double cabs1d(cd z) { return fabs(z.x) + fabs(z.y); }

// C (r x c) = A (r x k) * B (k x c), plus Cin when given (column-major, leading dimension =
// rows); one output entry per thread, the sum over k in order.
__device__ void cmm(int r, int c, int k, const cd *A, const cd *B, const cd *Cin, cd *C) {
  for (int e = threadIdx.x; e < r * c; e += blockDim.x) {
    const int i = e % r, j = e / r;
    cd s = mkcd(0, 0);
    for (int t = 0; t < k; ++t) s = s + A[i + t * r] * B[t + j * k];
    C[e] = Cin ? Cin[e] + s : s;
  }
  __syncthreads();
}

// X (m x nr) = M^-1 R by Gauss-Jordan elimination with partial pivoting, M given as
// I - P Q with P (m x m) and Q (m x m) from global memory; R (m x nr) from global memory.
// Shared memory: M [m][m] and R [m][nr], column-major.  Returns the solution in X (global).
__device__ void gj_solve_ipq(int m, int nr, const cd *P, const cd *Q, const cd *R, cd *X, cd *sM, cd *sR,
                             int *spiv, int *sing) {
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
    const int i = e % m, j = e / m;
    cd s = mkcd(0, 0);
    for (int t = 0; t < m; ++t) s = s + P[i + t * m] * Q[t + j * m];
    sM[e] = mkcd(i == j ? 1.0 : 0.0, 0.0) - s;
  }
  for (int e = threadIdx.x; e < m * nr; e += blockDim.x) sR[e] = R[e];
  __syncthreads();
  for (int j = 0; j < m; ++j) {
    if (threadIdx.x == 0) {  // pivot: largest |re| + |im| at or below the diagonal, first on ties
      int p = j;
      double best = cabs1d(sM[j + j * m]);
      for (int r = j + 1; r < m; ++r) {
        const double v = cabs1d(sM[r + j * m]);
        if (v > best) { best = v; p = r; }
      }
      *spiv = p;
      if (best == 0.0) *sing = 1;
    }
    __syncthreads();
    const int p = *spiv;
    if (p != j) {  // swap rows j and p of M (columns j..m-1) and R
      for (int c = threadIdx.x; c < m + nr; c += blockDim.x) {
        if (c < m) {
          if (c >= j) { const cd t = sM[j + c * m]; sM[j + c * m] = sM[p + c * m]; sM[p + c * m] = t; }
        } else {
          const int cc = c - m;
          const cd t = sR[j + cc * m]; sR[j + cc * m] = sR[p + cc * m]; sR[p + cc * m] = t;
        }
      }
      __syncthreads();
    }
    const cd piv = sM[j + j * m];
    const cd inv = (cabs1d(piv) > 0.0) ? mkcd(1.0, 0.0) / piv : mkcd(0.0, 0.0);
    __syncthreads();
    // scale row j (columns j+1.. of M, all of R); M[j][j] = 1
    for (int c = threadIdx.x; c < m + nr; c += blockDim.x) {
      if (c < m) { if (c > j) sM[j + c * m] = sM[j + c * m] * inv; }
      else sR[j + (c - m) * m] = sR[j + (c - m) * m] * inv;
    }
    __syncthreads();
    // eliminate column j from every other row: row_r -= M[r][j] * row_j
    for (int e = threadIdx.x; e < m * (m + nr); e += blockDim.x) {
      const int r = e % m, c = e / m;
      if (r == j) continue;
      const cd f = sM[r + j * m];
      if (c < m) { if (c > j) sM[r + c * m] = sM[r + c * m] - f * sM[j + c * m]; }
      else sR[r + (c - m) * m] = sR[r + (c - m) * m] - f * sR[j + (c - m) * m];
    }
    __syncthreads();
    for (int r = threadIdx.x; r < m; r += blockDim.x)
      if (r != j) sM[r + j * m] = mkcd(0, 0);
    __syncthreads();
  }
  for (int e = threadIdx.x; e < m * nr; e += blockDim.x) X[e] = sR[e];
  __syncthreads();
}

struct CascadeArgs {
  int npts, nblk;
  const int *dims;        // nblk + 1 mode counts
  const long long *goff;  // nblk + 1: offset (complex entries) of block k inside a point's GSM record; goff[nblk] = record size
  long long poff_total;   // complex entries of a point's propagation record
  const cd *gsm, *prop;
  cd *out, *scratch;
  long long scratch_per_point;
  int *sing;              // per point: a singular star-product system met
};

__global__ void __launch_bounds__(kCascadeThreads) k_cascade(CascadeArgs a) {
  extern __shared__ __align__(16) unsigned char csm[];
  const int pt = blockIdx.x;
  const int D = kCascadeMaxModes;
  cd *sM = (cd *)csm, *sR = sM + D * D;
  __shared__ int spiv, ssing;
  if (threadIdx.x == 0) ssing = 0;
  cd *w = a.scratch + (size_t)pt * a.scratch_per_point;
  cd *A11 = w, *A12 = A11 + D * D, *A21 = A12 + D * D, *A22 = A21 + D * D;
  cd *N11 = A22 + D * D, *N12 = N11 + D * D, *N21 = N12 + D * D, *N22 = N21 + D * D;
  cd *G = N22 + D * D, *T = G + D * D;
  const cd *prop = a.prop + (size_t)pt * a.poff_total;
  const cd *rec = a.gsm + (size_t)pt * a.goff[a.nblk];
  const int n0 = a.dims[0];
  // identity GSM of region 0 propagated through layer 0: s12 = s21 = diag(p0), s11 = s22 = 0
  for (int e = threadIdx.x; e < n0 * n0; e += blockDim.x) {
    const int i = e % n0, j = e / n0;
    A11[e] = mkcd(0, 0);
    A22[e] = mkcd(0, 0);
    A12[e] = i == j ? prop[i] : mkcd(0, 0);
    A21[e] = i == j ? prop[i] : mkcd(0, 0);
  }
  __syncthreads();
  int poff = n0;
  for (int k = 0; k < a.nblk; ++k) {
    const int m = a.dims[k], n2 = a.dims[k + 1];
    const cd *B = rec + a.goff[k];
    const cd *B11 = B, *B12 = B11 + m * m, *B21 = B12 + m * n2, *B22 = B21 + n2 * m;
    // G1 = (I - A22 B11)^-1 A21  (m x n0)
    gj_solve_ipq(m, n0, A22, B11, A21, G, sM, sR, &spiv, &ssing);
    cmm(n2, n0, m, B21, G, nullptr, N21);   // s21 = B21 G1
    cmm(m, n0, m, B11, G, nullptr, T);      // T = B11 G1
    cmm(n0, n0, m, A12, T, A11, N11);       // s11 = A11 + A12 T
    // G2 = (I - B11 A22)^-1 B12  (m x n2)
    gj_solve_ipq(m, n2, B11, A22, B12, G, sM, sR, &spiv, &ssing);
    cmm(n0, n2, m, A12, G, nullptr, N12);   // s12 = A12 G2
    cmm(m, n2, m, A22, G, nullptr, T);      // T = A22 G2
    cmm(n2, n2, m, B21, T, B22, N22);       // s22 = B22 + B21 T
    // propagation of the region-2 ports through the layer behind the block
    const cd *p = prop + poff;
    for (int e = threadIdx.x; e < n0 * n2; e += blockDim.x) A12[e] = N12[e] * p[e / n0];
    for (int e = threadIdx.x; e < n2 * n0; e += blockDim.x) {
      const int i = e % n2;
      A21[e] = N21[e] * p[i];
    }
    for (int e = threadIdx.x; e < n2 * n2; e += blockDim.x) {
      const int i = e % n2, j = e / n2;
      A22[e] = (N22[e] * p[i]) * p[j];
    }
    for (int e = threadIdx.x; e < n0 * n0; e += blockDim.x) A11[e] = N11[e];
    __syncthreads();
    poff += n2;
  }
  const int nK = a.dims[a.nblk];
  cd *o = a.out + (size_t)pt * ((size_t)n0 * n0 + 2 * (size_t)n0 * nK + (size_t)nK * nK);
  for (int e = threadIdx.x; e < n0 * n0; e += blockDim.x) o[e] = A11[e];
  o += n0 * n0;
  for (int e = threadIdx.x; e < n0 * nK; e += blockDim.x) o[e] = A12[e];
  o += n0 * nK;
  for (int e = threadIdx.x; e < nK * n0; e += blockDim.x) o[e] = A21[e];
  o += nK * n0;
  for (int e = threadIdx.x; e < nK * nK; e += blockDim.x) o[e] = A22[e];
  if (threadIdx.x == 0) a.sing[pt] = ssing;
}

struct ScopedDev {
  void *p = nullptr;
  ~ScopedDev() {
    if (p) cudaFree(p);
  }
};

}  // namespace

extern "C" int pss_cascade(pss_ctx *ctx, int npts, int nblk, const int *dims, const double *gsm, const double *prop,
                           double *out, int *status) {
  if (!ctx || !dims || !gsm || !prop || !out || !status || npts <= 0 || nblk <= 0 || nblk > 256) {
    pss_set_error("invalid argument");
    return -1;
  }
  for (int k = 0; k <= nblk; ++k)
    if (dims[k] < 1 || dims[k] > kCascadeMaxModes) {
      pss_set_error("mode count %d of region %d outside 1..%d", dims[k], k, kCascadeMaxModes);
      return -1;
    }
  int dev = 0;
  if (pss_ctx_device(ctx, &dev)) return -1;
  PSS_CUDA_TRY(cudaSetDevice(dev));
  std::vector<long long> goff(nblk + 1, 0);
  long long ptot = dims[0];
  for (int k = 0; k < nblk; ++k) {
    const long long m = dims[k], n2 = dims[k + 1];
    goff[k + 1] = goff[k] + m * m + 2 * m * n2 + n2 * n2;
    ptot += n2;
  }
  const int n0 = dims[0], nK = dims[nblk];
  const size_t out_per = (size_t)n0 * n0 + 2 * (size_t)n0 * nK + (size_t)nK * nK;
  const long long spp = 10LL * kCascadeMaxModes * kCascadeMaxModes;
  const size_t b_gsm = (size_t)npts * goff[nblk] * sizeof(cd), b_prop = (size_t)npts * ptot * sizeof(cd);
  const size_t b_out = (size_t)npts * out_per * sizeof(cd), b_scr = (size_t)npts * spp * sizeof(cd);
  ScopedDev dg, dp, dout, dscr, dgo, ddims, dsing;
  PSS_CUDA_TRY(cudaMalloc(&dg.p, b_gsm));
  PSS_CUDA_TRY(cudaMalloc(&dp.p, b_prop));
  PSS_CUDA_TRY(cudaMalloc(&dout.p, b_out));
  PSS_CUDA_TRY(cudaMalloc(&dscr.p, b_scr));
  PSS_CUDA_TRY(cudaMalloc(&dgo.p, (nblk + 1) * sizeof(long long)));
  PSS_CUDA_TRY(cudaMalloc(&ddims.p, (nblk + 1) * sizeof(int)));
  PSS_CUDA_TRY(cudaMalloc(&dsing.p, npts * sizeof(int)));
  PSS_CUDA_TRY(cudaMemcpy(dg.p, gsm, b_gsm, cudaMemcpyHostToDevice));
  PSS_CUDA_TRY(cudaMemcpy(dp.p, prop, b_prop, cudaMemcpyHostToDevice));
  PSS_CUDA_TRY(cudaMemcpy(dgo.p, goff.data(), (nblk + 1) * sizeof(long long), cudaMemcpyHostToDevice));
  PSS_CUDA_TRY(cudaMemcpy(ddims.p, dims, (nblk + 1) * sizeof(int), cudaMemcpyHostToDevice));
  const int smem = 2 * kCascadeMaxModes * kCascadeMaxModes * (int)sizeof(cd);
  static DeviceOnce once;
  if (int rc = device_once(once, [&] {
        PSS_CUDA_TRY(cudaFuncSetAttribute(k_cascade, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        return 0;
      }))
    return rc;
  CascadeArgs a{npts, nblk, (const int *)ddims.p, (const long long *)dgo.p, ptot, (const cd *)dg.p,
                (const cd *)dp.p, (cd *)dout.p, (cd *)dscr.p, spp, (int *)dsing.p};
  pss_count_launch();
  k_cascade<<<npts, kCascadeThreads, smem>>>(a);
  PSS_CUDA_TRY(cudaGetLastError());
  PSS_CUDA_TRY(cudaMemcpy(out, dout.p, b_out, cudaMemcpyDeviceToHost));
  std::vector<int> hs(npts);
  PSS_CUDA_TRY(cudaMemcpy(hs.data(), dsing.p, npts * sizeof(int), cudaMemcpyDeviceToHost));
  for (int i = 0; i < npts; ++i) status[i] = hs[i] ? PSS_STATUS_SINGULAR : 0;
  return 0;
}
