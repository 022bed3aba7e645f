// K1: spectral modal tables of the layered periodic Green's function.
//
// Restates PGF.jl:196-365 (electric_modal_sum_funcs) and PGF.jl:478-629
// (magnetic_modal_sum_funcs) for sm_100a:
//   * every (m,n) summand of rings 0..R is computed by its own thread (the layer
//     impedance/admittance recursion of Eqs. 5.14 / 5.24, FP64);
//   * each ring's sum is reduced by one CTA in a fixed tree order, giving the
//     convergence flags of PGF.jl:285-288;
//   * one thread per point replays the reference's adaptive mmax sequence
//     (0, then the next even 2·3·5-smooth number, until 40 consecutive rings pass)
//     on those flags, so the chosen mmax is the reference's;
//   * the mmax x mmax 2-D DFT (FFTW's fft! in the reference) is a Stockham
//     mixed-radix 2/3/5 FFT, one CTA per line in shared memory;
//   * the Eq. 5.32 phase, the 1/(2A) (or 1/A) factor and the periodic padding of
//     PGF.jl:316-357 / 593-621 are one elementwise kernel.
#include "pss_internal.cuh"

namespace {


__device__ __forceinline__ void stack_summands(const StackParams &S, const PointParams &P,
                                               double bsq, double ksq, double kap, cd &v1, cd &v2) {
  const int nl = S.nl, s = S.s;
  const bool mag = P.magnetic;
  const double k0sq = P.k0sq;
  cd g = mysqrtd(rsubc(bsq, (k0sq * S.eps[0]) * S.mu[0]));
  cd LTE, LTM, RTE, RTM;
  if (!mag) { LTE = S.mu[0] / g; LTM = g / S.eps[0]; }
  else { LTE = g / S.mu[0]; LTM = S.eps[0] / g; }
  for (int i = 2; i <= s; ++i) {
    cd gi = mysqrtd(rsubc(bsq, (k0sq * S.eps[i - 1]) * S.mu[i - 1]));
    cd Z0TE, Z0TM;
    if (!mag) { Z0TE = S.mu[i - 1] / gi; Z0TM = gi / S.eps[i - 1]; }
    else { Z0TE = gi / S.mu[i - 1]; Z0TM = S.eps[i - 1] / gi; }
    cd th = ctanhd(S.width[i - 1] * gi);
    LTE = (Z0TE * (LTE + Z0TE * th)) / (Z0TE + LTE * th);
    LTM = (Z0TM * (LTM + Z0TM * th)) / (Z0TM + LTM * th);
  }
  g = mysqrtd(rsubc(bsq, (k0sq * S.eps[nl - 1]) * S.mu[nl - 1]));
  if (!mag) { RTE = S.mu[nl - 1] / g; RTM = g / S.eps[nl - 1]; }
  else { RTE = g / S.mu[nl - 1]; RTM = S.eps[nl - 1] / g; }
  for (int i = nl - 1; i >= s + 1; --i) {
    cd gi = mysqrtd(rsubc(bsq, (k0sq * S.eps[i - 1]) * S.mu[i - 1]));
    cd Z0TE, Z0TM;
    if (!mag) { Z0TE = S.mu[i - 1] / gi; Z0TM = gi / S.eps[i - 1]; }
    else { Z0TE = gi / S.mu[i - 1]; Z0TM = S.eps[i - 1] / gi; }
    cd th = ctanhd(S.width[i - 1] * gi);
    RTE = (Z0TE * (RTE + Z0TE * th)) / (Z0TE + RTE * th);
    RTM = (Z0TM * (RTM + Z0TM * th)) / (Z0TM + RTM * th);
  }
  if (!mag) {
    cd ViTE = (LTE * RTE) / (LTE + RTE);
    cd ViTM = (LTM * RTM) / (LTM + RTM);
    ViTE = (2.0 * ViTE) / P.mutilde;
    v1 = ViTE - (mkcd(1.0, 0.0) + P.c3 / ksq) / kap;
    ViTM = (2.0 * P.epsbar) * ViTM;
    cd kk = ((k0sq * P.epsbar) * P.mutilde) * ViTE;
    v2 = (ViTM + kk) / bsq - (mkcd(1.0, 0.0) + P.d3 / ksq) / kap;
  } else {
    cd ytm = LTM + RTM;
    v1 = ytm - (P.f1 + P.f3 / ksq) / kap;
    cd num = (k0sq * ytm + LTE) + RTE;
    v2 = num / bsq - (P.p1 + P.p3 / ksq) / kap;
  }
}

// One thread per lattice point (m,n) with rlo <= max(|m|,|n|) <= rhi; dense (2R+1)^2 tables.
__global__ void k_ring_fill(StackParams S, const PointParams *__restrict__ Pv, int R, int rlo, int rhi,
                            cd *__restrict__ dense, size_t point_stride) {
  const int W = 2 * R + 1;
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)W * W) return;
  const int pt = blockIdx.y;
  const PointParams &P = Pv[pt];
  int m = (int)(t % W) - R, n = (int)(t / W) - R;
  int r = max(abs(m), abs(n));
  if (r < rlo || r > rhi) return;
  double bx = (P.b00[0] + (double)m * P.b1[0]) + (double)n * P.b2[0];
  double by = (P.b00[1] + (double)m * P.b1[1]) + (double)n * P.b2[1];
  double bsq = bx * bx + by * by;
  bsq = fmax(bsq, P.b2min);
  double ksq = bsq + P.u * P.u;
  double kap = sqrt(ksq);
  cd v1, v2;
  stack_summands(S, P, bsq, ksq, kap, v1, v2);
  cd *d1 = dense + pt * point_stride;
  cd *d2 = d1 + (size_t)W * W;
  d1[t] = v1;
  d2[t] = v2;
}

// One CTA per (ring, point): ring sum in a fixed tree order, convergence flag.
__global__ void k_ring_sums(const PointParams *__restrict__ Pv, int R, int rlo, const cd *__restrict__ dense,
                            size_t point_stride, double convtest, unsigned char *__restrict__ conv) {
  const int W = 2 * R + 1;
  const int r = rlo + blockIdx.x;
  const int pt = blockIdx.y;
  const cd *d1 = dense + pt * point_stride;
  const cd *d2 = d1 + (size_t)W * W;
  __shared__ cd s1[256], s2[256];
  cd a1 = mkcd(0, 0), a2 = mkcd(0, 0);
  const int len = ring_len(r);
  for (int i = threadIdx.x; i < len; i += blockDim.x) {
    int m, n;
    ring_mn(r, i, m, n);
    size_t idx = (size_t)(m + R) + (size_t)(n + R) * W;
    a1 = a1 + d1[idx];
    a2 = a2 + d2[idx];
  }
  s1[threadIdx.x] = a1;
  s2[threadIdx.x] = a2;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s1[threadIdx.x] = s1[threadIdx.x] + s1[threadIdx.x + w];
      s2[threadIdx.x] = s2[threadIdx.x] + s2[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    size_t c0 = (size_t)R + (size_t)R * W;
    double t1 = cabsd(s1[0] / d1[c0]);
    double t2 = cabsd(s2[0] / d2[c0]);
    conv[(size_t)pt * (R + 1) + r] = (t1 < convtest) && (t2 < convtest);
  }
  (void)Pv;
}

__device__ int next_even_235(int x) {
  for (;;) {
    int v = x + 1;
    for (;; ++v) {
      int t = v;
      while (t % 2 == 0) t /= 2;
      while (t % 3 == 0) t /= 3;
      while (t % 5 == 0) t /= 5;
      if (t == 1) break;
    }
    x = v;
    if (x % 2 == 0) return x;
  }
}

// Replays the mmax sequence of PGF.jl:223-298 on the ring flags.  out[pt] = mmax,
// flag[pt]: 0 converged, 1 cap reached, 2 needs rings beyond R.
__global__ void k_find_mmax(int npts, int R, const unsigned char *__restrict__ conv, int *out, int *flag) {
  int pt = blockIdx.x * blockDim.x + threadIdx.x;
  if (pt >= npts) return;
  const unsigned char *c = conv + (size_t)pt * (R + 1);
  int mmax = 0;
  for (;;) {
    int mo2 = mmax / 2;
    if (mo2 > R) { out[pt] = mmax; flag[pt] = 2; return; }
    if (mo2 >= PSS_CONVREPEAT) {
      bool all = true;
      for (int r = mo2 - PSS_CONVREPEAT + 1; r <= mo2; ++r) all = all && c[r];
      if (all) { out[pt] = mmax; flag[pt] = 0; return; }
    }
    if (mmax >= PSS_MMAX_CAP) { out[pt] = mmax; flag[pt] = 1; return; }
    mmax = next_even_235(mmax);
  }
}

// FFT input: a[p + q*mmax] = table[p - mo2, q - mo2] (PGF.jl:311-312).
__global__ void k_fft_gather(const cd *__restrict__ dense, int R, int mmax, cd *__restrict__ a1,
                             cd *__restrict__ a2) {
  const int W = 2 * R + 1;
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)mmax * mmax) return;
  int p = (int)(t % mmax), q = (int)(t / mmax);
  int mo2 = mmax / 2;
  size_t idx = (size_t)(p - mo2 + R) + (size_t)(q - mo2 + R) * W;
  a1[t] = dense[idx];
  a2[t] = dense[idx + (size_t)W * W];
}

__device__ __forceinline__ void dft_small(cd *v, int R) {
  if (R == 2) {
    cd a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
  } else if (R == 4) {
    cd t0 = v[0] + v[2], t1 = v[0] - v[2], t2 = v[1] + v[3], t3 = v[1] - v[3];
    cd mjt3 = mkcd(t3.y, -t3.x);  // -i*t3
    v[0] = t0 + t2;
    v[2] = t0 - t2;
    v[1] = t1 + mjt3;
    v[3] = t1 - mjt3;
  } else if (R == 3) {
    const double c1 = -0.5, s1 = 0.86602540378443864676;
    cd a = v[0], b = v[1], c = v[2];
    cd t = b + c;
    cd d = b - c;
    v[0] = a + t;
    cd m = a + c1 * t;
    cd js = mkcd(s1 * d.y, -s1 * d.x);  // -i*s1*d
    v[1] = m + js;
    v[2] = m - js;
  } else {  // R == 5
    const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
    const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
    cd a = v[0];
    cd b1 = v[1] + v[4], d1 = v[1] - v[4];
    cd b2 = v[2] + v[3], d2 = v[2] - v[3];
    v[0] = a + b1 + b2;
    cd m1 = a + c1 * b1 + c2 * b2;
    cd m2 = a + c2 * b1 + c1 * b2;
    cd e1 = s1 * d1 + s2 * d2;  // multiplied by -i below
    cd e2 = s2 * d1 - s1 * d2;
    cd je1 = mkcd(e1.y, -e1.x), je2 = mkcd(e2.y, -e2.x);
    v[1] = m1 + je1;
    v[4] = m1 - je1;
    v[2] = m2 + je2;
    v[3] = m2 - je2;
  }
}

struct Radices {
  int nf;
  int r[16];
};

// Forward DFT of one line per CTA (line l at base + l*line_stride, element stride es).
__global__ void k_fft_lines(cd *__restrict__ data, int n, long long line_stride, long long es, Radices rad) {
  extern __shared__ cd sm[];
  cd *A = sm, *B = sm + n;
  cd *line = data + (long long)blockIdx.x * line_stride;
  for (int i = threadIdx.x; i < n; i += blockDim.x) A[i] = line[(long long)i * es];
  __syncthreads();
  int Ns = 1;
  cd *src = A, *dst = B;
  for (int st = 0; st < rad.nf; ++st) {
    const int R = rad.r[st];
    const int nR = n / R;
    for (int j = threadIdx.x; j < nR; j += blockDim.x) {
      cd v[5];
      int jm = j % Ns;
      for (int r = 0; r < R; ++r) {
        cd x = src[j + r * nR];
        long long e = (long long)jm * r;
        if (e != 0) {
          double s, c;
          sincospi(-2.0 * (double)e / (double)(Ns * R), &s, &c);
          x = x * mkcd(c, s);
        }
        v[r] = x;
      }
      dft_small(v, R);
      int idxD = (j / Ns) * Ns * R + jm;
      for (int r = 0; r < R; ++r) dst[idxD + r * Ns] = v[r];
    }
    __syncthreads();
    cd *t = src; src = dst; dst = t;
    Ns *= R;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) line[(long long)i * es] = src[i];
}

__device__ __forceinline__ cd pad_value(const cd *__restrict__ A, int mmax, const PointParams &P, double scale,
                                        int a, int b) {
  // Interior value with the Eq. 5.32 phase and area factor.
  auto interior = [&](int p, int q) -> cd {
    double qterm = q * (PSS_PI - P.psi2 / mmax);
    double pterm = p * (PSS_PI - P.psi1 / mmax);
    cd cf = cisd(pterm + qterm) / scale;
    return A[(size_t)p + (size_t)q * mmax] * cf;
  };
  const bool mag = P.magnetic;
  cd c1 = cisd(-P.psi1), c2 = cisd(-P.psi2);
  auto ext = [&](int p, int q) -> cd {  // p,q in 0..mmax
    if (p < mmax && q < mmax) return interior(p, q);
    if (p == mmax && q < mmax) return c1 * interior(0, q);
    if (p < mmax && q == mmax) return c2 * interior(p, 0);
    cd c12 = mag ? cisd(-(P.psi1 + P.psi2)) : c1 * c2;
    return c12 * interior(0, 0);
  };
  cd ic1 = mag ? cisd(P.psi1) : mkcd(1.0, 0.0) / c1;
  cd ic2 = mag ? cisd(P.psi2) : mkcd(1.0, 0.0) / c2;
  if (a >= 0 && b >= 0) return ext(a, b);
  if (a == -1 && b >= 0) return ic1 * ext(mmax - 1, b);
  // b == -1, a in -1..mmax-1
  if (a >= 0) return ic2 * ext(a, mmax - 1);
  return ic2 * (ic1 * ext(mmax - 1, mmax - 1));
}

__global__ void k_phase_pad(const cd *__restrict__ a1, const cd *__restrict__ a2, int mmax,
                            const PointParams *__restrict__ Pp, cd *__restrict__ t1, cd *__restrict__ t2) {
  const int L = mmax + 2;
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)L * L) return;
  int a = (int)(t % L) - 1, b = (int)(t / L) - 1;
  if (a == mmax && b == -1) { t1[t] = mkcd(0, 0); t2[t] = mkcd(0, 0); return; }  // unused corner
  const PointParams &P = *Pp;
  double scale = P.magnetic ? P.area : 2.0 * P.area;
  t1[t] = pad_value(a1, mmax, P, scale, a, b);
  t2[t] = pad_value(a2, mmax, P, scale, a, b);
}

// Radix sequence for n = 2^a 3^b 5^c: radix-4 stages first, then 5, 3 and a last 2.
int factor235(int n, Radices &rad) {
  int k = 0;
  while (n % 4 == 0 && k < 16) { rad.r[k++] = 4; n /= 4; }
  while (n % 5 == 0 && k < 16) { rad.r[k++] = 5; n /= 5; }
  while (n % 3 == 0 && k < 16) { rad.r[k++] = 3; n /= 3; }
  while (n % 2 == 0 && k < 16) { rad.r[k++] = 2; n /= 2; }
  rad.nf = k;
  return n == 1 ? k : -1;
}

int fft2d(cd *a, int n, cudaStream_t st) {
  if (n <= 1) return 0;
  Radices rad;
  if (n > PSS_MMAX_CAP || factor235(n, rad) < 0) { pss_set_error("fft size %d not supported", n); return -2; }
  size_t smem = 2 * (size_t)n * sizeof(cd);
  int thr = 256;
  // columns: contiguous lines; rows: stride n
  pss_count_launch();
  k_fft_lines<<<n, thr, smem, st>>>(a, n, n, 1, rad);
  pss_count_launch();
  k_fft_lines<<<n, thr, smem, st>>>(a, n, 1, n, rad);
  return 0;
}

}  // namespace

// ---- host launchers (orchestrated by pss_api.cu) ----

void pss_tables_ring_fill(const StackParams &S, const PointParams *dP, int npts, int R, cd *dense,
                          size_t point_stride, cudaStream_t st) {
  long long W = 2LL * R + 1;
  pss_count_launch();
  k_ring_fill<<<dim3(cdiv_u(W * W, 256), npts), 256, 0, st>>>(S, dP, R, 0, R, dense, point_stride);
}

void pss_tables_ring_sums(const PointParams *dP, int npts, int R, const cd *dense, size_t point_stride,
                          double convtest, unsigned char *conv, cudaStream_t st) {
  pss_count_launch();
  k_ring_sums<<<dim3(R + 1, npts), 256, 0, st>>>(dP, R, 0, dense, point_stride, convtest, conv);
}

void pss_tables_find_mmax(int npts, int R, const unsigned char *conv, int *mmax, int *flag, cudaStream_t st) {
  pss_count_launch();
  k_find_mmax<<<cdiv_u(npts, 64), 64, 0, st>>>(npts, R, conv, mmax, flag);
}

// dense: this point's (2R+1)^2 x 2 tables; stage: >= 2*mmax^2 entries; t1/t2: (mmax+2)^2 each.
int pss_tables_finish(const cd *dense, int R, int mmax, const PointParams *dP1, cd *stage, cd *t1, cd *t2,
                      cudaStream_t st) {
  static DeviceOnce once;
  if (int rc = device_once(once, [] {
        PSS_CUDA_TRY(cudaFuncSetAttribute(k_fft_lines, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          2 * PSS_MMAX_CAP * (int)sizeof(cd)));
        return 0;
      }))
    return rc;
  long long nn = (long long)mmax * mmax;
  cd *a1 = stage, *a2 = stage + nn;
  if (nn > 0) {
    pss_count_launch();
    k_fft_gather<<<cdiv_u(nn, 256), 256, 0, st>>>(dense, R, mmax, a1, a2);
    int rc = fft2d(a1, mmax, st);
    if (rc) return rc;
    rc = fft2d(a2, mmax, st);
    if (rc) return rc;
  }
  long long L2 = (long long)(mmax + 2) * (mmax + 2);
  pss_count_launch();
  k_phase_pad<<<cdiv_u(L2, 256), 256, 0, st>>>(a1, a2, mmax, dP1, t1, t2);
  PSS_CUDA_TRY(cudaGetLastError());
  return 0;
}
