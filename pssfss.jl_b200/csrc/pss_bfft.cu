// K6: basis-function Fourier transforms, right-hand sides and modal projection.
//
// k_bfft restates RWG.jl:428-512 (rwgbfft!, McInturff-Simon transform of the modified
// RWG functions) as a gather: one thread per (basis function, mode) sums the
// contributions of that function's face incidences in a fixed order.  k_rhs forms
// v[n, j] = conj(F_j[n])·src_j (PSSFSS.jl:436, Eq. 7.39 / 7.64) and k_project the
// scattered partial GSM  dS[i, j] = w_i Σ_n (t_i·F_i[n]) x[n, j]  (PSSFSS.jl:444-452,
// Eqs. 6.18 / 6.37) with a fixed-order tree reduction.
#include "pss_internal.cuh"

namespace {

__device__ __forceinline__ double j0s(double x) {
  if (fabs(x) < 1e-3) { double x2 = x * x; return 1 - x2 / 6 * (1 - x2 / 20); }
  return sin(x) / x;
}
__device__ __forceinline__ double j1s(double x) {
  if (fabs(x) < 1e-3) return x * (1.0 / 3 - x * x / 30);
  double s, c;
  sincos(x, &s, &c);
  return (s / x - c) / x;
}

// Transform of face f's RWG half-function whose free vertex is local vertex i.
__device__ void face_ft(const SheetDev &G, int f, int i, double kx, double ky, cd &fx, cd &fy) {
  const int nxt[3] = {1, 2, 0};
  double r[3][2], lv[3][2], rc[3][2];
  for (int q = 0; q < 3; ++q) {
    int v = G.fv[3 * f + q];
    r[q][0] = G.rho[2 * v] / G.upm;
    r[q][1] = G.rho[2 * v + 1] / G.upm;
  }
  double lmax = 0;
  for (int q = 0; q < 3; ++q) {
    lv[q][0] = r[nxt[q]][0] - r[q][0];
    lv[q][1] = r[nxt[q]][1] - r[q][1];
    rc[q][0] = r[q][0] + 0.5 * lv[q][0];
    rc[q][1] = r[q][1] + 0.5 * lv[q][1];
    lmax = fmax(lmax, sqrt(lv[q][0] * lv[q][0] + lv[q][1] * lv[q][1]));
  }
  double kmagsq = kx * kx + ky * ky;
  double kmag = sqrt(kmagsq);
  if (kmag * lmax < 1e-4) {
    double cx = ((r[0][0] + r[1][0]) + r[2][0]) / 3, cy = ((r[0][1] + r[1][1]) + r[2][1]) / 3;
    cd cph = cisd(kx * cx + ky * cy);
    fx = (0.5 * (cx - r[i][0])) * cph;
    fy = (0.5 * (cy - r[i][1])) * cph;
    return;
  }
  double kfx = 2 * kx / kmagsq, kfy = 2 * ky / kmagsq;
  double darea = lv[0][0] * lv[1][1] - lv[0][1] * lv[1][0];
  double denom = darea * kmagsq;
  cd cs0 = mkcd(0, 0), cs1 = mkcd(0, 0);
  for (int n = 0; n < 3; ++n) {
    double zl = lv[n][0] * ky - lv[n][1] * kx;
    double dk = 0.5 * (kx * lv[n][0] + ky * lv[n][1]);
    double j0 = j0s(dk), j1 = j1s(dk);
    double rt0 = ((0.5 * zl) * j1) * lv[n][0], rt1 = ((0.5 * zl) * j1) * lv[n][1];
    cd cph = cisd(kx * rc[n][0] + ky * rc[n][1]);
    // ctrm1 = i*rc - kfact ; cjr = i*r[i]
    cd c10 = mkcd(-kfx, rc[n][0]) - mkcd(0.0, r[i][0]);
    cd c11 = mkcd(-kfy, rc[n][1]) - mkcd(0.0, r[i][1]);
    cd t0 = j0 * (mkcd(-lv[n][1], 0) + zl * c10);
    cd t1 = j0 * (mkcd(lv[n][0], 0) + zl * c11);
    cs0 = cs0 + cph * (t0 - mkcd(rt0, 0));
    cs1 = cs1 + cph * (t1 - mkcd(rt1, 0));
  }
  fx = cs0 / denom;
  fy = cs1 / denom;
}

__global__ void k_bfft(SheetDev G, int nmodes, const double *__restrict__ kvec, double psi1, double psi2,
                       cd *__restrict__ bf) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (n >= G.nbf) return;
  double kx = kvec[2 * j], ky = kvec[2 * j + 1];
  cd ff[5] = {mkcd(1, 0), mkcd(1, 0), cisd(-psi1), mkcd(1, 0), cisd(-psi2)};
  cd ax = mkcd(0, 0), ay = mkcd(0, 0);
  for (int a = 0; a < G.inc_cnt[n]; ++a) {
    int f = G.inc_face[4 * n + a], i = G.inc_loc[4 * n + a];
    cd fx, fy;
    face_ft(G, f, i, kx, ky, fx, fy);
    cd w = ff[G.inc_eci[4 * n + a]];
    if (G.inc_sgn[4 * n + a] > 0) {
      ax = ax + fx * w;
      ay = ay + fy * w;
    } else {
      ax = ax - fx * w;
      ay = ay - fy * w;
    }
  }
  size_t o = ((size_t)j * G.nbf + n) * 2;
  bf[o] = ax;
  bf[o + 1] = ay;
}

// rhs[n + j*nbf] = conj(F_j[n]) · src_j
__global__ void k_rhs(int nbf, int nmodes, const cd *__restrict__ bf, const cd *__restrict__ src,
                      cd *__restrict__ rhs) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (n >= nbf) return;
  size_t o = ((size_t)j * nbf + n) * 2;
  cd sx = src[2 * j], sy = src[2 * j + 1];
  rhs[(size_t)j * nbf + n] = conjd(bf[o]) * sx + conjd(bf[o + 1]) * sy;
}

// dS[i + j*nm] = w_i * Σ_n (t_i · F_i[n]) X[n + j*nbf]
__global__ void k_project(int nbf, int nm, const cd *__restrict__ bf, const double *__restrict__ tobs,
                          const cd *__restrict__ wobs, const cd *__restrict__ X, cd *__restrict__ dS) {
  int i = blockIdx.x, j = blockIdx.y;
  double tx = tobs[2 * i], ty = tobs[2 * i + 1];
  const cd *F = bf + (size_t)i * nbf * 2;
  const cd *x = X + (size_t)j * nbf;
  cd acc = mkcd(0, 0);
  for (int n = threadIdx.x; n < nbf; n += blockDim.x) {
    cd p = tx * F[2 * n] + ty * F[2 * n + 1];
    acc = acc + p * x[n];
  }
  __shared__ cd red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) dS[i + (size_t)j * nm] = wobs[i] * red[0];
}

// PT[n + i*nbf] = t_i · F_i[n]: the projection rows of dS = w ∘ (P X), transposed, which are
// the right-hand sides of the adjoint solve Z^T Lam = P^T.
__global__ void k_proj_rows(int nbf, const cd *__restrict__ bf, const double *__restrict__ tobs, cd *__restrict__ PT) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
  if (n >= nbf) return;
  const cd *F = bf + (size_t)i * nbf * 2;
  PT[(size_t)i * nbf + n] = tobs[2 * i] * F[2 * n] + tobs[2 * i + 1] * F[2 * n + 1];
}

}  // namespace

void pss_proj_rows(int nbf, int nmodes, const cd *bf, const double *tobs, cd *PT, cudaStream_t st) {
  pss_count_launch();
  k_proj_rows<<<dim3(cdiv_u(nbf, 256), nmodes), 256, 0, st>>>(nbf, bf, tobs, PT);
}

void pss_bfft(const SheetDev &G, int nmodes, const double *kvec, double psi1, double psi2, cd *bf,
              cudaStream_t st) {
  pss_count_launch();
  k_bfft<<<dim3(cdiv_u(G.nbf, 128), nmodes), 128, 0, st>>>(G, nmodes, kvec, psi1, psi2, bf);
}

void pss_rhs(int nbf, int nmodes, const cd *bf, const cd *src, cd *rhs, cudaStream_t st) {
  pss_count_launch();
  k_rhs<<<dim3(cdiv_u(nbf, 256), nmodes), 256, 0, st>>>(nbf, nmodes, bf, src, rhs);
}

void pss_project(int nbf, int nmodes, const cd *bf, const double *tobs, const cd *wobs, const cd *X, cd *dS,
                 cudaStream_t st) {
  pss_count_launch();
  k_project<<<dim3(nmodes, nmodes), 256, 0, st>>>(nbf, nmodes, bf, tobs, wobs, X, dS);
}
