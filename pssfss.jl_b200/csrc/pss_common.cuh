// Shared device helpers for the periodic MoM fill-and-solve library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#define PSS_PI 3.141592653589793
#define PSS_TWOPI 6.283185307179586
#define PSS_FOURPI 12.566370614359172
#define PSS_MU0 1.25663706212e-6
#define PSS_C0 299792458.0
#define PSS_MMAX_CAP 2048
#define PSS_JKRINGMAX 65
#define PSS_CONVREPEAT 40
#define PSS_MAXLAYERS 32

// Status bits reported per frequency point (no device traps: loops are capped).
enum {
  PSS_ST_TABLE_NOCONV = 1,   // modal tables hit mmax = 2048 without 40 converged rings
  PSS_ST_JK_NOCONV = 2,      // a spatial lattice sum hit 65 rings
  PSS_ST_SINGULAR = 4,       // zero pivot in the LU
  PSS_ST_REFINE_NOCONV = 8,  // iterative refinement did not reach its tolerance
  PSS_ST_NONFINITE = 16,     // NaN/Inf in the solution
  PSS_ST_FP64_FALLBACK = 32, // FP32 refinement stalled; the point was recomputed in FP64
  PSS_ST_DEVICE_TIMEOUT = 64, // a bounded device-side wait gave up; results are invalid
};

struct cd {
  double x, y;
};
struct cf {
  float x, y;
};

__host__ __device__ __forceinline__ cd mkcd(double x, double y) { return cd{x, y}; }
__host__ __device__ __forceinline__ cd operator+(cd a, cd b) { return cd{a.x + b.x, a.y + b.y}; }
__host__ __device__ __forceinline__ cd operator-(cd a, cd b) { return cd{a.x - b.x, a.y - b.y}; }
__host__ __device__ __forceinline__ cd operator-(cd a) { return cd{-a.x, -a.y}; }
__host__ __device__ __forceinline__ cd operator*(cd a, cd b) {
  return cd{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
__host__ __device__ __forceinline__ cd operator*(double s, cd a) { return cd{s * a.x, s * a.y}; }
__host__ __device__ __forceinline__ cd operator/(cd a, double s) { return cd{a.x / s, a.y / s}; }
__host__ __device__ __forceinline__ cd conjd(cd a) { return cd{a.x, -a.y}; }
// Real - Complex keeping the sign of a zero imaginary part: Complex(x - re, -im).
__host__ __device__ __forceinline__ cd rsubc(double x, cd z) { return cd{x - z.x, -z.y}; }

// Smith's complex division with scaling.
__host__ __device__ __forceinline__ cd operator/(cd a, cd b) {
  if (fabs(b.y) <= fabs(b.x)) {
    double r = b.y / b.x, d = b.x + b.y * r;
    return cd{(a.x + a.y * r) / d, (a.y - a.x * r) / d};
  } else {
    double r = b.x / b.y, d = b.y + b.x * r;
    return cd{(a.x * r + a.y) / d, (a.y * r - a.x) / d};
  }
}

__device__ __forceinline__ double cabsd(cd a) { return hypot(a.x, a.y); }

// Principal square root (branch cut on the negative real axis, sign of imag kept).
__device__ __forceinline__ cd csqrtd(cd z) {
  if (z.x == 0.0 && z.y == 0.0) return cd{0.0, z.y};
  double t = sqrt((fabs(z.x) + hypot(z.x, z.y)) * 0.5);
  if (z.x >= 0.0) return cd{t, z.y / (2.0 * t)};
  return cd{fabs(z.y) / (2.0 * t), copysign(t, z.y)};
}

// PGF.jl:116-120 mysqrt: flip a pure negative-imaginary root to positive imaginary.
__device__ __forceinline__ cd mysqrtd(cd z) {
  cd a = csqrtd(z);
  if (a.x == 0.0 && a.y < 0.0) a = cd{-a.x, -a.y};
  return a;
}

// Complex tanh (Kahan's formulation, as in C99 ctanh).
__device__ __forceinline__ cd ctanhd(cd z) {
  double x = z.x, y = z.y;
  if (fabs(x) > 22.0) {
    double e = exp(-2.0 * fabs(x));
    double s, c;
    sincos(y, &s, &c);
    return cd{copysign(1.0, x), 4.0 * s * c * e};
  }
  double t = tan(y);
  double beta = 1.0 + t * t;
  double sh = sinh(x);
  double rho = sqrt(1.0 + sh * sh);
  double den = 1.0 + beta * sh * sh;
  return cd{(beta * rho * sh) / den, t / den};
}

__device__ __forceinline__ cd cisd(double a) {
  double s, c;
  sincos(a, &s, &c);
  return cd{c, s};
}

// Rings.jl:14-55 -- element idx of summation ring r.
__host__ __device__ __forceinline__ void ring_mn(int r, int idx, int &m, int &n) {
  if (r == 0) { m = 0; n = 0; return; }
  int w = 2 * r + 1;
  if (idx < w) { m = r; n = -r + idx; return; }
  idx -= w;
  if (idx < w) { m = -r; n = -r + idx; return; }
  idx -= w;
  int h = 2 * r - 1;
  if (idx < h) { m = -r + 1 + idx; n = -r; return; }
  idx -= h;
  m = -r + 1 + idx;
  n = r;
}
__host__ __device__ __forceinline__ int ring_len(int r) { return r == 0 ? 1 : 8 * r; }

// 7-point triangle rule (Zint.jl:55-62)
__constant__ static double c_qxi[7] = {0.33333333333333330, 0.10128650732345633, 0.79742698535308730,
                                       0.10128650732345633, 0.47014206410511505, 0.05971587178976989,
                                       0.47014206410511505};
__constant__ static double c_qeta[7] = {0.33333333333333333, 0.79742698535308730, 0.10128650732345633,
                                        0.10128650732345633, 0.05971587178976989, 0.47014206410511505,
                                        0.47014206410511505};
__constant__ static double c_qw[7] = {0.1125, 0.06296959027241358, 0.06296959027241358,
                                      0.06296959027241358, 0.06619707639425308, 0.06619707639425308,
                                      0.06619707639425308};

#define PSS_CUDA_TRY(expr)                                                        \
  do {                                                                            \
    cudaError_t _e = (expr);                                                      \
    if (_e != cudaSuccess) {                                                      \
      pss_set_error("%s:%d %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(_e)); \
      return -3;                                                                  \
    }                                                                             \
  } while (0)

void pss_set_error(const char *fmt, ...);

static inline unsigned cdiv_u(long long a, long long b) { return (unsigned)((a + b - 1) / b); }
