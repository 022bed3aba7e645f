// C ABI of the library: contexts, device-resident sheets and the batched sweep.
//
// pss_partial_gsms is the drop-in for the hot body of calculate_jtype_gsm /
// calculate_mtype_gsm (PSSFSS.jl:391-457, 516-584) over a whole sweep:
//   1. modal tables of every point (K1; the only phase with host synchronisation, to
//      read back each point's mmax);
//   2. the J/K face-pair integrals (K2) when (ψ1, ψ2, u) differ from the cached key
//      (FillZY.jl:97-99): once per sweep at normal incidence or fixed ψ, per point for
//      θ steering;
//   3. per point on one of nworkers CUDA streams: pair terms (K3a), gather assembly (K3b),
//      LU (K4), basis transforms and right-hand sides (K6), solves (K5) with FP64
//      iterative refinement in the FP32 form, modal projection (K6);
//   4. one synchronisation, then dS and status are copied to the caller.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "pss_internal.cuh"
#include "pssfss_b200.h"

#include <atomic>

static thread_local char g_err[1024];
static std::atomic<long long> g_launches{0};

void pss_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

namespace {
struct KProf {
  std::vector<cudaEvent_t> e0, e1;
  std::vector<double> work;
  std::vector<int> kind;
};
thread_local KProf *g_kprof = nullptr;
}  // namespace

int pss_prof_begin(cudaStream_t st) {
  if (!g_kprof) return -1;
  cudaEvent_t a;
  if (cudaEventCreate(&a) != cudaSuccess) return -1;
  cudaEventRecord(a, st);
  g_kprof->e0.push_back(a);
  return (int)g_kprof->e0.size() - 1;
}

void pss_prof_end(int token, cudaStream_t st, int kind, double work) {
  if (token < 0 || !g_kprof) return;
  cudaEvent_t b;
  cudaEventCreate(&b);
  cudaEventRecord(b, st);
  g_kprof->e1.push_back(b);
  g_kprof->work.push_back(work);
  g_kprof->kind.push_back(kind);
}

void pss_set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

namespace {

constexpr int kRing0 = 160;  // ring budget of the first table pass (mmax <= 320)
constexpr int kTableChunk = 16;
constexpr int kMaxRefine = 10;  // refinement steps before the FP64 fallback (zcgesv allows 30)

struct DevBuf {
  void *p = nullptr;
  size_t n = 0;
  int ensure(size_t bytes) {
    if (bytes <= n) return 0;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    if (bytes == 0) return 0;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      pss_set_error("cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
      p = nullptr;
      return -3;
    }
    n = bytes;
    return 0;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  template <class T>
  T *as() const { return (T *)p; }
};

// A DevBuf owned by one scope: freed when it goes out of scope (DevBuf itself is a plain
// handle, copied into containers, and never frees on its own).
struct LocalBuf : DevBuf {
  LocalBuf() = default;
  LocalBuf(const LocalBuf &) = delete;
  LocalBuf &operator=(const LocalBuf &) = delete;
  LocalBuf(LocalBuf &&o) noexcept {
    p = o.p;
    n = o.n;
    o.p = nullptr;
    o.n = 0;
  }
  ~LocalBuf() { release(); }
};

struct JKBufs {
  DevBuf buf;
  JKDev jk{};
  int ensure(int nufp) {
    size_t c = (size_t)nufp * sizeof(cd), d = (size_t)nufp * sizeof(double);
    if (buf.ensure(6 * c + 3 * d + 64)) return -3;
    char *b = (char *)buf.p;
    jk.J = (cd *)b; jk.Jxi = (cd *)(b + c); jk.Jeta = (cd *)(b + 2 * c);
    jk.K = (cd *)(b + 3 * c); jk.Kxi = (cd *)(b + 4 * c); jk.Keta = (cd *)(b + 5 * c);
    jk.rho_r = (double *)(b + 6 * c);
    jk.rinv = (double *)(b + 6 * c + 2 * d);
    return 0;
  }
};

__global__ void k_info_to_status(int nb, int *info, int *status);

// One CUDA stream with buffers for a batch of up to `cap` frequency points: their matrices,
// pivots, right-hand sides and solutions side by side (matrix b at offset b*n*n, vectors
// at b*n*nrhs), factored and solved together by the batched LU and solve kernels.
struct Worker {
  cudaStream_t st = nullptr;
  int cap = 1;  // batch capacity (points)
  DevBuf zb, z64, zr, zi, ipiv, info, bstat, bf, rhs, X, R, D, nonconv, luws, solvews;
  JKBufs jk, jkx[kJKGroup - 1];  // face integrals of the points whose phasing varies: slots 0..kJKGroup
  SolveWS sws;
  JKDev jk_slot(int q) const { return q == 0 ? jk.jk : jkx[q - 1].jk; }
  int ensure_solver(int n, int nrhs, int nb) {
    if (ipiv.ensure((size_t)nb * n * sizeof(int)) || info.ensure((size_t)nb * sizeof(int)) ||
        bstat.ensure((size_t)nb * sizeof(int)))
      return -3;
    if (luws.ensure(std::max(pss_lu_ws_bytes(n, 0, nb), pss_lu_ws_bytes(n, 1, nb)))) return -3;
    if (solvews.ensure(pss_solve_ws_bytes(n, nb))) return -3;
    sws.bind(solvews.p, n, nb);
    const size_t v = (size_t)nb * n * nrhs * sizeof(cd);
    if (rhs.ensure(v) || X.ensure(v) || R.ensure(v) || D.ensure(v)) return -3;
    return 0;
  }
  // Leading dimension of the FP32 planes: rows padded to 32 floats (128 bytes), so every row
  // starts on a 16-byte boundary - the tensor-core update's TMA reduce-add epilogue needs
  // that - and the panel and interchange kernels move whole 128-byte lines.
  static long long ld32(int n) { return ((long long)n + 31) & ~31LL; }
  // LU of the worker's first nb matrices (FP64 in z64, or FP32 planes zr/zi) and solves
  // rhs -> X, refined against z64 in FP32 mode.  Status bits go to status[0..nb) (device).
  int factor_solve(int n, int nb, int prec, int nrhs, int maxit, int *status, int panel_w = 0, int outer_nb = 0) {
    int rc;
    const long long ld = n, ms = (long long)n * n, vs = (long long)n * nrhs;
    const long long ldf = ld32(n), msf = (long long)n * ldf;
    if (prec == PSS_FP64)
      rc = pss_lu64_batched(n, nb, z64.as<cd>(), ld, ms, ipiv.as<int>(), info.as<int>(), luws.p, luws.n, st);
    else
      rc = pss_lu32_batched(n, nb, zr.as<float>(), zi.as<float>(), ldf, msf, ipiv.as<int>(), info.as<int>(), luws.p,
                            luws.n, st, panel_w, outer_nb);
    if (rc) return rc;
    pss_count_launch();
    k_info_to_status<<<1, 32, 0, st>>>(nb, info.as<int>(), status);
    const cd *L64 = prec == PSS_FP64 ? z64.as<cd>() : nullptr;
    const float *Lr = prec == PSS_FP64 ? nullptr : zr.as<float>();
    const float *Li = prec == PSS_FP64 ? nullptr : zi.as<float>();
    const long long fld = L64 ? ld : ldf, fms = L64 ? ms : msf;  // the factor's layout
    if ((rc = pss_solve_prepare(sws, nb, L64, Lr, Li, fld, fms, ipiv.as<int>(), st))) return rc;
    if ((rc = pss_solve_lu(sws, nb, L64, Lr, Li, fld, fms, nrhs, rhs.as<cd>(), X.as<cd>(), vs, 0, st))) return rc;
    if (prec == PSS_FP32_REFINE &&
        (rc = pss_refine(sws, nb, z64.as<cd>(), ld, ms, Lr, Li, ldf, msf, nrhs, rhs.as<cd>(), X.as<cd>(), R.as<cd>(),
                         D.as<cd>(), vs, maxit, status, st)))
      return rc;
    pss_solve_status(sws, nb, status, st);
    return 0;
  }
};

// Batch-local status words OR-ed into the points' status words.
constexpr int kMaxBatch = 32;
struct StatusMap {
  int idx[kMaxBatch];
};
__global__ void k_status_scatter(int cnt, const int *bstat, int *status, StatusMap sm) {
  for (int b = threadIdx.x; b < cnt; b += blockDim.x) status[sm.idx[b]] |= bstat[b];
}

__global__ void k_info_to_status(int nb, int *info, int *status) {
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    if (info[b] > 0) status[b] |= PSS_ST_SINGULAR;
    if (info[b] < 0) status[b] |= PSS_ST_DEVICE_TIMEOUT;
    info[b] = 0;
  }
}
__global__ void k_nonconv_to_status(int *nonconv, int *status) {
  if (*nonconv) *status |= PSS_ST_JK_NOCONV;
  *nonconv = 0;
}

// c3_calc / d3_calc (PGF.jl:138-162)
cd c3_calc(double k0, double u, cd mu1, cd eps1, cd mu2, cd eps2) {
  cd w1 = ((k0 * k0) * mu1) * eps1 + mkcd(u * u, 0);
  cd w2 = ((k0 * k0) * mu2) * eps2 + mkcd(u * u, 0);
  return (mu1 * w2 + mu2 * w1) / (2.0 * (mu1 + mu2));
}
cd d3_calc(double k0, double u, cd mu1, cd eps1, cd mu2, cd eps2) {
  cd w1 = ((k0 * k0) * mu1) * eps1 + mkcd(u * u, 0);
  cd w2 = ((k0 * k0) * mu2) * eps2 + mkcd(u * u, 0);
  cd num = mu1 * (w2 * (2.0 * eps1 + eps2) - w1 * eps1) + mu2 * (w1 * (2.0 * eps2 + eps1) - w2 * eps2);
  return num / ((2.0 * (mu1 + mu2)) * (eps1 + eps2));
}
cd hcis(double a) { return mkcd(std::cos(a), std::sin(a)); }

}  // namespace

struct pss_ctx {
  int device = 0;
  int nworkers = 1;
  int batch = 12;  // points per batched factorisation (PSS_BATCH, 1..32)
  std::vector<Worker> w;
  DevBuf params, dense, conv, mm, stage, tables, bigdense, modes, dS, status;
  std::vector<DevBuf> bigtables;
  double last_ms[8] = {0};
  bool prof_on = false;
  double prof[3 * PSS_PROF_KINDS] = {};  // per kind: launches, summed ms, summed algorithmic work
};

struct pss_sheet {
  pss_ctx *ctx = nullptr;
  char cls = 'J';
  double upm = 1.0;
  double s1[2], s2[2], b1[2], b2[2];
  int nnode = 0, nface = 0, nbf = 0, nufp = 0;
  DevBuf rho, fv, ufpm, rep, fr, ls, a48, inc_cnt, inc_face, inc_loc, inc_sgn, inc_eci;
  SheetDev G{};
  JKBufs cache;
  bool jk_valid = false;
  double jk_psi1 = 0, jk_psi2 = 0, jk_u = 0;
  int jk_nonconv = 0;
};

namespace {

int set_device(pss_ctx *c) {
  PSS_CUDA_TRY(cudaSetDevice(c->device));
  return 0;
}

template <class T>
int upload(DevBuf &b, const T *h, size_t n) {
  if (b.ensure(std::max<size_t>(n, 1) * sizeof(T))) return -3;
  if (n) PSS_CUDA_TRY(cudaMemcpy(b.p, h, n * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

int make_stack(int nl, const double *eps, const double *mu, const double *width, int s, StackParams &S) {
  if (nl < 2 || nl > PSS_MAXLAYERS) { pss_set_error("layer count %d outside 2..%d", nl, PSS_MAXLAYERS); return -1; }
  if (s < 1 || s >= nl) { pss_set_error("interface %d outside 1..%d", s, nl - 1); return -1; }
  S.nl = nl;
  S.s = s;
  for (int i = 0; i < nl; ++i) {
    S.eps[i] = mkcd(eps[2 * i], eps[2 * i + 1]);
    S.mu[i] = mkcd(mu[2 * i], mu[2 * i + 1]);
    S.width[i] = width[i];
    if (!std::isfinite(eps[2 * i]) || !std::isfinite(eps[2 * i + 1]) || !std::isfinite(mu[2 * i]) ||
        !std::isfinite(mu[2 * i + 1]) || !std::isfinite(width[i])) {
      pss_set_error("non-finite layer parameter in layer %d", i + 1);
      return -1;
    }
  }
  return 0;
}

// Per-point scalars: FillZY.jl:60-77 / 282-322 and PGF.jl:202-210 / 483-499.
void make_params(int magnetic, const StackParams &S, const double b1m[2], const double b2m[2], double u,
                 double k0, double psi1, double psi2, PointParams &P) {
  memset(&P, 0, sizeof(P));
  P.magnetic = magnetic;
  P.k0 = k0;
  P.u = u;
  P.psi1 = psi1;
  P.psi2 = psi2;
  P.omega = k0 * PSS_C0;
  for (int d = 0; d < 2; ++d) {
    P.b1[d] = b1m[d];
    P.b2[d] = b2m[d];
    P.b00[d] = (psi1 * b1m[d] + psi2 * b2m[d]) / PSS_TWOPI;
  }
  double cr = b1m[0] * b2m[1] - b1m[1] * b2m[0];
  P.area = 4.0 * (PSS_PI * PSS_PI) / std::fabs(cr);
  P.k0sq = k0 * k0;
  P.b2min = 1e-10 * P.k0sq;
  const int s = S.s;
  cd mus = S.mu[s - 1], mus1 = S.mu[s], epss = S.eps[s - 1], epss1 = S.eps[s];
  P.mutilde = ((2.0 * mus) * mus1) / (mus + mus1);
  P.epsbar = (epss + epss1) / 2.0;
  if (!magnetic) {
    P.c3 = c3_calc(k0, u, mus, epss, mus1, epss1);
    P.d3 = d3_calc(k0, u, mus, epss, mus1, epss1);
  } else {
    cd c3s = c3_calc(k0, u, epss, mus, epss, mus);
    cd c3sp1 = c3_calc(k0, u, epss1, mus1, epss1, mus1);
    cd d3s = d3_calc(k0, u, epss, mus, epss, mus);
    cd d3sp1 = d3_calc(k0, u, epss1, mus1, epss1, mus1);
    P.f1 = 2.0 * P.epsbar;
    P.f3 = epss * c3s + epss1 * c3sp1;
    P.p1 = mkcd(2.0, 0) / P.mutilde;
    P.p3 = d3s / mus + d3sp1 / mus1;
    cd fc3s = c3_calc(k0, u, mus, epss, mus, epss);
    cd fc3sp1 = c3_calc(k0, u, mus1, epss1, mus1, epss1);
    cd fd3s = d3_calc(k0, u, mus, epss, mus, epss);
    cd fd3sp1 = d3_calc(k0, u, mus1, epss1, mus1, epss1);
    P.I1fact = mkcd(PSS_PI, 0) / P.epsbar;
    P.KFfact = (fc3s * epss + fc3sp1 * epss1) / (u * (2.0 * P.epsbar));
    P.I2fact = PSS_PI * P.mutilde;
    P.KPfact = (P.mutilde / (2 * u)) * (fd3s / mus + fd3sp1 / mus1);
  }
  P.ff[0] = P.ff[1] = P.ff[3] = mkcd(1, 0);
  P.ff[2] = hcis(-psi1);
  P.ff[4] = hcis(-psi2);
}

// Tables of npts points (params already on the device at dP).  Fills tabs[i] and ORs
// PSS_ST_TABLE_NOCONV into hstatus[i].  Synchronises the ctx's first stream.
int build_tables(pss_ctx *c, const StackParams &S, const PointParams *dP, int npts, double convtest,
                 std::vector<TableDev> &tabs, std::vector<int> &hstatus, int base = 0) {
  cudaStream_t st = c->w[0].st;
  const int R0 = kRing0;
  const size_t W0 = 2 * (size_t)R0 + 1;
  const size_t pstride = 2 * W0 * W0;
  const int chunk = std::min(npts, kTableChunk);
  const size_t cap0 = (size_t)(2 * R0 + 2) * (2 * R0 + 2);
  if (c->dense.ensure((size_t)chunk * pstride * sizeof(cd))) return -3;
  if (c->conv.ensure((size_t)chunk * (R0 + 1) + 64)) return -3;
  if (c->mm.ensure(2 * sizeof(int) * (size_t)chunk + 64)) return -3;
  if (c->stage.ensure(2 * (size_t)(2 * R0) * (2 * R0) * sizeof(cd))) return -3;
  // points base .. base+npts-1 of the call; a multi-problem call sizes the table store for
  // all its points before the first problem, so this never reallocates under earlier tables
  if (c->tables.ensure((size_t)(base + npts) * 2 * cap0 * sizeof(cd))) return -3;
  if ((int)c->bigtables.size() < base + npts) c->bigtables.resize(base + npts);
  if ((int)tabs.size() < base + npts) tabs.resize(base + npts, TableDev{});
  if ((int)hstatus.size() < base + npts) hstatus.resize(base + npts, 0);
  std::vector<int> hm(2 * chunk);
  for (int c0 = 0; c0 < npts; c0 += chunk) {
    const int nc = std::min(chunk, npts - c0);
    int *dmm = c->mm.as<int>();
    pss_tables_ring_fill(S, dP + c0, nc, R0, c->dense.as<cd>(), pstride, st);
    pss_tables_ring_sums(dP + c0, nc, R0, c->dense.as<cd>(), pstride, convtest, c->conv.as<unsigned char>(), st);
    pss_tables_find_mmax(nc, R0, c->conv.as<unsigned char>(), dmm, dmm + chunk, st);
    PSS_CUDA_TRY(cudaMemcpyAsync(hm.data(), dmm, 2 * chunk * sizeof(int), cudaMemcpyDeviceToHost, st));
    PSS_CUDA_TRY(cudaStreamSynchronize(st));
    for (int q = 0; q < nc; ++q) {
      const int il = c0 + q, i = base + il;  // local (params) and global (storage) index
      int mmax = hm[q], flag = hm[chunk + q];
      if (flag == 2) {
        // rings beyond the first budget: full-size pass for this point only
        const int R1 = PSS_MMAX_CAP / 2;
        const size_t W1 = 2 * (size_t)R1 + 1;
        if (c->bigdense.ensure(2 * W1 * W1 * sizeof(cd))) return -3;
        if (c->conv.ensure((size_t)(R1 + 1) + 64)) return -3;
        pss_tables_ring_fill(S, dP + il, 1, R1, c->bigdense.as<cd>(), 0, st);
        pss_tables_ring_sums(dP + il, 1, R1, c->bigdense.as<cd>(), 0, convtest, c->conv.as<unsigned char>(), st);
        pss_tables_find_mmax(1, R1, c->conv.as<unsigned char>(), dmm, dmm + 1, st);
        int h2[2];
        PSS_CUDA_TRY(cudaMemcpyAsync(h2, dmm, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
        PSS_CUDA_TRY(cudaStreamSynchronize(st));
        mmax = h2[0];
        if (h2[1] == 1) hstatus[i] |= PSS_ST_TABLE_NOCONV;
        size_t cap = pss_table_cap(mmax);
        if (c->bigtables[i].ensure(2 * cap * sizeof(cd))) return -3;
        if (c->stage.ensure(2 * (size_t)mmax * mmax * sizeof(cd))) return -3;
        tabs[i].t1 = c->bigtables[i].as<cd>();
        tabs[i].t2 = tabs[i].t1 + cap;
        tabs[i].mmax = mmax;
        int rc = pss_tables_finish(c->bigdense.as<cd>(), R1, mmax, dP + il, c->stage.as<cd>(), tabs[i].t1,
                                   tabs[i].t2, st);
        if (rc) return rc;
        continue;
      }
      if (flag == 1) hstatus[i] |= PSS_ST_TABLE_NOCONV;
      tabs[i].t1 = c->tables.as<cd>() + (size_t)i * 2 * cap0;
      tabs[i].t2 = tabs[i].t1 + cap0;
      tabs[i].mmax = mmax;
      int rc = pss_tables_finish(c->dense.as<cd>() + (size_t)q * pstride, R0, mmax, dP + il, c->stage.as<cd>(),
                                 tabs[i].t1, tabs[i].t2, st);
      if (rc) return rc;
    }
  }
  PSS_CUDA_TRY(cudaStreamSynchronize(st));
  return 0;
}

bool jk_key_stale(const pss_sheet *sh, double psi1, double psi2, double ulocal) {
  return !sh->jk_valid || psi1 != sh->jk_psi1 || psi2 != sh->jk_psi2 || sh->jk_u == 0 ||
         std::fabs((ulocal - sh->jk_u) / sh->jk_u) > 1e-4;
}

int refresh_jk_cache(pss_sheet *sh, double psi1, double psi2, double ulocal, cudaStream_t st) {
  if (!jk_key_stale(sh, psi1, psi2, ulocal)) return 0;
  if (sh->cache.ensure(sh->nufp)) return -3;
  DevBuf nc;
  if (nc.ensure(sizeof(int))) return -3;
  PSS_CUDA_TRY(cudaMemsetAsync(nc.p, 0, sizeof(int), st));
  pss_filljk(sh->G, ulocal, psi1, psi2, sh->s1, sh->s2, sh->cache.jk, nc.as<int>(), st);
  int h = 0;
  PSS_CUDA_TRY(cudaMemcpyAsync(&h, nc.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  PSS_CUDA_TRY(cudaStreamSynchronize(st));
  nc.release();
  sh->jk_valid = true;
  sh->jk_psi1 = psi1;
  sh->jk_psi2 = psi2;
  sh->jk_u = ulocal;
  sh->jk_nonconv = h;
  return 0;
}

int ensure_worker_dims(Worker &w, int nufp, int nbf, int nm, int precision, bool own_jk, int nb) {
  const size_t n = nbf;
  if (w.zb.ensure((size_t)nufp * 9 * sizeof(cd))) return -3;
  if (w.z64.ensure((size_t)nb * n * n * sizeof(cd))) return -3;
  if (precision == PSS_FP32_REFINE) {
    const size_t pl = (size_t)nb * n * (size_t)Worker::ld32((int)n) * sizeof(float);
    if (w.zr.ensure(pl) || w.zi.ensure(pl)) return -3;
  }
  if (w.nonconv.ensure(kJKGroup * sizeof(int))) return -3;
  if (w.bf.ensure((size_t)nb * nm * n * 2 * sizeof(cd))) return -3;
  if (w.ensure_solver((int)n, nm, nb)) return -3;
  if (own_jk) {
    if (w.jk.ensure(nufp)) return -3;
    for (auto &x : w.jkx)
      if (x.ensure(nufp)) return -3;
  }
  PSS_CUDA_TRY(cudaMemsetAsync(w.info.p, 0, (size_t)nb * sizeof(int), w.st));
  PSS_CUDA_TRY(cudaMemsetAsync(w.nonconv.p, 0, kJKGroup * sizeof(int), w.st));
  return 0;
}

int ensure_worker(Worker &w, const pss_sheet *sh, int nm, int precision, bool own_jk, int nb) {
  return ensure_worker_dims(w, sh->nufp, sh->nbf, nm, precision, own_jk, nb);
}

}  // namespace

size_t pss_table_cap(int mmax) { return (size_t)(mmax + 2) * (mmax + 2); }

extern "C" {

const char *pss_last_error(void) { return g_err; }
int pss_version(void) { return 100; }
int64_t pss_kernel_launches(void) { return (int64_t)g_launches.load(); }

int pss_ctx_create(int device, int nworkers, pss_ctx **out) {
  if (!out) { pss_set_error("null output pointer"); return -1; }
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    pss_set_error("no CUDA device available: %s", cudaGetErrorString(e));
    return -3;
  }
  if (device < 0 || device >= ndev) { pss_set_error("device %d outside 0..%d", device, ndev - 1); return -1; }
  pss_ctx *c = new pss_ctx();
  c->device = device;
  c->nworkers = std::max(1, std::min(nworkers, 16));
  if (const char *bs = std::getenv("PSS_BATCH")) c->batch = std::max(1, std::min(atoi(bs), kMaxBatch));
  if (set_device(c)) { delete c; return -3; }
  c->w.resize(c->nworkers);
  for (auto &w : c->w) {
    if (cudaStreamCreateWithFlags(&w.st, cudaStreamNonBlocking) != cudaSuccess) {
      pss_set_error("cudaStreamCreate failed");
      delete c;
      return -3;
    }
  }
  *out = c;
  return 0;
}

int pss_ctx_destroy(pss_ctx *c) {
  if (!c) return 0;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  for (auto &w : c->w) {
    for (DevBuf *b : {&w.zb, &w.z64, &w.zr, &w.zi, &w.ipiv, &w.info, &w.bstat, &w.bf, &w.rhs, &w.X, &w.R, &w.D, &w.nonconv,
                      &w.luws, &w.solvews})
      b->release();
    w.jk.buf.release();
    for (auto &x : w.jkx) x.buf.release();
    if (w.st) cudaStreamDestroy(w.st);
  }
  for (DevBuf *b : {&c->params, &c->dense, &c->conv, &c->mm, &c->stage, &c->tables, &c->bigdense, &c->modes,
                    &c->dS, &c->status})
    b->release();
  for (auto &b : c->bigtables) b.release();
  delete c;
  return 0;
}

int pss_sheet_create(pss_ctx *ctx, char cls, double units_per_meter, const double *s1, const double *s2,
                     const double *beta1, const double *beta2, int64_t nnode, const double *rho,
                     int64_t nface, const int64_t *fv, const int64_t *fe, const double *fr, int64_t nedge,
                     int64_t nbf, const int64_t *bff, const int64_t *ebf, const int64_t *eci, int64_t nufp,
                     const int64_t *ufpm, const int64_t *ufp_rep, pss_sheet **out) {
  if (!ctx || !out) { pss_set_error("null argument"); return -1; }
  *out = nullptr;
  if (cls != 'J' && cls != 'M') { pss_set_error("sheet class must be 'J' or 'M'"); return -1; }
  if (nface <= 0 || nbf <= 0 || nnode <= 0 || nufp <= 0 || nface > 46000 || nbf > 100000) {
    pss_set_error("invalid sizes nnode=%lld nface=%lld nbf=%lld nufp=%lld", (long long)nnode, (long long)nface,
                  (long long)nbf, (long long)nufp);
    return -1;
  }
  if (!(units_per_meter > 0)) { pss_set_error("units_per_meter must be positive"); return -1; }
  if (set_device(ctx)) return -3;
  pss_sheet *sh = new pss_sheet();
  sh->ctx = ctx;
  sh->cls = cls;
  sh->upm = units_per_meter;
  for (int d = 0; d < 2; ++d) {
    sh->s1[d] = s1[d]; sh->s2[d] = s2[d]; sh->b1[d] = beta1[d]; sh->b2[d] = beta2[d];
  }
  sh->nnode = (int)nnode; sh->nface = (int)nface; sh->nbf = (int)nbf; sh->nufp = (int)nufp;
  // host conversion to 0-based int32 + validation
  std::vector<int> hfv(3 * nface);
  for (int64_t i = 0; i < 3 * nface; ++i) {
    if (fv[i] < 1 || fv[i] > nnode) { pss_set_error("fv[%lld] out of range", (long long)i); delete sh; return -1; }
    hfv[i] = (int)(fv[i] - 1);
    if (fe[i] < 1 || fe[i] > nedge) { pss_set_error("fe[%lld] out of range", (long long)i); delete sh; return -1; }
  }
  // device copy in the reference's order (match face fastest): the assembly gathers a column
  // of a Z tile - consecutive match faces against one source face - whose classes are then
  // consecutive entries of this map
  std::vector<int> hufpm((size_t)nface * nface);
  for (size_t i = 0; i < hufpm.size(); ++i) {
    if (ufpm[i] < 1 || ufpm[i] > nufp) { pss_set_error("ufpm entry out of range"); delete sh; return -1; }
    hufpm[i] = (int)(ufpm[i] - 1);
  }
  std::vector<int> hrep(nufp);
  for (int64_t i = 0; i < nufp; ++i) {
    if (ufp_rep[i] < 1 || ufp_rep[i] > nface * nface) { pss_set_error("ufp_rep out of range"); delete sh; return -1; }
    hrep[i] = (int)(ufp_rep[i] - 1);
  }
  // basis-function incidences: (face, local edge, sign, edge code), fixed order
  std::vector<int> icnt(nbf, 0), iface(4 * nbf, 0), iloc(4 * nbf, 0), isgn(4 * nbf, 0), ieci(4 * nbf, 0);
  for (int64_t f = 0; f < nface; ++f)
    for (int k = 0; k < 3; ++k) {
      int64_t e = fe[3 * f + k];
      int64_t b = ebf[e - 1];
      if (b == 0) continue;
      if (b < 1 || b > nbf) { pss_set_error("ebf entry out of range"); delete sh; return -1; }
      int sgn;
      if (bff[2 * (b - 1)] - 1 == f) sgn = 1;
      else if (bff[2 * (b - 1) + 1] - 1 == f) sgn = -1;
      else { pss_set_error("Impossible situation in edge loop (face %lld, bf %lld)", (long long)f + 1, (long long)b); delete sh; return -1; }
      int &cnt = icnt[b - 1];
      if (cnt >= 4) { pss_set_error("basis function %lld has more than 4 face incidences", (long long)b); delete sh; return -1; }
      int64_t code = eci[e - 1];
      if (code < 0 || code > 4) { pss_set_error("eci entry out of range"); delete sh; return -1; }
      iface[4 * (b - 1) + cnt] = (int)f;
      iloc[4 * (b - 1) + cnt] = k;
      isgn[4 * (b - 1) + cnt] = sgn;
      ieci[4 * (b - 1) + cnt] = (int)code;
      ++cnt;
    }
  // per-face edge lengths (m) and 48|area| (m^2) for the surface-resistance terms
  std::vector<double> hls(3 * nface), ha48(nface);
  for (int64_t f = 0; f < nface; ++f) {
    double r[3][2];
    for (int k = 0; k < 3; ++k) {
      int64_t v = fv[3 * f + k] - 1;
      r[k][0] = rho[2 * v] / units_per_meter;
      r[k][1] = rho[2 * v + 1] / units_per_meter;
    }
    double a32x = r[2][0] - r[1][0], a32y = r[2][1] - r[1][1];
    double a12x = r[0][0] - r[1][0], a12y = r[0][1] - r[1][1];
    double a13x = r[0][0] - r[2][0], a13y = r[0][1] - r[2][1];
    hls[3 * f] = std::sqrt(a32x * a32x + a32y * a32y);
    hls[3 * f + 1] = std::sqrt(a13x * a13x + a13y * a13y);
    hls[3 * f + 2] = std::sqrt(a12x * a12x + a12y * a12y);
    ha48[f] = 48 * std::fabs(0.5 * (a32x * a12y - a32y * a12x));
  }
  std::vector<double> hfr(fr, fr + nface);
  int rc = 0;
  rc |= upload(sh->rho, rho, 2 * (size_t)nnode);
  rc |= upload(sh->fv, hfv.data(), hfv.size());
  rc |= upload(sh->ufpm, hufpm.data(), hufpm.size());
  rc |= upload(sh->rep, hrep.data(), hrep.size());
  rc |= upload(sh->fr, hfr.data(), hfr.size());
  rc |= upload(sh->ls, hls.data(), hls.size());
  rc |= upload(sh->a48, ha48.data(), ha48.size());
  rc |= upload(sh->inc_cnt, icnt.data(), icnt.size());
  rc |= upload(sh->inc_face, iface.data(), iface.size());
  rc |= upload(sh->inc_loc, iloc.data(), iloc.size());
  rc |= upload(sh->inc_sgn, isgn.data(), isgn.size());
  rc |= upload(sh->inc_eci, ieci.data(), ieci.size());
  if (rc) { delete sh; return -3; }
  SheetDev &G = sh->G;
  G.nface = sh->nface; G.nbf = sh->nbf; G.nufp = sh->nufp; G.nnode = sh->nnode; G.upm = units_per_meter;
  G.rho = sh->rho.as<double>(); G.fv = sh->fv.as<int>(); G.ufpm = sh->ufpm.as<int>(); G.ufp_rep = sh->rep.as<int>();
  G.fr = sh->fr.as<double>(); G.face_ls = sh->ls.as<double>(); G.face_a48 = sh->a48.as<double>();
  G.inc_cnt = sh->inc_cnt.as<int>(); G.inc_face = sh->inc_face.as<int>(); G.inc_loc = sh->inc_loc.as<int>();
  G.inc_sgn = sh->inc_sgn.as<int>(); G.inc_eci = sh->inc_eci.as<int>();
  *out = sh;
  return 0;
}

int pss_sheet_destroy(pss_sheet *sh) {
  if (!sh) return 0;
  cudaSetDevice(sh->ctx->device);
  cudaDeviceSynchronize();
  for (DevBuf *b : {&sh->rho, &sh->fv, &sh->ufpm, &sh->rep, &sh->fr, &sh->ls, &sh->a48, &sh->inc_cnt,
                    &sh->inc_face, &sh->inc_loc, &sh->inc_sgn, &sh->inc_eci})
    b->release();
  sh->cache.buf.release();
  delete sh;
  return 0;
}

int pss_ctx_device(const pss_ctx *c, int *dev) {
  if (!c) { pss_set_error("null context"); return -1; }
  *dev = c->device;
  return 0;
}

int pss_sheet_clear_cache(pss_sheet *sh) {
  if (!sh) { pss_set_error("null argument"); return -1; }
  sh->jk_valid = false;
  return 0;
}

}  // extern "C"

namespace {

// One problem of a (multi-problem) sweep call: a sheet, its layer region and its points, with
// the FP32 tile shape and batch size to use (0: defaults), plus what the call derives for it.
struct Problem {
  pss_sheet *sh = nullptr;
  StackParams S{};
  double u = 0;
  int npts = 0, nm = 0;
  const double *k0 = nullptr, *psi = nullptr, *kvec = nullptr, *src = nullptr, *tobs = nullptr, *wobs = nullptr;
  double *dS = nullptr;
  int *status = nullptr;
  int batch = 0, panel_w = 0, outer_nb = 0;
  // derived
  int p0 = 0;                       // first global point index
  size_t kb = 0, sb = 0, tb = 0, wb = 0, db = 0;  // bases in the mode and dS arrays (elements)
  bool own_jk = false;              // face integrals per point (else the sheet's cache)
};

// Validate one problem's arguments and fill its StackParams.
int check_problem(const pss_problem &q, int precision, Problem &P) {
  if (!q.sheet || !q.k0 || !q.psi || !q.dS || !q.status || !q.kvec || !q.src || !q.tobs || !q.wobs || !q.eps ||
      !q.mu || !q.width) {
    pss_set_error("null argument");
    return -1;
  }
  if (q.npts <= 0 || q.nmodes <= 0 || q.nmodes > 4096) { pss_set_error("invalid npts/nmodes"); return -1; }
  if (precision != PSS_FP64 && precision != PSS_FP32_REFINE) { pss_set_error("unknown precision %d", precision); return -1; }
  if (!(q.u > 0)) { pss_set_error("smoothing parameter u must be positive"); return -1; }
  if (q.batch < 0 || q.batch > kMaxBatch) { pss_set_error("batch %d outside 0..%d", q.batch, kMaxBatch); return -1; }
  if (!(q.panel_w == 0 || q.panel_w == 8 || q.panel_w == 16 || q.panel_w == 32) ||
      !(q.outer_nb == 0 || q.outer_nb == 64 || q.outer_nb == 128)) {
    pss_set_error("tile shape: panel_w must be 0, 8, 16 or 32 and outer_nb 0, 64 or 128");
    return -1;
  }
  if (make_stack(q.nl, q.eps, q.mu, q.width, q.s, P.S)) return -1;
  for (int i = 0; i < q.npts; ++i)
    if (!(q.k0[i] > 0) || !std::isfinite(q.psi[2 * i]) || !std::isfinite(q.psi[2 * i + 1])) {
      pss_set_error("invalid k0/psi at point %d", i);
      return -1;
    }
  P.sh = q.sheet; P.u = q.u; P.npts = q.npts; P.nm = q.nmodes;
  P.k0 = q.k0; P.psi = q.psi; P.kvec = q.kvec; P.src = q.src; P.tobs = q.tobs; P.wobs = q.wobs;
  P.dS = q.dS; P.status = q.status;
  P.batch = q.batch; P.panel_w = q.panel_w; P.outer_nb = q.outer_nb;
  return 0;
}

// The adjoint stage of a sweep (pss_partial_gsms_adj): problems 1..K of the call are the
// perturbed input sets of problem 0 - their tables, face integrals and mode data are prepared
// with the sweep, but they take no factorisation; after each batched factorisation of problem
// 0's points the adjoint solves Lam = Z^-T P^T run on the same factors, and every set k gets
//   dSp[k][i] = wobs_k o (P_k X)   and   G[k][i] = Lam^T (R_k - Z_k X)   (device, nm^2 each).
struct AdjSpec {
  int K = 0;
  cd *dSp = nullptr;
  cd *G = nullptr;
};

// The sweep of every problem on one context: tables of all points, then a shared work list of
// batches of like-N points (of one or several problems), largest first, taken by one host thread
// per worker stream; each item runs fill -> batched LU -> solves (+ refinement) -> projection
// on its worker.  FP32 points whose refinement stalls are redone in FP64; then dS and status
// go back to each problem's caller arrays.
int sweep_impl(pss_ctx *c, std::vector<Problem> &PR, int precision, const AdjSpec *adj = nullptr) {
  if (set_device(c)) return -3;
  // global point numbering, mode-array bases, parameters
  int total = 0;
  size_t nk = 0, ns = 0, nt = 0, nw = 0, nd = 0;
  for (auto &P : PR) {
    if (P.sh->ctx != c) { pss_set_error("every sheet of a call must belong to the same context"); return -1; }
    P.p0 = total;
    P.kb = nk; P.sb = ns; P.tb = nt; P.wb = nw; P.db = nd;
    const size_t nmp = (size_t)P.npts * P.nm;
    nk += nmp * 2; ns += nmp * 2; nt += nmp * 2; nw += nmp; nd += (size_t)P.npts * P.nm * P.nm;
    total += P.npts;
  }
  std::vector<PointParams> hP(total);
  for (auto &P : PR) {
    const pss_sheet *sh = P.sh;
    const double b1m[2] = {sh->b1[0] * sh->upm, sh->b1[1] * sh->upm};
    const double b2m[2] = {sh->b2[0] * sh->upm, sh->b2[1] * sh->upm};
    for (int i = 0; i < P.npts; ++i)
      make_params(sh->cls == 'M', P.S, b1m, b2m, P.u, P.k0[i], P.psi[2 * i], P.psi[2 * i + 1], hP[P.p0 + i]);
  }
  if (upload(c->params, hP.data(), hP.size())) return -3;
  const PointParams *dP = c->params.as<PointParams>();
  cudaEvent_t span0, span1;
  PSS_CUDA_TRY(cudaEventCreate(&span0));
  PSS_CUDA_TRY(cudaEventCreate(&span1));
  PSS_CUDA_TRY(cudaEventRecord(span0, c->w[0].st));
  // modal tables of every point (the table store is sized for all points first)
  std::vector<int> hstatus(total, 0);
  std::vector<TableDev> tabs(total);
  {
    const size_t cap0 = (size_t)(2 * kRing0 + 2) * (2 * kRing0 + 2);
    if (c->tables.ensure((size_t)total * 2 * cap0 * sizeof(cd))) return -3;
    for (auto &P : PR)
      if (int rc = build_tables(c, P.S, dP + P.p0, P.npts, 1e-7, tabs, hstatus, P.p0)) return rc;
  }
  float tables_ms = 0;
  {
    cudaEvent_t t;
    PSS_CUDA_TRY(cudaEventCreate(&t));
    PSS_CUDA_TRY(cudaEventRecord(t, c->w[0].st));
    PSS_CUDA_TRY(cudaEventSynchronize(t));
    cudaEventElapsedTime(&tables_ms, span0, t);
    cudaEventDestroy(t);
  }
  // mode data of every point of every problem
  const size_t off_k = 0, off_s = off_k + nk * sizeof(double), off_t = off_s + ns * sizeof(cd),
               off_w = off_t + nt * sizeof(double), tot = off_w + nw * sizeof(cd);
  if (c->modes.ensure(tot)) return -3;
  char *mb = c->modes.as<char>();
  const double *dkv = (const double *)(mb + off_k), *dtob = (const double *)(mb + off_t);
  const cd *dsrc = (const cd *)(mb + off_s), *dwob = (const cd *)(mb + off_w);
  for (auto &P : PR) {
    const size_t nmp = (size_t)P.npts * P.nm;
    PSS_CUDA_TRY(cudaMemcpy(mb + off_k + P.kb * sizeof(double), P.kvec, nmp * 2 * sizeof(double), cudaMemcpyHostToDevice));
    PSS_CUDA_TRY(cudaMemcpy(mb + off_s + P.sb * sizeof(cd), P.src, nmp * 2 * sizeof(cd), cudaMemcpyHostToDevice));
    PSS_CUDA_TRY(cudaMemcpy(mb + off_t + P.tb * sizeof(double), P.tobs, nmp * 2 * sizeof(double), cudaMemcpyHostToDevice));
    PSS_CUDA_TRY(cudaMemcpy(mb + off_w + P.wb * sizeof(cd), P.wobs, nmp * sizeof(cd), cudaMemcpyHostToDevice));
  }
  if (c->dS.ensure(std::max<size_t>(nd, 1) * sizeof(cd)) || c->status.ensure((size_t)total * sizeof(int))) return -3;
  PSS_CUDA_TRY(cudaMemset(c->status.p, 0, (size_t)total * sizeof(int)));
  int *dstatus = c->status.as<int>();

  // Face-pair integrals: a problem whose points share (ψ1, ψ2) uses its sheet's cache,
  // refreshed here, unless another problem of the call needs the same sheet at another key
  // (then both compute per point, like problems whose ψ varies).
  {
    std::vector<bool> same(PR.size());
    for (size_t p = 0; p < PR.size(); ++p) {
      const Problem &P = PR[p];
      bool sp = true;
      for (int i = 1; i < P.npts; ++i) sp = sp && P.psi[2 * i] == P.psi[0] && P.psi[2 * i + 1] == P.psi[1];
      same[p] = sp;
      PR[p].own_jk = !sp;
    }
    for (size_t p = 0; p < PR.size(); ++p)
      for (size_t q = 0; q < PR.size(); ++q)
        if (p != q && PR[p].sh == PR[q].sh && same[p] && same[q] &&
            (PR[p].psi[0] != PR[q].psi[0] || PR[p].psi[1] != PR[q].psi[1] || PR[p].u != PR[q].u))
          PR[p].own_jk = true;
    for (auto &P : PR) {
      if (P.own_jk) continue;
      if (int rc = refresh_jk_cache(P.sh, P.psi[0], P.psi[1], P.u / P.sh->upm, c->w[0].st)) return rc;
      if (P.sh->jk_nonconv)
        for (int i = 0; i < P.npts; ++i) hstatus[P.p0 + i] |= PSS_ST_JK_NOCONV;
    }
  }
  // work list: batches of up to B points with the same unknown and mode counts - points of one
  // problem, or of several problems whose sheets have the same N - largest matrices first
  struct Item { int cnt; int p[kMaxBatch]; int i[kMaxBatch]; };
  std::vector<Item> items;
  {
    std::vector<std::pair<int, int>> pts;  // (problem, point); with an adjoint stage only problem 0
    for (size_t p = 0; p < (adj ? 1 : PR.size()); ++p)
      for (int i = 0; i < PR[p].npts; ++i) pts.push_back({(int)p, i});
    std::stable_sort(pts.begin(), pts.end(), [&](const std::pair<int, int> &a, const std::pair<int, int> &b) {
      const Problem &A = PR[a.first], &Bq = PR[b.first];
      if (A.sh->nbf != Bq.sh->nbf) return A.sh->nbf > Bq.sh->nbf;
      return A.nm < Bq.nm;
    });
    // runs of points that may share a batch (same unknown and mode counts and LU tile shape),
    // each cut into near-equal batches of at most B points; a call that is one run (a single
    // sweep) takes a multiple of the worker count, while its batches stay at least half full,
    // so the workers' last rounds end together
    std::vector<std::pair<size_t, size_t>> runs;  // [begin, end) in pts
    for (size_t k = 0; k < pts.size();) {
      const Problem &P = PR[pts[k].first];
      size_t e = k + 1;
      while (e < pts.size() && PR[pts[e].first].sh->nbf == P.sh->nbf && PR[pts[e].first].nm == P.nm &&
             PR[pts[e].first].panel_w == P.panel_w && PR[pts[e].first].outer_nb == P.outer_nb)
        ++e;
      runs.push_back({k, e});
      k = e;
    }
    for (const auto &rn : runs) {
      const Problem &P = PR[pts[rn.first].first];
      const int B = std::max(1, std::min(P.batch > 0 ? P.batch : c->batch, kMaxBatch));
      const long long cnt = (long long)(rn.second - rn.first);
      long long nbat = (cnt + B - 1) / B;
      const long long nw = c->nworkers;
      if (runs.size() == 1 && nbat > 1 && nbat % nw) {
        const long long up = (nbat + nw - 1) / nw * nw;
        if (2 * cnt >= up * (long long)B) nbat = up;  // batches of at least B/2 points
      }
      size_t k = rn.first;
      for (long long q = 0; q < nbat; ++q) {
        const long long sz = cnt / nbat + (q < cnt % nbat ? 1 : 0);
        Item it{};
        for (long long t = 0; t < sz; ++t, ++k) {
          it.p[it.cnt] = pts[k].first;
          it.i[it.cnt] = pts[k].second;
          ++it.cnt;
        }
        items.push_back(it);
      }
    }
  }
  // every worker sized once for the largest item of the call
  const int nwk = c->nworkers;
  {
    int mufp = 0, mn = 0, mnm = 0, mB = 1;
    bool ojk = false;
    for (auto &it : items) {
      for (int b = 0; b < it.cnt; ++b) {
        const Problem &P = PR[it.p[b]];
        mufp = std::max(mufp, P.sh->nufp); mn = std::max(mn, P.sh->nbf); mnm = std::max(mnm, P.nm);
        ojk = ojk || P.own_jk;
      }
      mB = std::max(mB, it.cnt);
    }
    for (auto &P : PR) {  // the perturbed sets' pair terms go through the same buffers
      mufp = std::max(mufp, P.sh->nufp);
      ojk = ojk || P.own_jk;
    }
    for (int k = 0; k < nwk; ++k)
      if (int rc = ensure_worker_dims(c->w[k], mufp, mn, mnm, precision, ojk, mB)) return rc;
  }
  // adjoint-stage buffers of every worker: PT, Lam, scratch W (a batch each), R_k and the
  // set's transforms (one point each), the contraction's CTA shares, refinement scratch
  struct AdjBufs { LocalBuf v, rtw, part; };
  std::vector<AdjBufs> ab(adj ? nwk : 0);
  long long adj_mB = 0;
  if (adj) {
    const int n0 = PR[0].sh->nbf, nm0 = PR[0].nm;
    const size_t vs0 = (size_t)n0 * nm0;
    for (auto &it : items) adj_mB = std::max<long long>(adj_mB, it.cnt);
    for (auto &A : ab)
      if (A.v.ensure((3 * (size_t)adj_mB + 3) * vs0 * sizeof(cd)) ||
          A.rtw.ensure(precision == PSS_FP32_REFINE ? pss_refine_trans_ws_bytes(n0, nm0, (int)adj_mB) : 0) ||
          A.part.ensure(pss_adj_part_bytes(n0, nm0)))
        return -3;
  }
  std::vector<cudaEvent_t> ev;  // phase events of worker 0's batches (pushed by its thread only)
  std::vector<KProf> kprofs(nwk);
  // One batch: per point its problem's fill, transforms and right-hand sides into matrix slot
  // b; one batched LU + solve (+ refinement) of all cnt matrices; per point the projection.
  auto run_batch = [&](const Item &it, int prec, Worker &w, bool rec) -> int {
    cudaStream_t st = w.st;
    const int cnt = it.cnt;
    const Problem &P0 = PR[it.p[0]];
    const int n = P0.sh->nbf, nm = P0.nm;
    const long long ld = n, msz = (long long)n * n, vsz = (long long)n * nm;
    const long long ldf = Worker::ld32(n), msf = (long long)n * ldf;
    const size_t nm2 = (size_t)nm * nm;
    int mufp = 0;
    bool ojk = false;
    for (int b = 0; b < cnt; ++b) {
      mufp = std::max(mufp, PR[it.p[b]].sh->nufp);
      ojk = ojk || PR[it.p[b]].own_jk;
    }
    if (int rc = ensure_worker_dims(w, mufp, n, nm, prec, ojk, cnt)) return rc;
    cudaEvent_t e[8];
    if (rec) {
      for (int q = 0; q < 8; ++q) { cudaEventCreate(&e[q]); ev.push_back(e[q]); }
      cudaEventRecord(e[0], st);
      cudaEventRecord(e[1], st);
    }
    float *zr = prec == PSS_FP32_REFINE ? w.zr.as<float>() : nullptr;
    float *zi = prec == PSS_FP32_REFINE ? w.zi.as<float>() : nullptr;
    for (int b = 0; b < cnt;) {
      // points whose phasing varies take their face integrals in groups of up to kJKGroup
      // points of one sheet (one launch per group), the others read their sheet's cache
      const Problem &P = PR[it.p[b]];
      pss_sheet *sh = P.sh;
      int gsz = 1;
      JKDev jks[kJKGroup];
      if (P.own_jk) {
        while (gsz < kJKGroup && b + gsz < cnt && PR[it.p[b + gsz]].own_jk && PR[it.p[b + gsz]].sh == sh &&
               PR[it.p[b + gsz]].u == P.u)
          ++gsz;
        double p1[kJKGroup], p2[kJKGroup];
        for (int q = 0; q < gsz; ++q) {
          const Problem &Q = PR[it.p[b + q]];
          p1[q] = Q.psi[2 * it.i[b + q]];
          p2[q] = Q.psi[2 * it.i[b + q] + 1];
          jks[q] = w.jk_slot(q);
        }
        pss_filljk_group(sh->G, P.u / sh->upm, gsz, p1, p2, sh->s1, sh->s2, jks, w.nonconv.as<int>(), st);
        for (int q = 0; q < gsz; ++q) {
          pss_count_launch();
          k_nonconv_to_status<<<1, 1, 0, st>>>(w.nonconv.as<int>() + q, dstatus + PR[it.p[b + q]].p0 + it.i[b + q]);
        }
      } else {
        jks[0] = sh->cache.jk;
      }
      for (int q = 0; q < gsz; ++q, ++b) {
        const int g = PR[it.p[b]].p0 + it.i[b];
        const PointParams *Pi = dP + g;
        pss_fill_pairs(sh->G, Pi, jks[q], tabs[g].t1, tabs[g].t2, tabs[g].mmax, w.zb.as<cd>(), st);
        pss_fill_assemble(sh->G, Pi, w.zb.as<cd>(), w.z64.as<cd>() + b * msz, zr ? zr + b * msf : nullptr,
                          zi ? zi + b * msf : nullptr, ld, ldf, st);
      }
    }
    if (rec) cudaEventRecord(e[2], st);
    for (int b = 0; b < cnt; ++b) {
      const Problem &P = PR[it.p[b]];
      const int i = it.i[b];
      const double *kv = dkv + P.kb + (size_t)i * nm * 2;
      const cd *sv = dsrc + P.sb + (size_t)i * nm * 2;
      cd *bf = w.bf.as<cd>() + (size_t)b * nm * n * 2;
      pss_bfft(P.sh->G, nm, kv, P.psi[2 * i], P.psi[2 * i + 1], bf, st);
      pss_rhs(n, nm, bf, sv, w.rhs.as<cd>() + b * vsz, st);
    }
    if (rec) { cudaEventRecord(e[3], st); cudaEventRecord(e[4], st); }
    PSS_CUDA_TRY(cudaMemsetAsync(w.bstat.p, 0, (size_t)cnt * sizeof(int), st));
    int rc2 = w.factor_solve(n, cnt, prec, nm, kMaxRefine, w.bstat.as<int>(), P0.panel_w, P0.outer_nb);
    if (rc2) return rc2;
    if (adj) {
      AdjBufs &A = ab[&w - c->w.data()];
      cd *PT = A.v.as<cd>(), *Lam = PT + adj_mB * vsz, *Wt = Lam + adj_mB * vsz, *Rk = Wt + adj_mB * vsz;
      cd *bfk = Rk + vsz;
      for (int b = 0; b < cnt; ++b) {
        const Problem &P = PR[it.p[b]];
        pss_proj_rows(n, nm, w.bf.as<cd>() + (size_t)b * nm * n * 2, dtob + P.tb + (size_t)it.i[b] * nm * 2,
                      PT + b * vsz, st);
      }
      const cd *L64 = prec == PSS_FP64 ? w.z64.as<cd>() : nullptr;
      const long long fld = L64 ? ld : ldf, fms = L64 ? msz : msf;
      if ((rc2 = pss_solve_lu_trans(w.sws, cnt, L64, zr, zi, fld, fms, nm, PT, Lam, Wt, vsz, 0, st))) return rc2;
      if (prec == PSS_FP32_REFINE &&
          (rc2 = pss_refine_trans(w.sws, cnt, w.z64.as<cd>(), ld, msz, zr, zi, ldf, msf, nm, PT, Lam, w.R.as<cd>(),
                                  w.D.as<cd>(), Wt, A.rtw.p, A.rtw.n, vsz, kMaxRefine, w.bstat.as<int>(), st)))
        return rc2;
      pss_solve_status(w.sws, cnt, w.bstat.as<int>(), st);
      const int np0 = PR[0].npts;
      for (int b = 0; b < cnt; ++b) {
        const int i = it.i[b];
        const cd *Xb = w.X.as<cd>() + b * vsz;
        for (int k = 0; k < adj->K; ++k) {
          const Problem &Q = PR[1 + k];
          const int gq = Q.p0 + i;
          JKDev jq;
          if (!Q.own_jk) {
            jq = Q.sh->cache.jk;
          } else {
            jq = w.jk.jk;
            pss_filljk(Q.sh->G, Q.u / Q.sh->upm, Q.psi[2 * i], Q.psi[2 * i + 1], Q.sh->s1, Q.sh->s2, jq,
                       w.nonconv.as<int>(), st);
            pss_count_launch();
            k_nonconv_to_status<<<1, 1, 0, st>>>(w.nonconv.as<int>(), dstatus + PR[0].p0 + i);
          }
          pss_fill_pairs(Q.sh->G, dP + gq, jq, tabs[gq].t1, tabs[gq].t2, tabs[gq].mmax, w.zb.as<cd>(), st);
          pss_bfft(Q.sh->G, nm, dkv + Q.kb + (size_t)i * nm * 2, Q.psi[2 * i], Q.psi[2 * i + 1], bfk, st);
          pss_rhs(n, nm, bfk, dsrc + Q.sb + (size_t)i * nm * 2, Rk, st);
          const size_t o = ((size_t)k * np0 + i) * nm2;
          pss_project(n, nm, bfk, dtob + Q.tb + (size_t)i * nm * 2, dwob + Q.wb + (size_t)i * nm, Xb, adj->dSp + o,
                      st);
          pss_adj_contract(Q.sh->G, dP + gq, w.zb.as<cd>(), Xb, Rk, Lam + b * vsz, nm, A.part.as<cd>(), adj->G + o,
                           st);
        }
      }
    }
    StatusMap sm{};
    for (int b = 0; b < cnt; ++b) sm.idx[b] = PR[it.p[b]].p0 + it.i[b];
    pss_count_launch();
    k_status_scatter<<<1, 32, 0, st>>>(cnt, w.bstat.as<int>(), dstatus, sm);
    if (rec) cudaEventRecord(e[5], st);
    for (int b = 0; b < cnt; ++b) {
      const Problem &P = PR[it.p[b]];
      const int i = it.i[b];
      const double *tv = dtob + P.tb + (size_t)i * nm * 2;
      const cd *wv = dwob + P.wb + (size_t)i * nm;
      pss_project(n, nm, w.bf.as<cd>() + (size_t)b * nm * n * 2, tv, wv, w.X.as<cd>() + b * vsz,
                  c->dS.as<cd>() + P.db + (size_t)i * nm2, st);
    }
    if (rec) { cudaEventRecord(e[6], st); cudaEventRecord(e[7], st); }
    PSS_CUDA_TRY(cudaGetLastError());
    return 0;
  };
  // One host thread per worker stream, each taking the next item of the shared list, so a
  // stream whose launch queue is full blocks only its own thread.
  {
    std::atomic<int> next{0};
    std::vector<int> wrc(nwk, 0);
    std::vector<std::string> werr(nwk);
    auto feed = [&](int k) {
      if (cudaSetDevice(c->device) != cudaSuccess) {
        wrc[k] = -3;
        werr[k] = "cudaSetDevice failed in a worker thread";
        return;
      }
      g_kprof = c->prof_on ? &kprofs[k] : nullptr;
      for (int q = next.fetch_add(1); q < (int)items.size() && !wrc[k]; q = next.fetch_add(1))
        wrc[k] = run_batch(items[q], precision, c->w[k], k == 0);
      g_kprof = nullptr;
      if (wrc[k]) werr[k] = pss_last_error();
    };
    std::vector<std::thread> th;
    for (int k = 1; k < nwk; ++k) th.emplace_back(feed, k);
    feed(0);
    for (auto &t : th) t.join();
    for (int k = 0; k < nwk; ++k)
      if (wrc[k]) {
        pss_set_error("%s", werr[k].c_str());
        return wrc[k];
      }
  }
  for (auto &w : c->w) PSS_CUDA_TRY(cudaStreamSynchronize(w.st));
  std::vector<int> hst(total);
  PSS_CUDA_TRY(cudaMemcpy(hst.data(), c->status.p, (size_t)total * sizeof(int), cudaMemcpyDeviceToHost));
  // FP32 points whose refinement stalled (cond(Z) * eps32 too close to 1) or went
  // non-finite are recomputed with the FP64 LU; the status keeps a record of it.
  if (precision == PSS_FP32_REFINE) {
    std::vector<int> redo;
    for (int g = 0; g < total; ++g)
      if (hst[g] & (PSS_ST_REFINE_NOCONV | PSS_ST_NONFINITE)) redo.push_back(g);
    if (!redo.empty()) {
      std::vector<int> cleared(total);
      for (int g = 0; g < total; ++g) cleared[g] = hst[g] & ~(PSS_ST_REFINE_NOCONV | PSS_ST_NONFINITE);
      PSS_CUDA_TRY(cudaMemcpy(c->status.p, cleared.data(), (size_t)total * sizeof(int), cudaMemcpyHostToDevice));
      size_t k = 0;
      for (size_t p = 0; p < PR.size(); ++p) {
        Item it{};
        auto flush = [&]() -> int {
          if (!it.cnt) return 0;
          const int rc = run_batch(it, PSS_FP64, c->w[k++ % nwk], false);
          it.cnt = 0;
          return rc;
        };
        const int B = std::max(1, std::min(PR[p].batch > 0 ? PR[p].batch : c->batch, kMaxBatch));
        for (int g : redo) {
          if (g < PR[p].p0 || g >= PR[p].p0 + PR[p].npts) continue;
          it.p[it.cnt] = (int)p;
          it.i[it.cnt] = g - PR[p].p0;
          if (++it.cnt == B)
            if (int rc = flush()) return rc;
        }
        if (int rc = flush()) return rc;
      }
      for (auto &w : c->w) PSS_CUDA_TRY(cudaStreamSynchronize(w.st));
      PSS_CUDA_TRY(cudaMemcpy(hst.data(), c->status.p, (size_t)total * sizeof(int), cudaMemcpyDeviceToHost));
      for (int g : redo) hst[g] |= PSS_ST_FP64_FALLBACK;
    }
  }
  for (size_t k = 1; k < c->w.size(); ++k) {
    cudaEvent_t j;
    PSS_CUDA_TRY(cudaEventCreate(&j));
    PSS_CUDA_TRY(cudaEventRecord(j, c->w[k].st));
    PSS_CUDA_TRY(cudaStreamWaitEvent(c->w[0].st, j, 0));
    cudaEventDestroy(j);
  }
  PSS_CUDA_TRY(cudaEventRecord(span1, c->w[0].st));
  PSS_CUDA_TRY(cudaEventSynchronize(span1));
  float span_ms = 0;
  cudaEventElapsedTime(&span_ms, span0, span1);
  cudaEventDestroy(span0);
  cudaEventDestroy(span1);
  for (auto &P : PR) {
    const size_t nm2 = (size_t)P.nm * P.nm;
    PSS_CUDA_TRY(cudaMemcpy(P.dS, c->dS.as<cd>() + P.db, (size_t)P.npts * nm2 * sizeof(cd), cudaMemcpyDeviceToHost));
    for (int i = 0; i < P.npts; ++i) P.status[i] = hst[P.p0 + i] | hstatus[P.p0 + i];
  }
  for (int q = 0; q < 8; ++q) c->last_ms[q] = 0;
  for (size_t b = 0; b + 8 <= ev.size(); b += 8) {
    float ms;
    const int map[6][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 4}, {4, 5}, {5, 6}};
    for (int q = 0; q < 6; ++q) {
      cudaEventElapsedTime(&ms, ev[b + map[q][0]], ev[b + map[q][1]]);
      c->last_ms[q + 1] += ms;
    }
  }
  for (double &v : c->prof) v = 0;
  for (auto &kprof : kprofs) {
    for (size_t q = 0; q < kprof.e1.size(); ++q) {
      float ms = 0;
      cudaEventElapsedTime(&ms, kprof.e0[q], kprof.e1[q]);
      const int k = kprof.kind[q];
      if (k < 0 || k >= PSS_PROF_KINDS) continue;
      c->prof[3 * k] += 1;
      c->prof[3 * k + 1] += ms;
      c->prof[3 * k + 2] += kprof.work[q];
    }
    for (auto e : kprof.e0) cudaEventDestroy(e);
    for (auto e : kprof.e1) cudaEventDestroy(e);
  }
  c->last_ms[0] = tables_ms;
  c->last_ms[7] = span_ms;
  for (auto e : ev) cudaEventDestroy(e);
  return 0;
}

}  // namespace

extern "C" {

int pss_partial_gsms(pss_sheet *sh, int nl, const double *eps, const double *mu, const double *width, int s,
                     double u, int npts, const double *k0, const double *psi, int nmodes, const double *kvec,
                     const double *src, const double *tobs, const double *wobs, int precision, double *dS,
                     int *status) {
  if (!sh) { pss_set_error("null argument"); return -1; }
  pss_problem q{sh, nl, eps, mu, width, s, u, npts, k0, psi, nmodes, kvec, src, tobs, wobs, 0, 0, 0, dS, status};
  std::vector<Problem> PR(1);
  if (int rc = check_problem(q, precision, PR[0])) return rc;
  return sweep_impl(sh->ctx, PR, precision);
}

int pss_partial_gsms_multi(int nprob, const pss_problem *probs, int precision) {
  if (nprob <= 0 || !probs) { pss_set_error("null or empty problem list"); return -1; }
  std::vector<Problem> PR(nprob);
  for (int p = 0; p < nprob; ++p)
    if (int rc = check_problem(probs[p], precision, PR[p])) {
      const std::string m = pss_last_error();
      pss_set_error("problem %d: %s", p, m.c_str());
      return rc;
    }
  return sweep_impl(probs[0].sheet->ctx, PR, precision);
}

int pss_last_timings(pss_ctx *c, double *ms8) {
  if (!c || !ms8) return -1;
  for (int q = 0; q < 8; ++q) ms8[q] = c->last_ms[q];
  return 0;
}

int pss_profile(pss_ctx *c, int enable) {
  if (!c) { pss_set_error("null context"); return -1; }
  c->prof_on = enable != 0;
  return 0;
}

int pss_profile_result(pss_ctx *c, double *out) {
  if (!c || !out) { pss_set_error("null argument"); return -1; }
  for (int q = 0; q < 3 * PSS_PROF_KINDS; ++q) out[q] = c->prof[q];
  return 0;
}

int pss_fill_matrix(pss_sheet *sh, int nl, const double *eps, const double *mu, const double *width, int s,
                    double u, double k0, double psi1, double psi2, double *Z, int *mmax_out) {
  if (!sh || !Z) { pss_set_error("null argument"); return -1; }
  pss_ctx *c = sh->ctx;
  if (set_device(c)) return -3;
  StackParams S;
  if (make_stack(nl, eps, mu, width, s, S)) return -1;
  const double b1m[2] = {sh->b1[0] * sh->upm, sh->b1[1] * sh->upm};
  const double b2m[2] = {sh->b2[0] * sh->upm, sh->b2[1] * sh->upm};
  PointParams P;
  make_params(sh->cls == 'M', S, b1m, b2m, u, k0, psi1, psi2, P);
  if (upload(c->params, &P, 1)) return -3;
  std::vector<int> hs(1, 0);
  std::vector<TableDev> tabs;
  int rc = build_tables(c, S, c->params.as<PointParams>(), 1, 1e-7, tabs, hs);
  if (rc) return rc;
  Worker &w = c->w[0];
  if ((rc = refresh_jk_cache(sh, psi1, psi2, u / sh->upm, w.st))) return rc;
  if ((rc = ensure_worker(w, sh, 1, PSS_FP64, false, 1))) return rc;
  pss_fill_pairs(sh->G, c->params.as<PointParams>(), sh->cache.jk, tabs[0].t1, tabs[0].t2, tabs[0].mmax,
                 w.zb.as<cd>(), w.st);
  pss_fill_assemble(sh->G, c->params.as<PointParams>(), w.zb.as<cd>(), w.z64.as<cd>(), nullptr, nullptr, sh->nbf, sh->nbf,
                    w.st);
  PSS_CUDA_TRY(cudaStreamSynchronize(w.st));
  const size_t n = sh->nbf;
  std::vector<cd> h(n * n);
  PSS_CUDA_TRY(cudaMemcpy(h.data(), w.z64.p, n * n * sizeof(cd), cudaMemcpyDeviceToHost));
  for (size_t m = 0; m < n; ++m)
    for (size_t q = 0; q < n; ++q) {  // row-major device -> column-major caller
      Z[2 * (m + q * n)] = h[m * n + q].x;
      Z[2 * (m + q * n) + 1] = h[m * n + q].y;
    }
  if (mmax_out) *mmax_out = tabs[0].mmax;
  return 0;
}

int pss_modal_tables(pss_ctx *c, int magnetic, int nl, const double *eps, const double *mu, const double *width,
                     int s, double k0, double u, double psi1, double psi2, const double *b1, const double *b2,
                     double convtest, int64_t cap, double *t1, double *t2, int *mmax_out, int *status) {
  if (!c || !t1 || !t2 || !mmax_out) { pss_set_error("null argument"); return -1; }
  if (set_device(c)) return -3;
  StackParams S;
  if (make_stack(nl, eps, mu, width, s, S)) return -1;
  PointParams P;
  make_params(magnetic, S, b1, b2, u, k0, psi1, psi2, P);
  if (upload(c->params, &P, 1)) return -3;
  std::vector<int> hs(1, 0);
  std::vector<TableDev> tabs;
  int rc = build_tables(c, S, c->params.as<PointParams>(), 1, convtest, tabs, hs);
  if (rc) return rc;
  size_t need = pss_table_cap(tabs[0].mmax);
  *mmax_out = tabs[0].mmax;
  if (status) *status = hs[0];
  if ((int64_t)need > cap) { pss_set_error("table capacity %lld < %zu", (long long)cap, need); return -2; }
  PSS_CUDA_TRY(cudaMemcpy(t1, tabs[0].t1, need * sizeof(cd), cudaMemcpyDeviceToHost));
  PSS_CUDA_TRY(cudaMemcpy(t2, tabs[0].t2, need * sizeof(cd), cudaMemcpyDeviceToHost));
  return 0;
}

int pss_face_integrals(pss_sheet *sh, double ulocal, double psi1, double psi2, double *J, double *Jxi,
                       double *Jeta, double *K, double *Kxi, double *Keta, double *rho_r, double *rinv,
                       int *nonconv) {
  if (!sh) { pss_set_error("null argument"); return -1; }
  if (set_device(sh->ctx)) return -3;
  sh->jk_valid = false;
  int rc = refresh_jk_cache(sh, psi1, psi2, ulocal, sh->ctx->w[0].st);
  if (rc) return rc;
  const size_t c = (size_t)sh->nufp * sizeof(cd), d = (size_t)sh->nufp * sizeof(double);
  const JKDev &jk = sh->cache.jk;
  PSS_CUDA_TRY(cudaMemcpy(J, jk.J, c, cudaMemcpyDeviceToHost));
  PSS_CUDA_TRY(cudaMemcpy(Jxi, jk.Jxi, c, cudaMemcpyDeviceToHost));
  PSS_CUDA_TRY(cudaMemcpy(Jeta, jk.Jeta, c, cudaMemcpyDeviceToHost));
  PSS_CUDA_TRY(cudaMemcpy(K, jk.K, c, cudaMemcpyDeviceToHost));
  PSS_CUDA_TRY(cudaMemcpy(Kxi, jk.Kxi, c, cudaMemcpyDeviceToHost));
  PSS_CUDA_TRY(cudaMemcpy(Keta, jk.Keta, c, cudaMemcpyDeviceToHost));
  PSS_CUDA_TRY(cudaMemcpy(rho_r, jk.rho_r, 2 * d, cudaMemcpyDeviceToHost));
  PSS_CUDA_TRY(cudaMemcpy(rinv, jk.rinv, d, cudaMemcpyDeviceToHost));
  if (nonconv) *nonconv = sh->jk_nonconv;
  return 0;
}

int pss_basis_transforms(pss_sheet *sh, int nmodes, const double *kvec, double psi1, double psi2, double *F) {
  if (!sh || !kvec || !F || nmodes <= 0) { pss_set_error("invalid argument"); return -1; }
  pss_ctx *c = sh->ctx;
  if (set_device(c)) return -3;
  Worker &w = c->w[0];
  LocalBuf kb;
  if (upload(kb, kvec, 2 * (size_t)nmodes)) return -3;
  if (w.bf.ensure((size_t)nmodes * sh->nbf * 2 * sizeof(cd))) return -3;
  pss_bfft(sh->G, nmodes, kb.as<double>(), psi1, psi2, w.bf.as<cd>(), w.st);
  PSS_CUDA_TRY(cudaStreamSynchronize(w.st));
  PSS_CUDA_TRY(cudaMemcpy(F, w.bf.p, (size_t)nmodes * sh->nbf * 2 * sizeof(cd), cudaMemcpyDeviceToHost));
  kb.release();
  return 0;
}

int pss_lu_solve(pss_ctx *c, int n, const double *Z, int nrhs, const double *B, int precision, double *X,
                 int *status) {
  if (!c || !Z || !B || !X || n <= 0 || nrhs <= 0) { pss_set_error("invalid argument"); return -1; }
  if (set_device(c)) return -3;
  Worker &w = c->w[0];
  cudaStream_t st = w.st;
  const size_t nn = (size_t)n * n;
  std::vector<cd> h(nn);
  for (size_t m = 0; m < (size_t)n; ++m)
    for (size_t q = 0; q < (size_t)n; ++q) h[m * n + q] = mkcd(Z[2 * (m + q * n)], Z[2 * (m + q * n) + 1]);
  if (w.z64.ensure(nn * sizeof(cd)) || w.ensure_solver(n, nrhs, 1)) return -3;
  DevBuf st_buf;
  if (st_buf.ensure(sizeof(int))) return -3;
  PSS_CUDA_TRY(cudaMemset(st_buf.p, 0, sizeof(int)));
  PSS_CUDA_TRY(cudaMemset(w.info.p, 0, sizeof(int)));
  PSS_CUDA_TRY(cudaMemcpy(w.z64.p, h.data(), nn * sizeof(cd), cudaMemcpyHostToDevice));
  PSS_CUDA_TRY(cudaMemcpy(w.rhs.p, B, (size_t)n * nrhs * sizeof(cd), cudaMemcpyHostToDevice));
  int rc;
  if (precision == PSS_FP32_REFINE) {
    const size_t ldf = (size_t)Worker::ld32(n), nf = (size_t)n * ldf;
    if (w.zr.ensure(nf * sizeof(float)) || w.zi.ensure(nf * sizeof(float))) return -3;
    std::vector<float> hr(nf, 0.f), hi(nf, 0.f);
    for (size_t m = 0; m < (size_t)n; ++m)
      for (size_t q = 0; q < (size_t)n; ++q) {
        hr[m * ldf + q] = (float)h[m * n + q].x;
        hi[m * ldf + q] = (float)h[m * n + q].y;
      }
    PSS_CUDA_TRY(cudaMemcpy(w.zr.p, hr.data(), nf * sizeof(float), cudaMemcpyHostToDevice));
    PSS_CUDA_TRY(cudaMemcpy(w.zi.p, hi.data(), nf * sizeof(float), cudaMemcpyHostToDevice));
  }
  if ((rc = w.factor_solve(n, 1, precision, nrhs, kMaxRefine, st_buf.as<int>()))) return rc;
  PSS_CUDA_TRY(cudaStreamSynchronize(st));
  PSS_CUDA_TRY(cudaGetLastError());
  int hs = 0;
  PSS_CUDA_TRY(cudaMemcpy(&hs, st_buf.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (precision == PSS_FP32_REFINE && (hs & (PSS_ST_REFINE_NOCONV | PSS_ST_NONFINITE))) {
    // stalled refinement: FP64 factorisation of the original matrix
    PSS_CUDA_TRY(cudaMemset(st_buf.p, 0, sizeof(int)));
    PSS_CUDA_TRY(cudaMemcpy(w.z64.p, h.data(), nn * sizeof(cd), cudaMemcpyHostToDevice));
    if ((rc = w.factor_solve(n, 1, PSS_FP64, nrhs, 0, st_buf.as<int>()))) return rc;
    PSS_CUDA_TRY(cudaStreamSynchronize(st));
    PSS_CUDA_TRY(cudaMemcpy(&hs, st_buf.p, sizeof(int), cudaMemcpyDeviceToHost));
    hs |= PSS_ST_FP64_FALLBACK;
  }
  PSS_CUDA_TRY(cudaMemcpy(X, w.X.p, (size_t)n * nrhs * sizeof(cd), cudaMemcpyDeviceToHost));
  if (status) *status = hs;
  st_buf.release();
  return 0;
}

int pss_lu32_factor(pss_ctx *c, int n, const double *Z, float *LU, int *ipiv, int *info) {
  if (!c || !Z || !LU || !ipiv || !info || n <= 0) { pss_set_error("invalid argument"); return -1; }
  if (set_device(c)) return -3;
  Worker &w = c->w[0];
  cudaStream_t st = w.st;
  const size_t ldf = (size_t)Worker::ld32(n), nf = (size_t)n * ldf;
  if (w.ensure_solver(n, 1, 1) || w.zr.ensure(nf * sizeof(float)) || w.zi.ensure(nf * sizeof(float))) return -3;
  std::vector<float> hr(nf, 0.f), hi(nf, 0.f);  // row-major planes, row pitch ldf
  for (size_t m = 0; m < (size_t)n; ++m)
    for (size_t q = 0; q < (size_t)n; ++q) {
      hr[m * ldf + q] = (float)Z[2 * (m + q * n)];
      hi[m * ldf + q] = (float)Z[2 * (m + q * n) + 1];
    }
  PSS_CUDA_TRY(cudaMemcpy(w.zr.p, hr.data(), nf * sizeof(float), cudaMemcpyHostToDevice));
  PSS_CUDA_TRY(cudaMemcpy(w.zi.p, hi.data(), nf * sizeof(float), cudaMemcpyHostToDevice));
  PSS_CUDA_TRY(cudaMemsetAsync(w.info.p, 0, sizeof(int), st));
  if (int rc = pss_lu32_batched(n, 1, w.zr.as<float>(), w.zi.as<float>(), (long long)ldf, (long long)nf,
                                w.ipiv.as<int>(), w.info.as<int>(), w.luws.p, w.luws.n, st))
    return rc;
  PSS_CUDA_TRY(cudaStreamSynchronize(st));
  PSS_CUDA_TRY(cudaGetLastError());
  PSS_CUDA_TRY(cudaMemcpy(hr.data(), w.zr.p, nf * sizeof(float), cudaMemcpyDeviceToHost));
  PSS_CUDA_TRY(cudaMemcpy(hi.data(), w.zi.p, nf * sizeof(float), cudaMemcpyDeviceToHost));
  std::vector<int> hp(n);
  PSS_CUDA_TRY(cudaMemcpy(hp.data(), w.ipiv.p, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost));
  PSS_CUDA_TRY(cudaMemcpy(info, w.info.p, sizeof(int), cudaMemcpyDeviceToHost));
  PSS_CUDA_TRY(cudaMemset(w.info.p, 0, sizeof(int)));
  for (size_t m = 0; m < (size_t)n; ++m)
    for (size_t q = 0; q < (size_t)n; ++q) {
      LU[2 * (m + q * n)] = hr[m * ldf + q];
      LU[2 * (m + q * n) + 1] = hi[m * ldf + q];
    }
  for (int j = 0; j < n; ++j) ipiv[j] = hp[j] + 1;
  return 0;
}

int pss_schur_update(pss_ctx *c, int m, int n, int k, const float *Lr, const float *Li, const float *Ur,
                     const float *Ui, float *Cr, float *Ci, int *status) {
  if (!c || !Lr || !Li || !Ur || !Ui || !Cr || !Ci || m <= 0 || n <= 0 || k <= 0) {
    pss_set_error("invalid argument");
    return -1;
  }
  if (set_device(c)) return -3;
  Worker &w = c->w[0];
  cudaStream_t st = w.st;
  // One (k + m) x (k + n) row-major matrix: U top right, L bottom left, C bottom right.
  const long long ld = k + n, rows = k + m;
  const size_t total = (size_t)rows * ld;
  std::vector<float> hr(total, 0.f), hi(total, 0.f);
  for (long long r = 0; r < k; ++r)
    for (long long q = 0; q < n; ++q) { hr[r * ld + k + q] = Ur[r * n + q]; hi[r * ld + k + q] = Ui[r * n + q]; }
  for (long long r = 0; r < m; ++r) {
    for (long long q = 0; q < k; ++q) { hr[(k + r) * ld + q] = Lr[r * k + q]; hi[(k + r) * ld + q] = Li[r * k + q]; }
    for (long long q = 0; q < n; ++q) {
      hr[(k + r) * ld + k + q] = Cr[r * n + q];
      hi[(k + r) * ld + k + q] = Ci[r * n + q];
    }
  }
  const size_t tcb = pss_tc_ws_bytes(m, n, (k + 15) / 16 * 16);
  LocalBuf ar, ai, ws, err;
  if (ar.ensure(total * sizeof(float)) || ai.ensure(total * sizeof(float)) || ws.ensure(tcb) ||
      err.ensure(sizeof(int)))
    return -3;
  PSS_CUDA_TRY(cudaMemcpyAsync(ar.p, hr.data(), total * sizeof(float), cudaMemcpyHostToDevice, st));
  PSS_CUDA_TRY(cudaMemcpyAsync(ai.p, hi.data(), total * sizeof(float), cudaMemcpyHostToDevice, st));
  PSS_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(int), st));
  int rc = pss_cgemm_tc(ar.as<float>(), ai.as<float>(), ld, 0, 1, k, m, k, n, 0, k, ws.p, ws.n, err.as<int>(), st);
  if (rc) return rc;
  PSS_CUDA_TRY(cudaMemcpyAsync(hr.data(), ar.p, total * sizeof(float), cudaMemcpyDeviceToHost, st));
  PSS_CUDA_TRY(cudaMemcpyAsync(hi.data(), ai.p, total * sizeof(float), cudaMemcpyDeviceToHost, st));
  int herr = 0;
  PSS_CUDA_TRY(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  PSS_CUDA_TRY(cudaStreamSynchronize(st));
  for (long long r = 0; r < m; ++r)
    for (long long q = 0; q < n; ++q) {
      Cr[r * n + q] = hr[(k + r) * ld + k + q];
      Ci[r * n + q] = hi[(k + r) * ld + k + q];
    }
  if (status) *status = herr ? PSS_ST_DEVICE_TIMEOUT : 0;
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Linearised partial GSMs for gradients with one factorisation per point.  For each perturbed
// input set k (another sheet of the same topology, other layers, smoothing parameter, modes):
//     dS_k = wobs_k o (P_k Z^-1 R_k + P Z^-1 (R - Z_k X)),   X = Z^-1 R,
// the first-order value of the perturbed partial GSM from the factors of Z, so that central
// differences of dS_k give dS/dp to O(h^2).  Forward solves only: R_k are extra right-hand
// sides of the first solve, R - Z_k X those of a second solve on the same factors.
namespace {

// Y[:, j] = B[:, j] - A X[:, j] for row-major A (n x n, row stride ld): one warp per row.
__global__ void k_lin_resid(int n, int nrhs, const cd *__restrict__ A, long long ld, const cd *__restrict__ X,
                            const cd *__restrict__ B, cd *__restrict__ Y) {
  const int row = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (row >= n) return;  // uniform per warp
  const cd *a = A + (long long)row * ld;
  for (int j = 0; j < nrhs; ++j) {
    const cd *x = X + (long long)j * n;
    double sr = 0.0, si = 0.0;
    for (int c = lane; c < n; c += 32) {
      const cd p = a[c] * x[c];
      sr += p.x;
      si += p.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, o);
      si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane == 0) Y[(long long)j * n + row] = B[(long long)j * n + row] - mkcd(sr, si);
  }
}

// The tables of one point, copied out of the context's table buffers (which the next
// build_tables call reuses).
int point_tables(pss_ctx *c, const StackParams &S, const PointParams *dP, DevBuf &own, TableDev &t, int &hstat) {
  std::vector<TableDev> tabs;
  std::vector<int> hs(1, 0);
  if (int rc = build_tables(c, S, dP, 1, 1e-7, tabs, hs)) return rc;
  const size_t used = (size_t)(tabs[0].mmax + 2) * (tabs[0].mmax + 2);
  if (own.ensure(2 * used * sizeof(cd))) return -3;
  cudaStream_t st = c->w[0].st;
  PSS_CUDA_TRY(cudaMemcpyAsync(own.p, tabs[0].t1, used * sizeof(cd), cudaMemcpyDeviceToDevice, st));
  PSS_CUDA_TRY(cudaMemcpyAsync(own.as<cd>() + used, tabs[0].t2, used * sizeof(cd), cudaMemcpyDeviceToDevice, st));
  t.t1 = own.as<cd>();
  t.t2 = own.as<cd>() + used;
  t.mmax = tabs[0].mmax;
  hstat |= hs[0];
  return 0;
}

}  // namespace

extern "C" int pss_partial_gsms_lin(pss_sheet *sh, int nl, const double *eps, const double *mu, const double *width,
                                    int s, double u, int npts, const double *k0, const double *psi, int nmodes,
                                    const double *kvec, const double *src, const double *tobs, const double *wobs,
                                    int npert, pss_sheet *const *psh, const double *peps, const double *pmu,
                                    const double *pwidth, const double *pu, const double *ppsi, const double *pkvec,
                                    const double *psrc, const double *ptobs, const double *pwobs, int precision,
                                    double *dS, double *dSp, int *status) {
  if (!sh || !k0 || !psi || !dS || !status || !kvec || !src || !tobs || !wobs) {
    pss_set_error("null argument");
    return -1;
  }
  if (npts <= 0 || nmodes <= 0 || nmodes > 4096 || npert < 0 || npert > 64) {
    pss_set_error("invalid npts/nmodes/npert");
    return -1;
  }
  if (npert > 0 && (!psh || !peps || !pmu || !pwidth || !pu || !ppsi || !pkvec || !psrc || !ptobs || !pwobs || !dSp)) {
    pss_set_error("null perturbation argument");
    return -1;
  }
  if (precision != PSS_FP64 && precision != PSS_FP32_REFINE) { pss_set_error("unknown precision %d", precision); return -1; }
  for (int k = 0; k < npert; ++k)
    if (!psh[k] || psh[k]->ctx != sh->ctx || psh[k]->nbf != sh->nbf || psh[k]->cls != sh->cls) {
      pss_set_error("perturbed sheet %d is not a sheet of the same context, class and basis count", k);
      return -1;
    }
  if (!(u > 0)) { pss_set_error("smoothing parameter u must be positive"); return -1; }
  pss_ctx *c = sh->ctx;
  if (set_device(c)) return -3;
  const int magnetic = sh->cls == 'M';
  const int n = sh->nbf, nm = nmodes, K = npert;
  const long long ld = n, msz = (long long)n * n;
  StackParams S;
  if (make_stack(nl, eps, mu, width, s, S)) return -1;
  std::vector<StackParams> Sk(K);
  for (int k = 0; k < K; ++k) {
    if (make_stack(nl, peps + 2 * (size_t)k * nl, pmu + 2 * (size_t)k * nl, pwidth + (size_t)k * nl, s, Sk[k]))
      return -1;
    if (!(pu[k] > 0)) { pss_set_error("perturbed smoothing parameter %d must be positive", k); return -1; }
  }
  Worker &w = c->w[0];
  cudaStream_t st = w.st;
  const int nrhs1 = nm * (1 + K), nrhs2 = nm * K;
  int rc = ensure_worker(w, sh, nm, precision, false, 1 + K);
  if (rc) return rc;
  if ((rc = w.ensure_solver(n, std::max(nrhs1, 1), 1 + K))) return rc;
  int maxufp = sh->nufp;
  for (int k = 0; k < K; ++k) maxufp = std::max(maxufp, psh[k]->nufp);
  if (w.zb.ensure((size_t)maxufp * 9 * sizeof(cd))) return -3;
  LocalBuf pbuf, tb0, mbuf, Ybuf, Wbuf, out;
  std::vector<LocalBuf> tbk(K);
  if (pbuf.ensure((size_t)(1 + K) * sizeof(PointParams)) ||
      mbuf.ensure((size_t)(1 + K) * nm * (2 * sizeof(double) + 2 * sizeof(cd) + 2 * sizeof(double) + sizeof(cd))) ||
      Ybuf.ensure((size_t)n * std::max(nrhs2, 1) * sizeof(cd)) || Wbuf.ensure((size_t)n * std::max(nrhs2, 1) * sizeof(cd)) ||
      out.ensure((size_t)(1 + 2 * K) * nm * nm * sizeof(cd)))
    return -3;
  const size_t nmk = (size_t)nm * 2;  // doubles of one mode set's kvec / tobs; cd of its src
  // per mode set q (0 = unperturbed, k + 1 = perturbation k): kvec, src, tobs, wobs
  char *mb = mbuf.as<char>();
  auto kv_of = [&](int q) { return (double *)mb + (size_t)q * nmk; };
  auto src_of = [&](int q) { return (cd *)(mb + (size_t)(1 + K) * nmk * sizeof(double)) + (size_t)q * nmk; };
  auto tob_of = [&](int q) {
    return (double *)(mb + (size_t)(1 + K) * nmk * (sizeof(double) + sizeof(cd))) + (size_t)q * nmk;
  };
  auto wob_of = [&](int q) {
    return (cd *)(mb + (size_t)(1 + K) * nmk * (2 * sizeof(double) + sizeof(cd))) + (size_t)q * nm;
  };
  std::vector<cd> hdS((size_t)(1 + 2 * K) * nm * nm);
  float *zr = precision == PSS_FP32_REFINE ? w.zr.as<float>() : nullptr;
  float *zi = precision == PSS_FP32_REFINE ? w.zi.as<float>() : nullptr;
  const cd *L64 = precision == PSS_FP64 ? w.z64.as<cd>() : nullptr;
  for (int i = 0; i < npts; ++i) {
    if (!(k0[i] > 0) || !std::isfinite(psi[2 * i]) || !std::isfinite(psi[2 * i + 1])) {
      pss_set_error("invalid k0/psi at point %d", i);
      return -1;
    }
    int hst = 0;
    // point parameters and mode data of every set
    std::vector<PointParams> hP(1 + K);
    {
      const double b1m[2] = {sh->b1[0] * sh->upm, sh->b1[1] * sh->upm};
      const double b2m[2] = {sh->b2[0] * sh->upm, sh->b2[1] * sh->upm};
      make_params(magnetic, S, b1m, b2m, u, k0[i], psi[2 * i], psi[2 * i + 1], hP[0]);
    }
    for (int k = 0; k < K; ++k) {
      const pss_sheet *q = psh[k];
      const double b1m[2] = {q->b1[0] * q->upm, q->b1[1] * q->upm};
      const double b2m[2] = {q->b2[0] * q->upm, q->b2[1] * q->upm};
      const double *pp = ppsi + 2 * ((size_t)k * npts + i);
      make_params(magnetic, Sk[k], b1m, b2m, pu[k], k0[i], pp[0], pp[1], hP[1 + k]);
    }
    PSS_CUDA_TRY(cudaMemcpy(pbuf.p, hP.data(), hP.size() * sizeof(PointParams), cudaMemcpyHostToDevice));
    const PointParams *dP = pbuf.as<PointParams>();
    for (int q = 0; q <= K; ++q) {
      const size_t off = q == 0 ? (size_t)i * nm : ((size_t)(q - 1) * npts + i) * nm;
      const double *kv = q == 0 ? kvec : pkvec;
      const double *sv = q == 0 ? src : psrc;
      const double *tv = q == 0 ? tobs : ptobs;
      const double *wv = q == 0 ? wobs : pwobs;
      PSS_CUDA_TRY(cudaMemcpy(kv_of(q), kv + 2 * off, nm * 2 * sizeof(double), cudaMemcpyHostToDevice));
      PSS_CUDA_TRY(cudaMemcpy(src_of(q), sv + 4 * off, nm * 2 * sizeof(cd), cudaMemcpyHostToDevice));
      PSS_CUDA_TRY(cudaMemcpy(tob_of(q), tv + 2 * off, nm * 2 * sizeof(double), cudaMemcpyHostToDevice));
      PSS_CUDA_TRY(cudaMemcpy(wob_of(q), wv + 2 * off, nm * sizeof(cd), cudaMemcpyHostToDevice));
    }
    // tables and face-pair integrals of every set
    TableDev t0;
    std::vector<TableDev> tk(K);
    if ((rc = point_tables(c, S, dP, tb0, t0, hst))) return rc;
    for (int k = 0; k < K; ++k)
      if ((rc = point_tables(c, Sk[k], dP + 1 + k, tbk[k], tk[k], hst))) return rc;
    if ((rc = refresh_jk_cache(sh, psi[2 * i], psi[2 * i + 1], u / sh->upm, st))) return rc;
    if (sh->jk_nonconv) hst |= PSS_ST_JK_NOCONV;
    // Z into slot 0 (and the FP32 planes), fills and transforms of every set
    pss_fill_pairs(sh->G, dP, sh->cache.jk, t0.t1, t0.t2, t0.mmax, w.zb.as<cd>(), st);
    pss_fill_assemble(sh->G, dP, w.zb.as<cd>(), w.z64.as<cd>(), zr, zi, ld, Worker::ld32(n), st);
    cd *bf = w.bf.as<cd>();
    const size_t bfs = (size_t)nm * n * 2;
    pss_bfft(sh->G, nm, kv_of(0), psi[2 * i], psi[2 * i + 1], bf, st);
    pss_rhs(n, nm, bf, src_of(0), w.rhs.as<cd>(), st);
    for (int k = 0; k < K; ++k) {
      pss_sheet *q = psh[k];
      const double *pp = ppsi + 2 * ((size_t)k * npts + i);
      if ((rc = refresh_jk_cache(q, pp[0], pp[1], pu[k] / q->upm, st))) return rc;
      if (q->jk_nonconv) hst |= PSS_ST_JK_NOCONV;
      pss_fill_pairs(q->G, dP + 1 + k, q->cache.jk, tk[k].t1, tk[k].t2, tk[k].mmax, w.zb.as<cd>(), st);
      pss_fill_assemble(q->G, dP + 1 + k, w.zb.as<cd>(), w.z64.as<cd>() + (1 + k) * msz, nullptr, nullptr, ld, ld,
                        st);
      pss_bfft(q->G, nm, kv_of(1 + k), pp[0], pp[1], bf + (1 + k) * bfs, st);
      pss_rhs(n, nm, bf + (1 + k) * bfs, src_of(1 + k), w.rhs.as<cd>() + (size_t)(1 + k) * nm * n, st);
    }
    // one factorisation; solves of R and every R_k
    PSS_CUDA_TRY(cudaMemsetAsync(w.bstat.p, 0, sizeof(int), st));
    if ((rc = w.factor_solve(n, 1, precision, nrhs1, kMaxRefine, w.bstat.as<int>()))) return rc;
    // R - Z_k X (slot k + 1), then its solve on the same factors
    cd *X = w.X.as<cd>();
    for (int k = 0; k < K; ++k) {
      pss_count_launch();
      k_lin_resid<<<cdiv_u((long long)n * 32, 256), 256, 0, st>>>(n, nm, w.z64.as<cd>() + (1 + k) * msz, ld, X,
                                                                   w.rhs.as<cd>(), Ybuf.as<cd>() + (size_t)k * nm * n);
    }
    if (K > 0) {
      const long long vs2 = (long long)n * nrhs2;
      const long long fld = L64 ? ld : Worker::ld32(n), fms = (long long)n * fld;
      if ((rc = pss_solve_lu(w.sws, 1, L64, zr, zi, fld, fms, nrhs2, Ybuf.as<cd>(), Wbuf.as<cd>(), vs2, 0, st)))
        return rc;
      if (precision == PSS_FP32_REFINE &&
          (rc = pss_refine(w.sws, 1, w.z64.as<cd>(), ld, msz, zr, zi, fld, fms, nrhs2, Ybuf.as<cd>(), Wbuf.as<cd>(),
                           w.R.as<cd>(), w.D.as<cd>(), vs2, kMaxRefine, w.bstat.as<int>(), st)))
        return rc;
      pss_solve_status(w.sws, 1, w.bstat.as<int>(), st);
    }
    // projections: dS; P_k X_k' and P W_k for every k
    cd *o = out.as<cd>();
    const size_t nm2 = (size_t)nm * nm;
    pss_project(n, nm, bf, tob_of(0), wob_of(0), X, o, st);
    for (int k = 0; k < K; ++k) {
      pss_project(n, nm, bf + (1 + k) * bfs, tob_of(1 + k), wob_of(1 + k), X + (size_t)(1 + k) * nm * n,
                  o + (1 + 2 * k) * nm2, st);
      pss_project(n, nm, bf, tob_of(0), wob_of(1 + k), Wbuf.as<cd>() + (size_t)k * nm * n, o + (2 + 2 * k) * nm2, st);
    }
    int bst = 0;
    PSS_CUDA_TRY(cudaMemcpyAsync(hdS.data(), o, hdS.size() * sizeof(cd), cudaMemcpyDeviceToHost, st));
    PSS_CUDA_TRY(cudaMemcpyAsync(&bst, w.bstat.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    PSS_CUDA_TRY(cudaStreamSynchronize(st));
    status[i] = hst | bst;
    for (size_t e = 0; e < nm2; ++e) {
      dS[2 * ((size_t)i * nm2 + e)] = hdS[e].x;
      dS[2 * ((size_t)i * nm2 + e) + 1] = hdS[e].y;
    }
    for (int k = 0; k < K; ++k)
      for (size_t e = 0; e < nm2; ++e) {
        const cd v = hdS[(1 + 2 * k) * nm2 + e] + hdS[(2 + 2 * k) * nm2 + e];
        const size_t d = ((size_t)k * npts + i) * nm2 + e;
        dSp[2 * d] = v.x;
        dSp[2 * d + 1] = v.y;
      }
  }
  return 0;
}

// Adjoint form of the linearised partial GSMs (same inputs and outputs as
// pss_partial_gsms_lin):  dSp[k] = wobs_k o (P_k X + Lam^T (R_k - Z_k X)),  X = Z^-1 R,
// Lam = Z^-T P^T.  The points are swept as pss_partial_gsms sweeps them (batched fills and
// factorisations on the worker streams), the perturbed sets riding along as extra problems
// whose tables, face integrals and mode data are prepared with the sweep; after each batched
// factorisation the adjoint solves run on the same factors, and each perturbed set costs its
// pair terms (Green's-function table interpolations recomputed for the set), its basis
// transforms and one fused assemble-and-contract pass (pss_adj_contract) - no perturbed
// matrix is stored and no further solve is taken.
extern "C" int pss_partial_gsms_adj(pss_sheet *sh, int nl, const double *eps, const double *mu, const double *width,
                                    int s, double u, int npts, const double *k0, const double *psi, int nmodes,
                                    const double *kvec, const double *src, const double *tobs, const double *wobs,
                                    int npert, pss_sheet *const *psh, const double *peps, const double *pmu,
                                    const double *pwidth, const double *pu, const double *ppsi, const double *pkvec,
                                    const double *psrc, const double *ptobs, const double *pwobs, int precision,
                                    double *dS, double *dSp, int *status) {
  if (!sh || !k0 || !psi || !dS || !status || !kvec || !src || !tobs || !wobs) {
    pss_set_error("null argument");
    return -1;
  }
  if (npts <= 0 || nmodes <= 0 || nmodes > 1024 || npert < 0 || npert > 64) {
    pss_set_error("invalid npts/nmodes/npert");
    return -1;
  }
  if (npert > 0 && (!psh || !peps || !pmu || !pwidth || !pu || !ppsi || !pkvec || !psrc || !ptobs || !pwobs || !dSp)) {
    pss_set_error("null perturbation argument");
    return -1;
  }
  for (int k = 0; k < npert; ++k)
    if (!psh[k] || psh[k]->ctx != sh->ctx || psh[k]->nbf != sh->nbf || psh[k]->cls != sh->cls) {
      pss_set_error("perturbed sheet %d is not a sheet of the same context, class and basis count", k);
      return -1;
    }
  const int K = npert, nm = nmodes;
  const size_t nm2 = (size_t)nm * nm, per = (size_t)npts * nm;
  std::vector<Problem> PR(1 + K);
  pss_problem q0{sh, nl, eps, mu, width, s, u, npts, k0, psi, nmodes, kvec, src, tobs, wobs, 0, 0, 0, dS, status};
  if (int rc = check_problem(q0, precision, PR[0])) return rc;
  // the perturbed sets' own dS and status are not produced (they take no solve): scratch
  std::vector<double> kdS((size_t)std::max(K, 1) * npts * nm2 * 2);
  std::vector<int> kst((size_t)std::max(K, 1) * npts);
  for (int k = 0; k < K; ++k) {
    pss_problem qk{psh[k], nl, peps + 2 * (size_t)k * nl, pmu + 2 * (size_t)k * nl, pwidth + (size_t)k * nl, s,
                   pu[k], npts, k0, ppsi + 2 * (size_t)k * npts, nmodes, pkvec + 2 * k * per, psrc + 4 * k * per,
                   ptobs + 2 * k * per, pwobs + 2 * k * per, 0, 0, 0, kdS.data() + (size_t)k * npts * nm2 * 2,
                   kst.data() + (size_t)k * npts};
    if (int rc = check_problem(qk, precision, PR[1 + k])) {
      const std::string m = pss_last_error();
      pss_set_error("perturbed set %d: %s", k, m.c_str());
      return rc;
    }
  }
  pss_ctx *c = sh->ctx;
  if (set_device(c)) return -3;
  LocalBuf dbuf;
  if (dbuf.ensure(2 * std::max<size_t>((size_t)K * npts * nm2, 1) * sizeof(cd))) return -3;
  AdjSpec adj{K, dbuf.as<cd>(), dbuf.as<cd>() + std::max<size_t>((size_t)K * npts * nm2, 1)};
  if (int rc = sweep_impl(c, PR, precision, &adj)) return rc;
  if (K > 0) {
    std::vector<cd> hP((size_t)K * npts * nm2), hG((size_t)K * npts * nm2);
    PSS_CUDA_TRY(cudaMemcpy(hP.data(), adj.dSp, hP.size() * sizeof(cd), cudaMemcpyDeviceToHost));
    PSS_CUDA_TRY(cudaMemcpy(hG.data(), adj.G, hG.size() * sizeof(cd), cudaMemcpyDeviceToHost));
    for (int k = 0; k < K; ++k)
      for (int i = 0; i < npts; ++i) {
        const double *wk = pwobs + 2 * (k * per + (size_t)i * nm);
        for (size_t e = 0; e < nm2; ++e) {
          const size_t a = e % nm, d = ((size_t)k * npts + i) * nm2 + e;  // a: observation mode (row)
          const cd v = hP[d] + mkcd(wk[2 * a], wk[2 * a + 1]) * hG[d];
          dSp[2 * d] = v.x;
          dSp[2 * d + 1] = v.y;
        }
        status[i] |= kst[(size_t)k * npts + i];  // the sets' table / face-integral flags
      }
  }
  return 0;
}
