// K2 + K3: face-pair integrals and the MoM matrix fill.
//
// K2 k_filljk   restates Zint.jl:54-179 (filljk!) with PGF.jl:67-106 (jksums): eight
//               lanes per unique face pair, one lattice sum (quadrature point) per lane in
//               the reference's ring order, the seven sums gathered by warp shuffles and
//               accumulated in the 7-point rule's order, FP64.
// K3a k_pairs   restates Zint.jl:218-245 (zint) and the per-edge algebra of
//               FillZY.jl:141-197 / 362-419: one thread per unique face pair computes
//               the 3x3 unflagged edge-pair terms  zA*(ρc2[iml]·a_isl) - zP*φ.
// K3b k_assemble replaces the spin-locked scatter of FillZY.jl:160-239 by a gather:
//               each Z entry sums, in a fixed order, the <=2x2 face incidences of its
//               test and source basis functions, applying the Floquet/sign flags and the
//               surface-resistance terms of Eqs. 7-34/7-35 (FillZY.jl:221-230).
//               Deterministic, atomic-free; writes FP64 and/or split FP32 planes.
#include <algorithm>

#include "pss_internal.cuh"

namespace {

// Phase factors of the lattice terms, cis(-m psi1) and cis(-n psi2) for |m|, |n| <= 65 (the
// ring budget): kPhase entries each, index m + 65.  A term's factor cis(-(m psi1 + n psi2)) is
// their product, one complex multiply in place of a sincos per summand.
constexpr int kPhase = 2 * PSS_JKRINGMAX + 1;

// exp(-a), a >= 0, by Tang's table-driven method (P. T. P. Tang, "Table-driven implementation
// of the exponential function in IEEE floating-point arithmetic", ACM Trans. Math. Softw. 15
// (1989) 144-157): -a = (256 m + j) ln2/256 + r with |r| <= ln2/512 (k = 256 m + j the nearest
// integer to -a 256/ln2, found by adding 1.5 * 2^52; ln2/256 in two parts, so r keeps its full
// precision), exp(-a) = 2^m * 2^(j/256) * p(r) with p the degree-5 Taylor polynomial of e^r
// (remainder below r^6/720 < 1e-20 relative) and 2^(j/256) from a 256-entry table; 2^m enters
// through the exponent field.  About ten FP64 operations.  a >= 708 gives 0: such summands are
// far below the lattice sums' 1e-8 convergence test.
constexpr double kExpShift = 6755399441055744.0;  // 1.5 * 2^52
constexpr double kExpInvStep = 0x1.71547652b82fep+8;  // 256 / ln2
constexpr double kExpStepHi = 0x1.62e42fefa39efp-9;   // ln2 / 256, nearest double
constexpr double kExpStepLo = 0x1.abc9e3b39803fp-64;  // ln2 / 256 - kExpStepHi
__device__ __forceinline__ double exp_neg(double a, const double *__restrict__ tab) {
  if (!(a < 708.0)) return 0.0;
  const double sh = fma(-a, kExpInvStep, kExpShift);
  const int k = __double2loint(sh);  // nearest integer to -a 256/ln2, two's complement
  const double kf = sh - kExpShift;
  const double r = fma(kf, -kExpStepLo, fma(kf, -kExpStepHi, -a));
  double p = fma(r, 1.0 / 120, 1.0 / 24);
  p = fma(p, r, 1.0 / 6);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  const double t = tab[k & 255] * p;
  return __hiloint2double(__double2hiint(t) + ((k >> 8) << 20), __double2loint(t));
}

// jksums (PGF.jl:67-106): the spatial lattice sums J and K at one observation offset, ring by
// ring in the reference's order (rmin = 5, at most 65 rings, relative change 1e-8), for NP
// phasings at once.  A summand's distance, exp(-u r) and 1/r do not depend on the phasing, so
// they are evaluated once and weighted by each phasing's factor; every phasing keeps its own
// ring partials and stops accumulating at its own convergence ring, so its sums are those of
// a serial evaluation at that phasing alone, bit for bit.  Slots p >= np are idle.  Returns the
// mask of converged phasings.
template <int NP>
__device__ __forceinline__ unsigned jksums_group(double urx, double ury, int np, bool nophase, double us1x,
                                                 double us1y, double us2x, double us2y,
                                                 const cd (*__restrict__ ph1)[kPhase],
                                                 const cd (*__restrict__ ph2)[kPhase], const double *__restrict__ etab,
                                                 cd *jout, cd *kout) {
  const int rmin = 5;
  const double small = 1e-5, convtest = 1e-8;
  double arg = sqrt(urx * urx + ury * ury);
  double rterm = exp_neg(arg, etab);
  const cd k0 = mkcd(rterm, 0.0);
  const cd j0 = arg <= small ? mkcd((-arg / 6 + 0.5) * arg - 1, 0.0) : mkcd((rterm - 1) / arg, 0.0);
  cd jsum[NP], ksum[NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) { jsum[p] = j0; ksum[p] = k0; }
  unsigned live = (1u << np) - 1u, conv = 0;
  for (int r = 1; r <= PSS_JKRINGMAX && live; ++r) {
    cd jring[NP], kring[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) { jring[p] = mkcd(0, 0); kring[p] = mkcd(0, 0); }
    auto summand = [&](int m, int n, double dm, double dn) {
      double dx = urx - (dm * us1x + dn * us2x);
      double dy = ury - (dm * us1y + dn * us2y);
      // one reciprocal square root gives both the distance and the 1/r weight (two FP64
      // divisions fewer per summand than sqrt then term / r)
      const double d2 = dx * dx + dy * dy;
      const double ra = rsqrt(d2);
      const double a = d2 * ra;
      double er = exp_neg(a, etab);
      if (NP == 1 && nophase) {  // real terms: the imaginary parts stay exactly zero
        jring[0].x = jring[0].x + er * ra;
        kring[0].x = kring[0].x + er;
      } else {
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          const cd f = ph1[p][m + PSS_JKRINGMAX] * ph2[p][n + PSS_JKRINGMAX];
          const cd term = mkcd(er * f.x, er * f.y);
          jring[p] = jring[p] + mkcd(term.x * ra, term.y * ra);
          kring[p] = kring[p] + term;
        }
      }
    };
    // the ring's 8r lattice points in Ring's order (ring_mn): m = r with n = -r..r, m = -r with
    // n = -r..r, then n = -r and n = r with m = -r+1..r-1; the indices are also counted in
    // FP64 (exact integers), so no summand converts one
    {
      const double dr = (double)r;
      double dn = -dr;
      for (int i = -r; i <= r; ++i, dn += 1.0) summand(r, i, dr, dn);
      dn = -dr;
      for (int i = -r; i <= r; ++i, dn += 1.0) summand(-r, i, -dr, dn);
      double dm = 1.0 - dr;
      for (int i = 1 - r; i < r; ++i, dm += 1.0) summand(i, -r, dm, -dr);
      dm = 1.0 - dr;
      for (int i = 1 - r; i < r; ++i, dm += 1.0) summand(i, r, dm, dr);
    }
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      if (!((live >> p) & 1u)) continue;
      jsum[p] = jsum[p] + jring[p];
      ksum[p] = ksum[p] + kring[p];
      if (r > rmin) {
        double c1 = cabsd(jring[p] / jsum[p]), c2 = cabsd(kring[p] / ksum[p]);
        if (fmax(c1, c2) < convtest) { live &= ~(1u << p); conv |= 1u << p; }
      }
    }
  }
#pragma unroll
  for (int p = 0; p < NP; ++p) { jout[p] = jsum[p]; kout[p] = ksum[p]; }
  return conv;
}

__device__ __forceinline__ void face_vtx(const SheetDev &G, int f, double r[3][2], double scale) {
  for (int k = 0; k < 3; ++k) {
    int v = G.fv[3 * f + k];
    r[k][0] = G.rho[2 * v] * scale;
    r[k][1] = G.rho[2 * v + 1] * scale;
  }
}

// Eight lanes per unique face pair (four pairs per warp): lane q < 7 computes the lattice
// sums of quadrature point q (jksums, serial in the reference's ring order) for the group's
// np <= NP phasings; the pair's first lane gathers the seven results with warp shuffles and
// accumulates them in the 7-point rule's order, so each pair's integrals are those of a
// serial evaluation bit for bit.  The phasing-free parts (the smooth-term geometry, rho_r and
// the 1/R integral) are computed once and written to every phasing's slot.
template <int NP>
constexpr int jk_threads() { return NP == 1 ? 256 : 128; }

template <int NP>
__global__ void __launch_bounds__(jk_threads<NP>(), 3) k_filljk(SheetDev G, double ul, PsiGroup pg, double us1x, double us1y,
                                                double us2x, double us2y, JKGroup jk, int *nonconv) {
  __shared__ cd ph1[NP][kPhase], ph2[NP][kPhase];
  __shared__ double etab[256];  // 2^(j/256) for exp_neg
  for (int t = threadIdx.x; t < 256; t += blockDim.x) etab[t] = exp2((double)t / 256.0);
  const int np = NP == 1 ? 1 : pg.n;
  for (int t = threadIdx.x; t < NP * kPhase; t += blockDim.x) {
    const int p = t / kPhase;
    const double k = (double)(t % kPhase - PSS_JKRINGMAX);
    const double a1 = p < np ? pg.psi1[p] : 0.0, a2 = p < np ? pg.psi2[p] : 0.0;
    double s1, c1, s2, c2;
    sincos(-(k * a1), &s1, &c1);
    sincos(-(k * a2), &s2, &c2);
    ph1[p][t % kPhase] = mkcd(c1, s1);
    ph2[p][t % kPhase] = mkcd(c2, s2);
  }
  __syncthreads();
  const bool nophase = NP == 1 && pg.psi1[0] == 0.0 && pg.psi2[0] == 0.0;
  const int lane = threadIdx.x & 31, q = lane & 7, grp = lane & ~7;
  const long long gid = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 3;  // pair of this group
  const bool live = gid < G.nufp;
  const int iu = live ? (int)gid : G.nufp - 1;  // idle groups mirror the last pair, write nothing
  const int fp = G.ufp_rep[iu];
  const int ifm = fp % G.nface, ifs = fp / G.nface;
  double rs[3][2], rm[3][2];
  face_vtx(G, ifs, rs, 1.0);
  face_vtx(G, ifm, rm, 1.0);
  double rs32[2] = {rs[2][0] - rs[1][0], rs[2][1] - rs[1][1]};
  double rs12[2] = {rs[0][0] - rs[1][0], rs[0][1] - rs[1][1]};
  double area2 = (-rs32[1]) * rs12[0] + rs32[0] * rs12[1];
  double unz = 1.0;
  if (area2 < 0) { area2 = fabs(area2); unz = -1.0; }
  double rs31[2] = {rs[2][0] - rs[0][0], rs[2][1] - rs[0][1]};
  double rs21[2] = {-rs12[0], -rs12[1]};
  double rmc[2] = {((rm[0][0] + rm[1][0]) + rm[2][0]) / 3, ((rm[0][1] + rm[1][1]) + rm[2][1]) / 3};
  cd js[NP], ks[NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) { js[p] = mkcd(0, 0); ks[p] = mkcd(0, 0); }
  unsigned ok = (1u << np) - 1u;
  if (q < 7) {
    double rtx = (rs[0][0] + rs21[0] * c_qxi[q]) + rs31[0] * c_qeta[q];
    double rty = (rs[0][1] + rs21[1] * c_qxi[q]) + rs31[1] * c_qeta[q];
    ok = jksums_group<NP>(ul * (rmc[0] - rtx), ul * (rmc[1] - rty), np, nophase, us1x, us1y, us2x, us2y, ph1, ph2,
                          etab, js, ks);
  }
  // phasing-free terms (the pair's first lane only)
  double rr0 = 0, rr1 = 0, ri = 0;
  if (q == 0) {
    const int nxt[3] = {1, 2, 0};
    for (int i = 0; i < 3; ++i) {
      int ip1 = nxt[i];
      double lx = rs[ip1][0] - rs[i][0], ly = rs[ip1][1] - rs[i][1];
      double ln = sqrt(lx * lx + ly * ly);
      lx /= ln;
      ly /= ln;
      double ux = (-unz) * (-ly), uy = (-unz) * lx;
      double d0x = rs[i][0] - rmc[0], d0y = rs[i][1] - rmc[1];
      double d1x = rs[ip1][0] - rmc[0], d1y = rs[ip1][1] - rmc[1];
      double p0 = ux * d0x + uy * d0y;
      double p0sq = p0 * p0;
      double lp = lx * d1x + ly * d1y;
      double lm = lx * d0x + ly * d0y;
      double ledge = lp - lm;
      double pplus = sqrt(p0sq + lp * lp);
      double pminus = sqrt(p0sq + lm * lm);
      double factor;
      if (fabs(p0 / ledge) < 1e-4) {
        factor = lp * pplus - lm * pminus;
      } else {
        factor = p0 * log((pplus + lp) / (pminus + lm));
        ri += factor;
        factor = (factor * p0 + pplus * lp) - pminus * lm;
      }
      rr0 += ux * factor;
      rr1 += uy * factor;
    }
    rr0 *= 0.5;
    rr1 *= 0.5;
    rr0 /= area2;
    rr1 /= area2;
    ri /= (area2 * ul);
  }
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    cd aJ = mkcd(0, 0), aJx = aJ, aJe = aJ, aK = aJ, aKx = aJ, aKe = aJ;
    int bad = 0;
#pragma unroll
    for (int i = 0; i < 7; ++i) {  // every lane takes part in the shuffles; the group's lane 0 keeps the sums
      cd jv, kv;
      jv.x = __shfl_sync(0xffffffffu, js[p].x, grp + i);
      jv.y = __shfl_sync(0xffffffffu, js[p].y, grp + i);
      kv.x = __shfl_sync(0xffffffffu, ks[p].x, grp + i);
      kv.y = __shfl_sync(0xffffffffu, ks[p].y, grp + i);
      bad |= !((__shfl_sync(0xffffffffu, ok, grp + i) >> p) & 1u);
      cd jw = c_qw[i] * jv;
      aJx = aJx + c_qxi[i] * jw;
      aJe = aJe + c_qeta[i] * jw;
      aJ = aJ + jw;
      cd kw = c_qw[i] * kv;
      aKx = aKx + c_qxi[i] * kw;
      aKe = aKe + c_qeta[i] * kw;
      aK = aK + kw;
    }
    if (q != 0 || !live || p >= np) continue;
    const JKDev &o = jk.s[p];
    o.J[iu] = aJ; o.Jxi[iu] = aJx; o.Jeta[iu] = aJe;
    o.K[iu] = aK; o.Kxi[iu] = aKx; o.Keta[iu] = aKe;
    o.rho_r[2 * iu] = rr0;
    o.rho_r[2 * iu + 1] = rr1;
    o.rinv[iu] = ri;
    if (bad) atomicAdd(nonconv + p, 1);
  }
}

// Per-point coefficients that turn the face-pair integrals into Z terms:
//   a_isl = cI1*I1_i + sing + u*J_i + cK*K_i,   φ = cI2*I2 + u*(rinv + J) + cKP*K,
//   term(isl, iml) = zA*(ρc2[iml]·a_isl) - zP*φ.
struct PairCoef {
  cd cI1, cK, cI2, cKP, zA, zP;
};

__device__ __forceinline__ PairCoef pair_coef(const PointParams &P) {
  PairCoef c;
  const double eps0 = 1.0 / (PSS_MU0 * (PSS_C0 * PSS_C0));
  const double u = P.u, w = P.omega;
  if (!P.magnetic) {
    c.cI1 = mkcd(PSS_FOURPI, 0);
    c.cK = P.c3 / u;
    c.cI2 = mkcd(PSS_FOURPI, 0);
    c.cKP = P.d3 / u;
    c.zA = mkcd(0.0, w) * ((PSS_MU0 / PSS_FOURPI) * P.mutilde);
    c.zP = (mkcd(0.0, 1.0) / P.epsbar) * mkcd(1.0 / (PSS_TWOPI * w * eps0), 0.0);
  } else {
    c.cI1 = P.I1fact;
    c.cK = P.KFfact;
    c.cI2 = P.I2fact;
    c.cKP = P.KPfact;
    c.zA = mkcd(0.0, -w) * ((-eps0 / PSS_PI) * P.epsbar);
    c.zP = mkcd(0.0, 2.0) / ((PSS_PI * w * PSS_MU0) * P.mutilde);
  }
  return c;
}

__global__ void __launch_bounds__(128, 5) k_pairs(SheetDev G, const PointParams *__restrict__ Pp, JKDev jk,
                                               const cd *__restrict__ t1, const cd *__restrict__ t2, int mmax,
                                               cd *__restrict__ zb) {
  int iu = blockIdx.x * blockDim.x + threadIdx.x;
  if (iu >= G.nufp) return;
  const PointParams &P = *Pp;
  const PairCoef C = pair_coef(P);
  int fp = G.ufp_rep[iu];
  int ifm = fp % G.nface, ifs = fp / G.nface;
  const double inv = 1.0 / G.upm;
  double rs[3][2], rm[3][2];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    int vs = G.fv[3 * ifs + k], vm = G.fv[3 * ifm + k];
    rs[k][0] = G.rho[2 * vs] / G.upm;
    rs[k][1] = G.rho[2 * vs + 1] / G.upm;
    rm[k][0] = G.rho[2 * vm] / G.upm;
    rm[k][1] = G.rho[2 * vm + 1] / G.upm;
  }
  (void)inv;
  double rmc[2] = {((rm[0][0] + rm[1][0]) + rm[2][0]) / 3, ((rm[0][1] + rm[1][1]) + rm[2][1]) / 3};
  cd I1 = mkcd(0, 0), I1x = I1, I1e = I1, I2 = I1;
  for (int i = 0; i < 7; ++i) {
    double rtx = (rs[0][0] + (rs[1][0] - rs[0][0]) * c_qxi[i]) + (rs[2][0] - rs[0][0]) * c_qeta[i];
    double rty = (rs[0][1] + (rs[1][1] - rs[0][1]) * c_qxi[i]) + (rs[2][1] - rs[0][1]) * c_qeta[i];
    double dx = rmc[0] - rtx, dy = rmc[1] - rty;
    cd g1 = sigma_interp(t1, mmax, P, dx, dy);
    cd g2 = sigma_interp(t2, mmax, P, dx, dy);
    cd g1w = c_qw[i] * g1;
    I1x = I1x + c_qxi[i] * g1w;
    I1e = I1e + c_qeta[i] * g1w;
    I1 = I1 + g1w;
    I2 = I2 + c_qw[i] * g2;
  }
  cd J = jk.J[iu], Jx = jk.Jxi[iu], Je = jk.Jeta[iu];
  cd K = jk.K[iu], Kx = jk.Kxi[iu], Ke = jk.Keta[iu];
  double rinv = jk.rinv[iu], rr0 = jk.rho_r[2 * iu], rr1 = jk.rho_r[2 * iu + 1];
  cd I1z = (I1 - I1x) - I1e, Jz = (J - Jx) - Je, Kz = (K - Kx) - Ke;
  const double u = P.u;
  cd phi = (C.cI2 * I2 + u * (mkcd(rinv, 0) + J)) + C.cKP * K;
  cd zphi = C.zP * phi;
  double rc2[3][2];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    rc2[i][0] = 0.5 * (rmc[0] - rm[i][0]);
    rc2[i][1] = 0.5 * (rmc[1] - rm[i][1]);
  }
  cd *out = zb + iu;  // plane q at out[q * nufp]: consecutive classes, coalesced stores
#pragma unroll
  for (int isl = 0; isl < 3; ++isl) {
    double sing0 = rr0 + (u * rinv) * (rmc[0] - rs[isl][0]);
    double sing1 = rr1 + (u * rinv) * (rmc[1] - rs[isl][1]);
    cd av[2];
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      cd Ii = ((rs[0][d] * I1x + rs[1][d] * I1e) + rs[2][d] * I1z) - rs[isl][d] * I1;
      cd Ji = ((rs[0][d] * Jx + rs[1][d] * Je) + rs[2][d] * Jz) - rs[isl][d] * J;
      cd Ki = ((rs[0][d] * Kx + rs[1][d] * Ke) + rs[2][d] * Kz) - rs[isl][d] * K;
      double sg = d == 0 ? sing0 : sing1;
      av[d] = ((C.cI1 * Ii + mkcd(sg, 0)) + u * Ji) + C.cK * Ki;
    }
#pragma unroll
    for (int iml = 0; iml < 3; ++iml) {
      cd dp = rc2[iml][0] * av[0] + rc2[iml][1] * av[1];
      out[(size_t)(3 * isl + iml) * G.nufp] = C.zA * dp - zphi;
    }
  }
}

// Z[m, n] (m = test / match basis function, n = source) from the pair terms zb: the <= 4 x 4
// face incidences of the two basis functions in a fixed order, with the Floquet / sign flags
// and the surface-resistance terms of Eqs. 7-34/7-35 (FillZY.jl:221-230).
__device__ __forceinline__ cd assemble_entry(const SheetDev &G, const PointParams &P, const cd *__restrict__ zb,
                                             int m, int n) {
  cd acc = mkcd(0, 0);
  const int cm = G.inc_cnt[m], cn = G.inc_cnt[n];
  for (int a = 0; a < cm; ++a) {
    const int fa = G.inc_face[4 * m + a], ka = G.inc_loc[4 * m + a];
    const cd ffa = P.ff[G.inc_eci[4 * m + a]];
    const cd mflag = G.inc_sgn[4 * m + a] > 0 ? conjd(ffa) : -conjd(ffa);
    for (int b = 0; b < cn; ++b) {
      const int fb = G.inc_face[4 * n + b], kb = G.inc_loc[4 * n + b];
      const cd ffb = P.ff[G.inc_eci[4 * n + b]];
      const cd sflag = G.inc_sgn[4 * n + b] > 0 ? ffb : -ffb;
      const int iu = G.ufpm[(size_t)fa + (size_t)fb * G.nface];
      const cd v = zb[(size_t)(3 * kb + ka) * G.nufp + iu];
      acc = acc + (mflag * sflag) * v;
      if (!P.magnetic && fa == fb) {
        const double fr = G.fr[fa];
        if (fr != 0.0) {
          const double *ls = G.face_ls + 3 * fa;
          const double g = fr / G.face_a48[fa];
          if (ka == kb) {  // the other two edges of the face: next and previous slot
            double l1 = ls[(kb + 1) % 3], l2 = ls[(kb + 2) % 3], l0 = ls[kb];
            acc = acc + mkcd(g * (3 * (l1 * l1 + l2 * l2) - l0 * l0), 0.0);
          } else {
            double lt = ls[3 - ka - kb];  // the third edge
            double geo = ls[kb] * ls[kb] + ls[ka] * ls[ka] - 3 * (lt * lt);
            acc = acc + geo * ((g * sflag) * mflag);
          }
        }
      }
    }
  }
  return acc;
}

// Z[m, n], row-major (z64 with leading dimension ld, the FP32 planes with ldf), one 32 x 64
// tile per CTA of 32 x 8 threads.  The gathers run with a warp along the 32 rows of a tile
// column (consecutive match basis functions against one source basis function: consecutive
// match faces, so the class look-ups and most pair-term loads of a warp are contiguous); each
// thread takes 8 columns (independent gathers in flight); the tile then goes out through
// shared memory row by row, 64 consecutive entries per row.
__global__ void __launch_bounds__(256) k_assemble(SheetDev G, const PointParams *__restrict__ Pp,
                                                  const cd *__restrict__ zb, cd *__restrict__ z64,
                                                  float *__restrict__ zr, float *__restrict__ zi, long long ld,
                                                  long long ldf) {
  __shared__ cd tile[32][65];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int m0 = blockIdx.y * 32, n0 = blockIdx.x * 64;
  const int m = m0 + tx;
  const PointParams &P = *Pp;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int c = ty + 8 * k, n = n0 + c;
    tile[tx][c] = (m < G.nbf && n < G.nbf) ? assemble_entry(G, P, zb, m, n) : mkcd(0, 0);
  }
  __syncthreads();
#pragma unroll
  for (int rr = 0; rr < 4; ++rr) {
    const int r = ty * 4 + rr, mm = m0 + r;
    if (mm >= G.nbf) break;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int c = tx + 32 * h, n = n0 + c;
      if (n >= G.nbf) continue;
      const cd v = tile[r][c];
      if (z64) z64[(size_t)mm * ld + n] = v;
      if (zr) {
        zr[(size_t)mm * ldf + n] = (float)v.x;
        zi[(size_t)mm * ldf + n] = (float)v.y;
      }
    }
  }
}

// Adjoint contraction of one perturbed input set, without its matrix.  CTA (x, y) takes the 32
// rows m = 32x .. 32x+31 (threadIdx.x) and column chunk y of gridDim.y; its 8 warps split the
// chunk's columns (n = chunk start + threadIdx.y + 8j);
// each thread assembles Z_k[m, n] on the fly from the set's pair terms (recomputed
// Green's-function values, never stored) - a warp gathers one column's 32 rows, consecutive
// match faces, so its class look-ups are contiguous - and accumulates Z_k[m, n] X[n, b].  The
// 8 column shares of a row are added in a fixed order to form the chunk's part of
//     y[m, b] = R_k[m, b] - sum_n Z_k[m, n] X[n, b]
// (R_k in chunk 0's part) for the right-hand sides b0 .. b0+NB-1, and the CTA writes its share
// of G[a + b*nm] = sum_m Lam[m, a] y[m, b] to part[x + y*gridDim.x] (rows in a fixed order, no
// atomics: the shares are added in a fixed order by k_adj_reduce, so the result is deterministic).
// Vectors are nbf x nm column-major.
constexpr int kAdjNB = 8;
__global__ void __launch_bounds__(256) k_adj_contract(SheetDev G, const PointParams *__restrict__ Pp,
                                                      const cd *__restrict__ zb, const cd *__restrict__ X,
                                                      const cd *__restrict__ R, const cd *__restrict__ Lam, int nm,
                                                      int b0, cd *__restrict__ part) {
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int m = blockIdx.x * 32 + tx;
  const int nb = min(kAdjNB, nm - b0);
  const int nbf = G.nbf;
  const int csz = (nbf + gridDim.y - 1) / gridDim.y, c0 = blockIdx.y * csz, c1 = min(nbf, c0 + csz);
  __shared__ cd red[8][32][kAdjNB];
  __shared__ cd yrow[32][kAdjNB];
  cd acc[kAdjNB];
#pragma unroll
  for (int b = 0; b < kAdjNB; ++b) acc[b] = mkcd(0, 0);
  if (m < nbf) {
    const PointParams &P = *Pp;
    for (int n = c0 + ty; n < c1; n += 8) {
      const cd z = assemble_entry(G, P, zb, m, n);
#pragma unroll
      for (int b = 0; b < kAdjNB; ++b)
        if (b < nb) acc[b] = acc[b] + z * X[(size_t)(b0 + b) * nbf + n];
    }
  }
#pragma unroll
  for (int b = 0; b < kAdjNB; ++b) red[ty][tx][b] = acc[b];
  __syncthreads();
  if (ty == 0) {
    for (int b = 0; b < kAdjNB; ++b) {
      cd sdot = mkcd(0, 0);
      for (int w = 0; w < 8; ++w) sdot = sdot + red[w][tx][b];
      const cd rb = blockIdx.y == 0 ? R[(size_t)(b0 + b) * nbf + m] : mkcd(0, 0);
      yrow[tx][b] = (m < nbf && b < nb) ? rb - sdot : mkcd(0, 0);
    }
  }
  __syncthreads();
  // this CTA's share of G: thread e of the 256 covers entries e, e + 256, ...
  const int tid = ty * 32 + tx;
  for (int e = tid; e < nm * nb; e += 256) {
    const int a = e % nm, b = e / nm;
    cd sum = mkcd(0, 0);
    for (int r = 0; r < 32; ++r) {
      const int mr = blockIdx.x * 32 + r;
      if (mr < nbf) sum = sum + Lam[(size_t)a * nbf + mr] * yrow[r][b];
    }
    part[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * nm * nm + a + (size_t)(b0 + b) * nm] = sum;
  }
}

// G[e] = sum over the CTAs' shares, in a fixed order (strided partial sums, then a tree).
__global__ void __launch_bounds__(256) k_adj_reduce(int nparts, int ne, const cd *__restrict__ part, cd *__restrict__ G) {
  const int e = blockIdx.x;
  __shared__ cd red[256];
  cd s = mkcd(0, 0);
  for (int q = threadIdx.x; q < nparts; q += 256) s = s + part[(size_t)q * ne + e];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) G[e] = red[0];
}

}  // namespace

constexpr int kAdjChunks = 8;  // column chunks of the contraction grid
size_t pss_adj_part_bytes(int nbf, int nm) { return (size_t)cdiv_u(nbf, 32) * kAdjChunks * nm * nm * sizeof(cd); }

void pss_adj_contract(const SheetDev &G, const PointParams *dP1, const cd *zb, const cd *X, const cd *R,
                      const cd *Lam, int nm, cd *part, cd *Gout, cudaStream_t st) {
  const int nblk = cdiv_u(G.nbf, 32);
  for (int b0 = 0; b0 < nm; b0 += kAdjNB) {
    pss_count_launch();
    k_adj_contract<<<dim3(nblk, kAdjChunks), dim3(32, 8), 0, st>>>(G, dP1, zb, X, R, Lam, nm, b0, part);
  }
  pss_count_launch();
  k_adj_reduce<<<nm * nm, 256, 0, st>>>(nblk * kAdjChunks, nm * nm, part, Gout);
}

void pss_filljk_group(const SheetDev &G, double ulocal, int np, const double *psi1, const double *psi2,
                      const double s1[2], const double s2[2], const JKDev *jk, int *nonconv, cudaStream_t st) {
  if (G.nufp == 0 || np <= 0) return;
  PsiGroup pg{};
  JKGroup jg{};
  pg.n = std::min(np, kJKGroup);
  for (int p = 0; p < pg.n; ++p) {
    pg.psi1[p] = psi1[p];
    pg.psi2[p] = psi2[p];
    jg.s[p] = jk[p];
  }
  const double a = ulocal * s1[0], b = ulocal * s1[1], c = ulocal * s2[0], d = ulocal * s2[1];
  const long long lanes = (long long)G.nufp * 8;
  pss_count_launch();
  if (pg.n == 1)
    k_filljk<1><<<cdiv_u(lanes, jk_threads<1>()), jk_threads<1>(), 0, st>>>(G, ulocal, pg, a, b, c, d, jg, nonconv);
  else if (pg.n == 2)
    k_filljk<2><<<cdiv_u(lanes, jk_threads<2>()), jk_threads<2>(), 0, st>>>(G, ulocal, pg, a, b, c, d, jg, nonconv);
  else
    k_filljk<kJKGroup><<<cdiv_u(lanes, jk_threads<kJKGroup>()), jk_threads<kJKGroup>(), 0, st>>>(G, ulocal, pg, a, b,
                                                                                             c, d, jg, nonconv);
}

void pss_filljk(const SheetDev &G, double ulocal, double psi1, double psi2, const double s1[2], const double s2[2],
                JKDev jk, int *nonconv, cudaStream_t st) {
  pss_filljk_group(G, ulocal, 1, &psi1, &psi2, s1, s2, &jk, nonconv, st);
}

void pss_fill_pairs(const SheetDev &G, const PointParams *dP1, const JKDev &jk, const cd *t1, const cd *t2,
                    int mmax, cd *zb, cudaStream_t st) {
  if (G.nufp == 0) return;
  pss_count_launch();
  k_pairs<<<cdiv_u(G.nufp, 128), 128, 0, st>>>(G, dP1, jk, t1, t2, mmax, zb);
}

void pss_fill_assemble(const SheetDev &G, const PointParams *dP1, const cd *zb, cd *z64, float *zr, float *zi,
                       long long ld, long long ldf, cudaStream_t st) {
  dim3 blk(32, 8);
  dim3 grd(cdiv_u(G.nbf, 64), cdiv_u(G.nbf, 32));
  pss_count_launch();
  k_assemble<<<grd, blk, 0, st>>>(G, dP1, zb, z64, zr, zi, ld, ldf);
}
