/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the periodic MoM fill path.
 *
 * A plain-C FP64 restatement of the PSSFSS.jl algorithms that the CUDA library
 * accelerates.  It is used by the test-suite as the checker, and timed by bench.py as
 * the CPU baseline; the product (pssfss.jl_b200/) never links or calls it.
 *
 * Each function names the reference source it restates (file:line in PSSFSS.jl v0.1.4).
 * Summation orders follow the reference's serial order (ring order of Rings.jl,
 * 7-point quadrature order of Zint.jl) so the oracle is a close FP64 twin.  The 2-D
 * FFT the reference takes from FFTW (PGF.jl:313-314) is restated as an exact
 * mixed-radix 2/3/5 DFT; the LU/solve it takes from LAPACK is done by scipy's LAPACK
 * zgetrf/zgetrs in the Python wrapper.
 *
 * Parity pins: reference test golden values in test/FillZY_test.jl:45-46,77-78,
 * test/PGF_test.jl:40-44,56-60 (checked as in :71-83), test/RWGData_test.jl:46-48,56-58
 * (tests/golden/reference_golden.json).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

#define JKRINGMAX 65
#define MMAX_CAP 2048
#define CONVREPEAT 40

static const double TWOPI = 6.283185307179586;
static const double FOURPI = 12.566370614359172;
static const double PI = 3.141592653589793;
static const double MU0 = 1.25663706212e-6;
static const double C0 = 299792458.0;

static inline cplx mk(double re, double im) { return CMPLX(re, im); }
/* Julia Complex*Complex: (ac - bd, ad + bc) without C99 Annex-G NaN recovery. */
static inline cplx cmul(cplx a, cplx b) {
    double ar = creal(a), ai = cimag(a), br = creal(b), bi = cimag(b);
    return mk(ar * br - ai * bi, ar * bi + ai * br);
}
static inline cplx rmul(double x, cplx z) { return mk(x * creal(z), x * cimag(z)); }
static inline cplx cdivr(cplx z, double x) { return mk(creal(z) / x, cimag(z) / x); }
static inline cplx cadd(cplx a, cplx b) { return mk(creal(a) + creal(b), cimag(a) + cimag(b)); }
static inline cplx csub(cplx a, cplx b) { return mk(creal(a) - creal(b), cimag(a) - cimag(b)); }
static inline cplx cdiv(cplx a, cplx b) { return a / b; }
static inline cplx cis(double x) { return mk(cos(x), sin(x)); }
/* Julia Real - Complex: Complex(x - re, -im) */
static inline cplx rsubc(double x, cplx z) { return mk(x - creal(z), -cimag(z)); }

/* Rings.jl:14-55 -- element idx of ring r */
static inline void ring_mn(int r, int idx, int *m, int *n) {
    if (r == 0) { *m = 0; *n = 0; return; }
    int w = 2 * r + 1;
    if (idx < w) { *m = r; *n = -r + idx; return; }
    idx -= w;
    if (idx < w) { *m = -r; *n = -r + idx; return; }
    idx -= w;
    int h = 2 * r - 1;
    if (idx < h) { *m = -r + 1 + idx; *n = -r; return; }
    idx -= h;
    *m = -r + 1 + idx; *n = r;
}
static inline int ring_len(int r) { return r == 0 ? 1 : 8 * r; }

/* PGF.jl:116-120 */
static inline cplx mysqrt(cplx z) {
    cplx a = csqrt(z);
    if (creal(a) == 0.0 && cimag(a) < 0.0) a = mk(-creal(a), -cimag(a));
    return a;
}

/* Julia exp(z::Complex) = exp(re) * cis(im), returning Complex(er, im) when im == 0 */
static inline cplx jexp(double re, double im) {
    double er = exp(re);
    if (im == 0.0) return mk(er, im);
    return mk(er * cos(im), er * sin(im));
}

/* PGF.jl:67-106 -- frequency-independent spatial lattice sums J and K */
int ora_jksums(const double urho[2], double psi1, double psi2, const double us1[2],
               const double us2[2], int extract, double convtest, cplx *jout, cplx *kout) {
    const int rmin = 5;
    const double small = 1e-5;
    double arg = sqrt(urho[0] * urho[0] + urho[1] * urho[1]);
    double rterm = exp(-arg);
    cplx ksum = mk(rterm, 0.0), jsum;
    if (extract) {
        if (arg <= small) jsum = mk((-arg / 6 + 0.5) * arg - 1, 0.0);
        else jsum = mk((rterm - 1) / arg, 0.0);
    } else {
        jsum = mk(rterm / arg, 0.0);
    }
    int converged = 0;
    for (int r = 1; r <= JKRINGMAX; ++r) {
        cplx jring = 0, kring = 0;
        int len = ring_len(r);
        for (int t = 0; t < len; ++t) {
            int m, n;
            ring_mn(r, t, &m, &n);
            double dx = urho[0] - ((double)m * us1[0] + (double)n * us2[0]);
            double dy = urho[1] - ((double)m * us1[1] + (double)n * us2[1]);
            double a = sqrt(dx * dx + dy * dy);
            double ph = (double)m * psi1 + (double)n * psi2;
            cplx term = jexp(-a, -ph);
            jring = cadd(jring, cdivr(term, a));
            kring = cadd(kring, term);
        }
        jsum = cadd(jsum, jring);
        ksum = cadd(ksum, kring);
        if (r > rmin) {
            double c1 = cabs(jring / jsum), c2 = cabs(kring / ksum);
            double conv = c1 > c2 ? c1 : c2;
            if (conv < convtest) { converged = 1; break; }
        }
    }
    *jout = jsum;
    *kout = ksum;
    return converged;
}

/* PGF.jl:138-142 */
static cplx c3_calc(double k0, double u, cplx mu1, cplx eps1, cplx mu2, cplx eps2) {
    cplx w1sq = cadd(cmul(rmul(k0 * k0, mu1), eps1), mk(u * u, 0));
    cplx w2sq = cadd(cmul(rmul(k0 * k0, mu2), eps2), mk(u * u, 0));
    return cdiv(cadd(cmul(mu1, w2sq), cmul(mu2, w1sq)), rmul(2.0, cadd(mu1, mu2)));
}
/* PGF.jl:157-162 */
static cplx d3_calc(double k0, double u, cplx mu1, cplx eps1, cplx mu2, cplx eps2) {
    cplx w1sq = cadd(cmul(rmul(k0 * k0, mu1), eps1), mk(u * u, 0));
    cplx w2sq = cadd(cmul(rmul(k0 * k0, mu2), eps2), mk(u * u, 0));
    cplx t1 = csub(cmul(w2sq, cadd(rmul(2.0, eps1), eps2)), cmul(w1sq, eps1));
    cplx t2 = csub(cmul(w1sq, cadd(rmul(2.0, eps2), eps1)), cmul(w2sq, eps2));
    cplx num = cadd(cmul(mu1, t1), cmul(mu2, t2));
    return cdiv(num, cmul(rmul(2.0, cadd(mu1, mu2)), cadd(eps1, eps2)));
}

/* ---------------- exact mixed-radix DFT (stands in for FFTW's fft!) ---------------- */
/* Recursive decimation in time over factors 2,3,5; twiddles exp(-2πi k/N) computed from
 * the reduced integer k mod N so every twiddle is as accurate as one sin/cos call. */
static void dft_rec(const cplx *in, size_t stride, cplx *out, int n, int N_total, cplx *scratch) {
    if (n == 1) { out[0] = in[0]; return; }
    int p = (n % 2 == 0) ? 2 : (n % 3 == 0) ? 3 : 5;
    int mlen = n / p;
    for (int j = 0; j < p; ++j)
        dft_rec(in + j * stride, stride * p, out + j * mlen, mlen, N_total, scratch);
    /* butterflies: X[k + q*mlen] = sum_j W_n^{j(k+q mlen)} Y_j[k] */
    for (int k = 0; k < mlen; ++k) {
        cplx y[5];
        for (int j = 0; j < p; ++j) {
            long e = (long)j * k % n;
            double ang = -TWOPI * (double)e / (double)n;
            y[j] = (e == 0) ? out[j * mlen + k] : cmul(out[j * mlen + k], cis(ang));
        }
        for (int q = 0; q < p; ++q) {
            cplx s = y[0];
            for (int j = 1; j < p; ++j) {
                long e = (long)j * q % p;
                if (e == 0) s = cadd(s, y[j]);
                else s = cadd(s, cmul(y[j], cis(-TWOPI * (double)e / (double)p)));
            }
            scratch[q] = s;
        }
        for (int q = 0; q < p; ++q) out[k + q * mlen] = scratch[q];
    }
}

static void dft1(cplx *x, size_t stride, int n, cplx *buf_in, cplx *buf_out) {
    for (int i = 0; i < n; ++i) buf_in[i] = x[i * stride];
    cplx scratch[5];
    dft_rec(buf_in, 1, buf_out, n, n, scratch);
    for (int i = 0; i < n; ++i) x[i * stride] = buf_out[i];
}

/* In-place 2-D forward DFT of a column-major n x n matrix. */
static void dft2(cplx *a, int n) {
    #pragma omp parallel
    {
        cplx *bi = malloc(sizeof(cplx) * n), *bo = malloc(sizeof(cplx) * n);
        #pragma omp for schedule(static)
        for (int c = 0; c < n; ++c) dft1(a + (size_t)c * n, 1, n, bi, bo);
        #pragma omp for schedule(static)
        for (int r = 0; r < n; ++r) dft1(a + r, (size_t)n, n, bi, bo);
        free(bi); free(bo);
    }
}

static int nextprod235(int x) {
    for (int v = x;; ++v) {
        int t = v;
        while (t % 2 == 0) t /= 2;
        while (t % 3 == 0) t /= 3;
        while (t % 5 == 0) t /= 5;
        if (t == 1) return v;
    }
}

/* Layer-stack spectral summands for one (m, n) (PGF.jl:240-283 electric, 529-567 magnetic). */
typedef struct {
    int nl, s; /* s is 1-based interface index */
    const cplx *eps, *mu;
    const double *width;
    double k0sq, u;
    cplx mutilde, epsbar, c3, d3;      /* electric */
    cplx f1, f3, p1, p3;              /* magnetic */
} stack_t;

static void summand(const stack_t *S, int magnetic, double beta_sq, double kappa_sq,
                    double kappa, cplx *t1, cplx *t2) {
    int nl = S->nl, s = S->s;
    const cplx *eps = S->eps, *mu = S->mu;
    double k0sq = S->k0sq;
    cplx gam = mysqrt(rsubc(beta_sq, cmul(rmul(k0sq, eps[0]), mu[0])));
    cplx LTE, LTM, RTE, RTM;
    if (!magnetic) { LTE = cdiv(mu[0], gam); LTM = cdiv(gam, eps[0]); }
    else { LTE = cdiv(gam, mu[0]); LTM = cdiv(eps[0], gam); }
    for (int i = 2; i <= s; ++i) {
        cplx g = mysqrt(rsubc(beta_sq, cmul(rmul(k0sq, eps[i - 1]), mu[i - 1])));
        cplx Z0TE, Z0TM;
        if (!magnetic) { Z0TE = cdiv(mu[i - 1], g); Z0TM = cdiv(g, eps[i - 1]); }
        else { Z0TE = cdiv(g, mu[i - 1]); Z0TM = cdiv(eps[i - 1], g); }
        cplx th = ctanh(rmul(S->width[i - 1], g));
        LTE = cdiv(cmul(Z0TE, cadd(LTE, cmul(Z0TE, th))), cadd(Z0TE, cmul(LTE, th)));
        LTM = cdiv(cmul(Z0TM, cadd(LTM, cmul(Z0TM, th))), cadd(Z0TM, cmul(LTM, th)));
    }
    gam = mysqrt(rsubc(beta_sq, cmul(rmul(k0sq, eps[nl - 1]), mu[nl - 1])));
    if (!magnetic) { RTE = cdiv(mu[nl - 1], gam); RTM = cdiv(gam, eps[nl - 1]); }
    else { RTE = cdiv(gam, mu[nl - 1]); RTM = cdiv(eps[nl - 1], gam); }
    for (int i = nl - 1; i >= s + 1; --i) {
        cplx g = mysqrt(rsubc(beta_sq, cmul(rmul(k0sq, eps[i - 1]), mu[i - 1])));
        cplx Z0TE, Z0TM;
        if (!magnetic) { Z0TE = cdiv(mu[i - 1], g); Z0TM = cdiv(g, eps[i - 1]); }
        else { Z0TE = cdiv(g, mu[i - 1]); Z0TM = cdiv(eps[i - 1], g); }
        cplx th = ctanh(rmul(S->width[i - 1], g));
        RTE = cdiv(cmul(Z0TE, cadd(RTE, cmul(Z0TE, th))), cadd(Z0TE, cmul(RTE, th)));
        RTM = cdiv(cmul(Z0TM, cadd(RTM, cmul(Z0TM, th))), cadd(Z0TM, cmul(RTM, th)));
    }
    if (!magnetic) {
        cplx ViTE = cdiv(cmul(LTE, RTE), cadd(LTE, RTE));
        cplx ViTM = cdiv(cmul(LTM, RTM), cadd(LTM, RTM));
        ViTE = cdiv(rmul(2.0, ViTE), S->mutilde);
        *t1 = csub(ViTE, cdivr(cadd(mk(1.0, 0.0), cdivr(S->c3, kappa_sq)), kappa));
        ViTM = cmul(rmul(2.0, S->epsbar), ViTM);
        cplx kk = cmul(cmul(rmul(k0sq, S->epsbar), S->mutilde), ViTE);
        *t2 = csub(cdivr(cadd(ViTM, kk), beta_sq),
                   cdivr(cadd(mk(1.0, 0.0), cdivr(S->d3, kappa_sq)), kappa));
    } else {
        cplx ytm = cadd(LTM, RTM);
        *t1 = csub(ytm, cdivr(cadd(S->f1, cdivr(S->f3, kappa_sq)), kappa));
        cplx num = cadd(cadd(rmul(k0sq, ytm), LTE), RTE);
        *t2 = csub(cdivr(num, beta_sq), cdivr(cadd(S->p1, cdivr(S->p3, kappa_sq)), kappa));
    }
}

/*
 * PGF.jl:196-365 (electric, magnetic=0) and PGF.jl:478-629 (magnetic=1).
 * Builds the two padded interpolation tables, each (mmax+2)^2 complex, column-major,
 * index (m,n) in -1..mmax stored at (m+1) + (n+1)*(mmax+2).  Outputs must hold
 * (MMAX_CAP+2)^2 entries.  Returns mmax; *converged_out = 0 if the cap was hit.
 */
int ora_modal_tables(int magnetic, double k0, double u, double psi1, double psi2, int nl,
                     const cplx *eps, const cplx *mu, const double *width, int s,
                     const double b1[2], const double b2[2], const double b00[2],
                     double convtest, cplx *tab1_out, cplx *tab2_out, int *converged_out) {
    stack_t S;
    S.nl = nl; S.s = s; S.eps = eps; S.mu = mu; S.width = width; S.u = u;
    double k0sq = k0 * k0;
    S.k0sq = k0sq;
    double b2min = 1e-10 * k0sq;
    cplx mus = mu[s - 1], mus1 = mu[s], epss = eps[s - 1], epss1 = eps[s];
    S.mutilde = cdiv(cmul(rmul(2.0, mus), mus1), cadd(mus, mus1));
    S.epsbar = cdivr(cadd(epss, epss1), 2.0);
    double cr = b1[0] * b2[1] - b1[1] * b2[0];
    double area = 4.0 * (PI * PI) / fabs(cr);
    if (!magnetic) {
        S.c3 = c3_calc(k0, u, mus, epss, mus1, epss1);
        S.d3 = d3_calc(k0, u, mus, epss, mus1, epss1);
    } else {
        cplx c3s = c3_calc(k0, u, epss, mus, epss, mus);
        cplx c3sp1 = c3_calc(k0, u, epss1, mus1, epss1, mus1);
        cplx d3s = d3_calc(k0, u, epss, mus, epss, mus);
        cplx d3sp1 = d3_calc(k0, u, epss1, mus1, epss1, mus1);
        S.f1 = rmul(2.0, S.epsbar);
        S.f3 = cadd(cmul(epss, c3s), cmul(epss1, c3sp1));
        S.p1 = cdiv(mk(2.0, 0.0), S.mutilde);
        S.p3 = cadd(cdiv(d3s, mus), cdiv(d3sp1, mus1));
    }
    const int mg = MMAX_CAP / 2;
    const int W = 2 * mg + 1;
    cplx *t1 = calloc((size_t)W * W, sizeof(cplx));
    cplx *t2 = calloc((size_t)W * W, sizeof(cplx));
    char *convlist = calloc(mg + 1, 1);
#define TIX(m, n) ((size_t)((m) + mg) + (size_t)((n) + mg) * W)
    int mmax = 0, mmax_old = -2, first = 1, converged = 0;
    mmax = 16; /* mmax_list[1] ÷ 2: only needs to enter the loop (PGF.jl:219) */
    while (mmax < MMAX_CAP) {
        if (first) { mmax = 0; first = 0; }
        else {
            mmax = nextprod235(1 + mmax);
            while (mmax % 2 != 0) mmax = nextprod235(1 + mmax);
        }
        int mo2 = mmax / 2, oo2 = mmax_old / 2;
        /* Julia's ÷ truncates: (-2)÷2 = -1 */
        #pragma omp parallel for schedule(dynamic, 1)
        for (int r = oo2 + 1; r <= mo2; ++r) {
            cplx rs1 = 0, rs2 = 0;
            int len = ring_len(r);
            for (int t = 0; t < len; ++t) {
                int m, n;
                ring_mn(r, t, &m, &n);
                double bx = (b00[0] + (double)m * b1[0]) + (double)n * b2[0];
                double by = (b00[1] + (double)m * b1[1]) + (double)n * b2[1];
                double bsq = bx * bx + by * by;
                if (bsq < b2min) bsq = b2min;
                double ksq = bsq + u * u;
                double kap = sqrt(ksq);
                cplx v1, v2;
                summand(&S, magnetic, bsq, ksq, kap, &v1, &v2);
                t1[TIX(m, n)] = v1;
                t2[TIX(m, n)] = v2;
                rs1 = cadd(rs1, v1);
                rs2 = cadd(rs2, v2);
            }
            double test1 = cabs(rs1 / t1[TIX(0, 0)]);
            double test2 = cabs(rs2 / t2[TIX(0, 0)]);
            convlist[r] = (test1 < convtest) && (test2 < convtest);
        }
        if (mo2 >= CONVREPEAT) {
            int all = 1;
            for (int r = mo2 - CONVREPEAT + 1; r <= mo2; ++r) all &= convlist[r];
            if (all) { converged = 1; break; }
        }
        mmax_old = mmax;
    }
    *converged_out = converged;
    int mo2 = mmax / 2;
    /* table_t[p, q] = table[p - mo2, q - mo2], p,q in 0..mmax-1; then forward 2-D DFT */
    cplx *a1 = malloc(sizeof(cplx) * (size_t)mmax * mmax);
    cplx *a2 = malloc(sizeof(cplx) * (size_t)mmax * mmax);
    for (int q = 0; q < mmax; ++q)
        for (int p = 0; p < mmax; ++p) {
            a1[p + (size_t)q * mmax] = t1[TIX(p - mo2, q - mo2)];
            a2[p + (size_t)q * mmax] = t2[TIX(p - mo2, q - mo2)];
        }
    dft2(a1, mmax);
    dft2(a2, mmax);
    /* Eq. (5.32) phase and 1/(2A) (electric) or 1/A (magnetic): PGF.jl:316-324, 593-601 */
    double scale = magnetic ? area : 2 * area;
    for (int q = 0; q < mmax; ++q) {
        double qterm = q * (PI - psi2 / mmax);
        for (int p = 0; p < mmax; ++p) {
            double pterm = p * (PI - psi1 / mmax);
            cplx cf = cdivr(cis(pterm + qterm), scale);
            a1[p + (size_t)q * mmax] = cmul(a1[p + (size_t)q * mmax], cf);
            a2[p + (size_t)q * mmax] = cmul(a2[p + (size_t)q * mmax], cf);
        }
    }
    int L = mmax + 2;
#define PIX(m, n) ((size_t)((m) + 1) + (size_t)((n) + 1) * L)
    cplx *o[2] = {tab1_out, tab2_out};
    cplx *a[2] = {a1, a2};
    for (int k = 0; k < 2; ++k) {
        cplx *T = o[k], *A = a[k];
        memset(T, 0, sizeof(cplx) * (size_t)L * L);
        for (int q = 0; q < mmax; ++q)
            for (int p = 0; p < mmax; ++p) T[PIX(p, q)] = A[p + (size_t)q * mmax];
        if (!magnetic) {
            /* PGF.jl:339-357 */
            cplx c1 = cis(-psi1), c2 = cis(-psi2), c12 = cmul(c1, c2);
            for (int kk = 0; kk < mmax; ++kk) {
                T[PIX(mmax, kk)] = cmul(c1, T[PIX(0, kk)]);
                T[PIX(kk, mmax)] = cmul(c2, T[PIX(kk, 0)]);
            }
            T[PIX(mmax, mmax)] = cmul(c12, T[PIX(0, 0)]);
            cplx ic1 = cdiv(mk(1.0, 0.0), c1), ic2 = cdiv(mk(1.0, 0.0), c2);
            for (int kk = 0; kk <= mmax; ++kk) T[PIX(-1, kk)] = cmul(ic1, T[PIX(mmax - 1, kk)]);
            for (int kk = -1; kk <= mmax - 1; ++kk) T[PIX(kk, -1)] = cmul(ic2, T[PIX(kk, mmax - 1)]);
        } else {
            /* PGF.jl:611-621 */
            cplx c1 = cis(-psi1), c2 = cis(-psi2), c12 = cis(-(psi1 + psi2));
            for (int kk = 0; kk < mmax; ++kk) T[PIX(mmax, kk)] = cmul(c1, T[PIX(0, kk)]);
            for (int kk = 0; kk < mmax; ++kk) T[PIX(kk, mmax)] = cmul(c2, T[PIX(kk, 0)]);
            T[PIX(mmax, mmax)] = cmul(c12, T[PIX(0, 0)]);
            cplx p1 = cis(psi1), p2 = cis(psi2);
            for (int kk = 0; kk <= mmax; ++kk) T[PIX(-1, kk)] = cmul(p1, T[PIX(mmax - 1, kk)]);
            for (int kk = -1; kk <= mmax - 1; ++kk) T[PIX(kk, -1)] = cmul(p2, T[PIX(kk, mmax - 1)]);
        }
    }
#undef PIX
#undef TIX
    free(a1); free(a2); free(t1); free(t2); free(convlist);
    return mmax;
}

/* PGF.jl:392-443 -- 6-point interpolation (AMS-55 25.2.67) in a padded table. */
cplx ora_sigma(const cplx *T, int mmax, const double b1[2], const double b2[2], double psi1,
               double psi2, const double rho[2]) {
    double x1o = (b1[0] * rho[0] + b1[1] * rho[1]) / TWOPI;
    if (fabs(x1o) < 1e-8) x1o = 0.0;
    double x2o = (b2[0] * rho[0] + b2[1] * rho[1]) / TWOPI;
    if (fabs(x2o) < 1e-8) x2o = 0.0;
    double x1, x2, r;
    r = fmod(x1o, 1.0);
    x1 = (r == 0) ? copysign(r, 1.0) : ((r > 0) != 1) ? r + 1.0 : r;
    r = fmod(x2o, 1.0);
    x2 = (r == 0) ? copysign(r, 1.0) : ((r > 0) != 1) ? r + 1.0 : r;
    long mshift = lrint(x1o - x1), nshift = lrint(x2o - x2);
    int m = (int)trunc(mmax * x1);
    double p = mmax * x1 - m;
    int n = (int)trunc(mmax * x2);
    double q = mmax * x2 - n;
    double p2 = p * p, q2 = q * q, pq = p * q;
    int L = mmax + 2;
#define PIX(a, b) ((size_t)((a) + 1) + (size_t)((b) + 1) * L)
    cplx s = rmul(0.5 * (q2 - q), T[PIX(m, n - 1)]);
    s = cadd(s, rmul(0.5 * (p2 - p), T[PIX(m - 1, n)]));
    s = cadd(s, rmul(((1 + pq) - p2) - q2, T[PIX(m, n)]));
    s = cadd(s, rmul(0.5 * ((p2 - 2 * pq) + p), T[PIX(m + 1, n)]));
    s = cadd(s, rmul(0.5 * ((q2 - 2 * pq) + q), T[PIX(m, n + 1)]));
    s = cadd(s, rmul(pq, T[PIX(m + 1, n + 1)]));
#undef PIX
    if (mshift != 0 || nshift != 0) s = cmul(s, cis(-((double)mshift * psi1 + (double)nshift * psi2)));
    return s;
}

/* 7-point triangle rule (Zint.jl:55-62, 219-225) */
static const double QXI[7] = {0.33333333333333330, 0.10128650732345633, 0.79742698535308730,
                              0.10128650732345633, 0.47014206410511505, 0.05971587178976989,
                              0.47014206410511505};
static const double QETA[7] = {0.33333333333333333, 0.79742698535308730, 0.10128650732345633,
                               0.10128650732345633, 0.05971587178976989, 0.47014206410511505,
                               0.47014206410511505};
static const double QW[7] = {0.1125, 0.06296959027241358, 0.06296959027241358,
                             0.06296959027241358, 0.06619707639425308, 0.06619707639425308,
                             0.06619707639425308};

/* geometry helpers: fv is 3 x nface column-major, 1-based */
static inline void vtx(const double *rho, const int64_t *fv, int64_t f, int k, double out[2]) {
    int64_t v = fv[3 * f + k] - 1;
    out[0] = rho[2 * v];
    out[1] = rho[2 * v + 1];
}

/* Zint.jl:54-179 (filljk!) -- frequency-independent face-pair integrals for each unique pair.
 * rho: 2 x nnode (sheet units), ufp_rep: 1-based column-major face-pair index of each
 * class's first member.  Outputs per class: J, Jxi, Jeta, K, Kxi, Keta, rho_r[2], rinv. */
void ora_filljk(int64_t nface, const double *rho, const int64_t *fv, int64_t nufp,
                const int64_t *ufp_rep, double ulocal, double psi1, double psi2,
                const double s1[2], const double s2[2], cplx *J, cplx *Jxi, cplx *Jeta,
                cplx *K, cplx *Kxi, cplx *Keta, double *rho_r, double *rinv, int *nonconv) {
    const int next[3] = {1, 2, 0};
    double us1[2] = {ulocal * s1[0], ulocal * s1[1]};
    double us2[2] = {ulocal * s2[0], ulocal * s2[1]};
    int bad = 0;
    #pragma omp parallel for schedule(dynamic, 64) reduction(+ : bad)
    for (int64_t iu = 0; iu < nufp; ++iu) {
        int64_t fp = ufp_rep[iu] - 1;
        int64_t ifm = fp % nface, ifs = fp / nface;
        double rs[3][2], rm[3][2];
        for (int k = 0; k < 3; ++k) { vtx(rho, fv, ifs, k, rs[k]); vtx(rho, fv, ifm, k, rm[k]); }
        double rs32[2] = {rs[2][0] - rs[1][0], rs[2][1] - rs[1][1]};
        double rs12[2] = {rs[0][0] - rs[1][0], rs[0][1] - rs[1][1]};
        double area2 = (-rs32[1]) * rs12[0] + rs32[0] * rs12[1];
        double unz = 1.0;
        if (area2 < 0) { area2 = fabs(area2); unz = -1.0; }
        double rs31[2] = {rs[2][0] - rs[0][0], rs[2][1] - rs[0][1]};
        double rs21[2] = {-rs12[0], -rs12[1]};
        double rmc[2] = {((rm[0][0] + rm[1][0]) + rm[2][0]) / 3, ((rm[0][1] + rm[1][1]) + rm[2][1]) / 3};
        cplx aJ = 0, aJx = 0, aJe = 0, aK = 0, aKx = 0, aKe = 0;
        for (int i = 0; i < 7; ++i) {
            double rt[2] = {(rs[0][0] + rs21[0] * QXI[i]) + rs31[0] * QETA[i],
                            (rs[0][1] + rs21[1] * QXI[i]) + rs31[1] * QETA[i]};
            double ur[2] = {ulocal * (rmc[0] - rt[0]), ulocal * (rmc[1] - rt[1])};
            cplx js, ks;
            if (!ora_jksums(ur, psi1, psi2, us1, us2, 1, 1e-8, &js, &ks)) bad += 1;
            cplx jw = rmul(QW[i], js);
            aJx = cadd(aJx, rmul(QXI[i], jw));
            aJe = cadd(aJe, rmul(QETA[i], jw));
            aJ = cadd(aJ, jw);
            cplx kw = rmul(QW[i], ks);
            aKx = cadd(aKx, rmul(QXI[i], kw));
            aKe = cadd(aKe, rmul(QETA[i], kw));
            aK = cadd(aK, kw);
        }
        double rr[2] = {0, 0}, ri = 0;
        for (int i = 0; i < 3; ++i) {
            int ip1 = next[i];
            double lv[2] = {rs[ip1][0] - rs[i][0], rs[ip1][1] - rs[i][1]};
            double ln = sqrt(lv[0] * lv[0] + lv[1] * lv[1]);
            lv[0] /= ln; lv[1] /= ln;
            double uv[2] = {(-unz) * (-lv[1]), (-unz) * lv[0]};
            double d0[2] = {rs[i][0] - rmc[0], rs[i][1] - rmc[1]};
            double d1[2] = {rs[ip1][0] - rmc[0], rs[ip1][1] - rmc[1]};
            double p0 = uv[0] * d0[0] + uv[1] * d0[1];
            double p0sq = p0 * p0;
            double lp = lv[0] * d1[0] + lv[1] * d1[1];
            double lm = lv[0] * d0[0] + lv[1] * d0[1];
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
            rr[0] += uv[0] * factor;
            rr[1] += uv[1] * factor;
        }
        rr[0] *= 0.5; rr[1] *= 0.5;
        rr[0] /= area2; rr[1] /= area2;
        ri /= (area2 * ulocal);
        J[iu] = aJ; Jxi[iu] = aJx; Jeta[iu] = aJe;
        K[iu] = aK; Kxi[iu] = aKx; Keta[iu] = aKe;
        rho_r[2 * iu] = rr[0]; rho_r[2 * iu + 1] = rr[1];
        rinv[iu] = ri;
    }
    *nonconv = bad;
}

/*
 * FillZY.jl:50-245 (cls 'J') and FillZY.jl:273-457 (cls 'M').  Fills Z (or Y), an
 * nbf x nbf column-major complex matrix, given the J/K data of ora_filljk (computed
 * with ulocal = u/units_per_meter) and the two modal tables.
 * Arrays: rho 2 x nnode (sheet units), fv/fe 3 x nface, bff 2 x nbf, ebf/eci nedge,
 * ufpm nface x nface column-major 1-based class numbers, ufp_rep nufp.
 */
void ora_fill(int magnetic, double k0, double u, int nl, const cplx *eps, const cplx *mu,
              int s, double psi1, double psi2, int64_t nface, const double *rho,
              const int64_t *fv, const int64_t *fe, const double *fr, int64_t nbf,
              const int64_t *bff, const int64_t *ebf, const int64_t *eci, const int64_t *ufpm,
              int64_t nufp, const int64_t *ufp_rep, double units_per_meter,
              const double b1_m[2], const double b2_m[2], const cplx *JKJ, const cplx *JKJxi,
              const cplx *JKJeta, const cplx *JKK, const cplx *JKKxi, const cplx *JKKeta,
              const double *JKrho_r, const double *JKrinv, const cplx *tab1, const cplx *tab2,
              int mmax, cplx *Z) {
    const int next[3] = {1, 2, 0}, prev[3] = {2, 0, 1};
    const int third[3][3] = {{0, 2, 1}, {2, 0, 0}, {1, 0, 0}}; /* 0-based of [0 3 2;3 0 1;2 1 0] */
    (void)nl;
    cplx mus = mu[s - 1], mus1 = mu[s], epss = eps[s - 1], epss1 = eps[s];
    cplx mutilde = cdiv(cmul(rmul(2.0, mus), mus1), cadd(mus, mus1));
    cplx epsbar = magnetic ? rmul(0.5, cadd(epss, epss1)) : cdivr(cadd(epss, epss1), 2.0);
    double omega = k0 * C0;
    double eps0 = 1.0 / (MU0 * (C0 * C0));
    cplx c3 = 0, d3 = 0, I1fact = 0, KFfact = 0, I2fact = 0, KPfact = 0;
    if (!magnetic) {
        c3 = c3_calc(k0, u, mus, epss, mus1, epss1);
        d3 = d3_calc(k0, u, mus, epss, mus1, epss1);
    } else {
        cplx c3s = c3_calc(k0, u, mus, epss, mus, epss);
        cplx c3sp1 = c3_calc(k0, u, mus1, epss1, mus1, epss1);
        cplx d3s = d3_calc(k0, u, mus, epss, mus, epss);
        cplx d3sp1 = d3_calc(k0, u, mus1, epss1, mus1, epss1);
        I1fact = cdiv(mk(PI, 0), epsbar);
        KFfact = cdiv(cadd(cmul(c3s, epss), cmul(c3sp1, epss1)), rmul(u, rmul(2.0, epsbar)));
        I2fact = rmul(PI, mutilde);
        KPfact = cmul(cdivr(mutilde, 2 * u), cadd(cdiv(d3s, mus), cdiv(d3sp1, mus1)));
    }
    double b00[2] = {(psi1 * b1_m[0] + psi2 * b2_m[0]) / TWOPI, (psi1 * b1_m[1] + psi2 * b2_m[1]) / TWOPI};
    (void)b00;
    cplx ff[5] = {mk(1, 0), mk(1, 0), cis(-psi1), mk(1, 0), cis(-psi2)};

    /* Per unique pair: the 3x3 unflagged edge contributions plus self-pair data. */
    cplx *zb = malloc(sizeof(cplx) * 9 * (size_t)nufp);
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t iu = 0; iu < nufp; ++iu) {
        int64_t fp = ufp_rep[iu] - 1;
        int64_t ifm = fp % nface, ifs = fp / nface;
        double rs[3][2], rm[3][2];
        for (int k = 0; k < 3; ++k) {
            vtx(rho, fv, ifs, k, rs[k]); vtx(rho, fv, ifm, k, rm[k]);
            rs[k][0] /= units_per_meter; rs[k][1] /= units_per_meter;
            rm[k][0] /= units_per_meter; rm[k][1] /= units_per_meter;
        }
        double rmc[2] = {((rm[0][0] + rm[1][0]) + rm[2][0]) / 3, ((rm[0][1] + rm[1][1]) + rm[2][1]) / 3};
        /* zint (Zint.jl:218-245) */
        cplx I1 = 0, I1x = 0, I1e = 0, I2 = 0;
        for (int i = 0; i < 7; ++i) {
            double rt[2] = {(rs[0][0] + (rs[1][0] - rs[0][0]) * QXI[i]) + (rs[2][0] - rs[0][0]) * QETA[i],
                            (rs[0][1] + (rs[1][1] - rs[0][1]) * QXI[i]) + (rs[2][1] - rs[0][1]) * QETA[i]};
            double rd[2] = {rmc[0] - rt[0], rmc[1] - rt[1]};
            cplx g1 = ora_sigma(tab1, mmax, b1_m, b2_m, psi1, psi2, rd);
            cplx g2 = ora_sigma(tab2, mmax, b1_m, b2_m, psi1, psi2, rd);
            cplx g1w = rmul(QW[i], g1);
            I1x = cadd(I1x, rmul(QXI[i], g1w));
            I1e = cadd(I1e, rmul(QETA[i], g1w));
            I1 = cadd(I1, g1w);
            I2 = cadd(I2, rmul(QW[i], g2));
        }
        cplx J = JKJ[iu], Jx = JKJxi[iu], Je = JKJeta[iu];
        cplx K = JKK[iu], Kx = JKKxi[iu], Ke = JKKeta[iu];
        double rinv = JKrinv[iu], rr[2] = {JKrho_r[2 * iu], JKrho_r[2 * iu + 1]};
        cplx I1z = csub(csub(I1, I1x), I1e), Jz = csub(csub(J, Jx), Je), Kz = csub(csub(K, Kx), Ke);
        double rc2[3][2];
        for (int i = 0; i < 3; ++i) {
            rc2[i][0] = 0.5 * (rmc[0] - rm[i][0]);
            rc2[i][1] = 0.5 * (rmc[1] - rm[i][1]);
        }
        cplx phi;
        if (!magnetic)
            phi = cadd(cadd(rmul(FOURPI, I2), rmul(u, cadd(mk(rinv, 0), J))), cmul(cdivr(d3, u), K));
        else
            phi = cadd(cadd(cmul(I2fact, I2), rmul(u, cadd(mk(rinv, 0), J))), cmul(KPfact, K));
        for (int isl = 0; isl < 3; ++isl) {
            double sing[2] = {rr[0] + (u * rinv) * (rmc[0] - rs[isl][0]),
                              rr[1] + (u * rinv) * (rmc[1] - rs[isl][1])};
            cplx av[2];
            for (int d = 0; d < 2; ++d) {
                cplx Ii = csub(cadd(cadd(rmul(rs[0][d], I1x), rmul(rs[1][d], I1e)), rmul(rs[2][d], I1z)), rmul(rs[isl][d], I1));
                cplx Ji = csub(cadd(cadd(rmul(rs[0][d], Jx), rmul(rs[1][d], Je)), rmul(rs[2][d], Jz)), rmul(rs[isl][d], J));
                cplx Ki = csub(cadd(cadd(rmul(rs[0][d], Kx), rmul(rs[1][d], Ke)), rmul(rs[2][d], Kz)), rmul(rs[isl][d], K));
                if (!magnetic)
                    av[d] = cadd(cadd(cadd(rmul(FOURPI, Ii), mk(sing[d], 0)), rmul(u, Ji)), cmul(cdivr(c3, u), Ki));
                else
                    av[d] = cadd(cadd(cadd(cmul(I1fact, Ii), mk(sing[d], 0)), rmul(u, Ji)), cmul(KFfact, Ki));
            }
            for (int iml = 0; iml < 3; ++iml) {
                cplx dp = cadd(rmul(rc2[iml][0], av[0]), rmul(rc2[iml][1], av[1]));
                cplx val;
                if (!magnetic) {
                    /* match_flag*source_flag * (iω (μ0 μ̃/4π) ρc2·a  -  i/(ϵ̄ 2π ω ϵ0) φ) */
                    cplx A = cmul(rmul(MU0 / FOURPI, mutilde), dp);
                    cplx P = cmul(cdiv(mk(0, 1), epsbar), cdivr(phi, TWOPI * omega * eps0));
                    val = csub(cmul(mk(0, omega), A), P);
                } else {
                    cplx F = cmul(rmul(-eps0 / PI, epsbar), dp);
                    cplx P = cmul(cdiv(mk(0, 2), cmul(rmul(PI * omega * MU0, mk(1, 0)), mutilde)), phi);
                    val = csub(cmul(mk(0, -omega), F), P);
                }
                zb[9 * iu + 3 * isl + iml] = val;
            }
        }
    }

    /* Assembly: every face pair (m = match, n = source) scatters its 3x3 edge terms. */
    memset(Z, 0, sizeof(cplx) * (size_t)nbf * nbf);
    for (int64_t fs = 0; fs < nface; ++fs) {
        for (int64_t fm = 0; fm < nface; ++fm) {
            int64_t iu = ufpm[fm + fs * nface] - 1;
            const cplx *zc = zb + 9 * iu;
            int self_tri = (fm == fs);
            double ls[3] = {0, 0, 0}, area48 = 0;
            if (self_tri) {
                double r[3][2];
                for (int k = 0; k < 3; ++k) {
                    vtx(rho, fv, fs, k, r[k]);
                    r[k][0] /= units_per_meter; r[k][1] /= units_per_meter;
                }
                double a32[2] = {r[2][0] - r[1][0], r[2][1] - r[1][1]};
                double a12[2] = {r[0][0] - r[1][0], r[0][1] - r[1][1]};
                double a13[2] = {r[0][0] - r[2][0], r[0][1] - r[2][1]};
                ls[0] = sqrt(a32[0] * a32[0] + a32[1] * a32[1]);
                ls[1] = sqrt(a13[0] * a13[0] + a13[1] * a13[1]);
                ls[2] = sqrt(a12[0] * a12[0] + a12[1] * a12[1]);
                area48 = 48 * fabs(0.5 * (a32[0] * a12[1] - a32[1] * a12[0]));
            }
            for (int isl = 0; isl < 3; ++isl) {
                int64_t es = fe[3 * fs + isl];
                int64_t sbf = ebf[es - 1];
                if (sbf == 0) continue;
                cplx sflag = ff[eci[es - 1]];
                if (bff[2 * (sbf - 1)] - 1 == fs) { /* plus */ }
                else if (bff[2 * (sbf - 1) + 1] - 1 == fs) sflag = mk(-creal(sflag), -cimag(sflag));
                for (int iml = 0; iml < 3; ++iml) {
                    int64_t em = fe[3 * fm + iml];
                    int64_t mbf = ebf[em - 1];
                    if (mbf == 0) continue;
                    cplx mflag = conj(ff[eci[em - 1]]);
                    if (bff[2 * (mbf - 1)] - 1 == fm) { }
                    else if (bff[2 * (mbf - 1) + 1] - 1 == fm) mflag = mk(-creal(mflag), -cimag(mflag));
                    cplx v = cmul(cmul(mflag, sflag), zc[3 * isl + iml]);
                    if (!magnetic && self_tri && fr[fm] != 0) {
                        if (em == es) {
                            double l1 = ls[next[isl]], l2 = ls[prev[isl]], l0 = ls[isl];
                            v = cadd(v, mk(fr[fs] / area48 * (3 * (l1 * l1 + l2 * l2) - l0 * l0), 0));
                        } else {
                            double lt = ls[third[isl][iml]];
                            double g = ls[isl] * ls[isl] + ls[iml] * ls[iml] - 3 * (lt * lt);
                            v = cadd(v, rmul(g, cmul(rmul(fr[fs] / area48, sflag), mflag)));
                        }
                    }
                    size_t idx = (size_t)(mbf - 1) + (size_t)(sbf - 1) * nbf;
                    Z[idx] = cadd(Z[idx], v);
                }
            }
        }
    }
    free(zb);
}

static double j0s(double x) {
    if (fabs(x) < 1e-3) { double x2 = x * x; return 1 - x2 / 6 * (1 - x2 / 20); }
    return sin(x) / x;
}
static double j1s(double x) {
    if (fabs(x) < 1e-3) return x * (1.0 / 3 - x * x / 30);
    double s = sin(x), c = cos(x);
    return (s / x - c) / x;
}

/* RWG.jl:428-512 -- Fourier transforms of all basis functions at transform variable k
 * (1/m).  ft is nbf x 2 complex (x and y components interleaved per basis function). */
void ora_rwgbfft(int64_t nface, const double *rho, const int64_t *fv, const int64_t *fe,
                 int64_t nbf, const int64_t *bff, const int64_t *ebf, const int64_t *eci,
                 double one_meter, const double k[2], double psi1, double psi2, cplx *ft) {
    const int nxt[3] = {1, 2, 0};
    cplx ff[5] = {mk(1, 0), mk(1, 0), cis(-psi1), mk(1, 0), cis(-psi2)};
    memset(ft, 0, sizeof(cplx) * 2 * (size_t)nbf);
    double kmagsq = k[0] * k[0] + k[1] * k[1];
    double kmag = sqrt(kmagsq);
    for (int64_t f = 0; f < nface; ++f) {
        double r[3][2], lv[3][2], rc[3][2];
        for (int q = 0; q < 3; ++q) { vtx(rho, fv, f, q, r[q]); r[q][0] /= one_meter; r[q][1] /= one_meter; }
        double lmax = 0;
        for (int q = 0; q < 3; ++q) {
            lv[q][0] = r[nxt[q]][0] - r[q][0];
            lv[q][1] = r[nxt[q]][1] - r[q][1];
            rc[q][0] = r[q][0] + 0.5 * lv[q][0];
            rc[q][1] = r[q][1] + 0.5 * lv[q][1];
            double ln = sqrt(lv[q][0] * lv[q][0] + lv[q][1] * lv[q][1]);
            if (ln > lmax) lmax = ln;
        }
        if (kmag * lmax < 1e-4) {
            double cen[2] = {((r[0][0] + r[1][0]) + r[2][0]) / 3, ((r[0][1] + r[1][1]) + r[2][1]) / 3};
            cplx cph = cis(k[0] * cen[0] + k[1] * cen[1]);
            for (int i = 0; i < 3; ++i) {
                int64_t ie = fe[3 * f + i];
                int64_t ib = ebf[ie - 1];
                if (ib == 0) continue;
                double f0[2] = {0.5 * (cen[0] - r[i][0]), 0.5 * (cen[1] - r[i][1])};
                cplx w = cmul(cph, ff[eci[ie - 1]]);
                double sg = (bff[2 * (ib - 1)] - 1 == f) ? 1.0 : -1.0;
                for (int d = 0; d < 2; ++d) {
                    cplx t = rmul(f0[d], w);
                    ft[2 * (ib - 1) + d] = sg > 0 ? cadd(ft[2 * (ib - 1) + d], t) : csub(ft[2 * (ib - 1) + d], t);
                }
            }
        } else {
            double kf[2] = {2 * k[0] / kmagsq, 2 * k[1] / kmagsq};
            double darea = lv[0][0] * lv[1][1] - lv[0][1] * lv[1][0];
            double denom = darea * kmagsq;
            double zl[3], j0k[3], rt2[3][2];
            cplx ct1[3][2], cph[3];
            for (int n = 0; n < 3; ++n) {
                zl[n] = lv[n][0] * k[1] - lv[n][1] * k[0];
                ct1[n][0] = mk(-kf[0], rc[n][0]);
                ct1[n][1] = mk(-kf[1], rc[n][1]);
                double dk = 0.5 * (k[0] * lv[n][0] + k[1] * lv[n][1]);
                j0k[n] = j0s(dk);
                double jj = j1s(dk);
                rt2[n][0] = ((0.5 * zl[n]) * jj) * lv[n][0];
                rt2[n][1] = ((0.5 * zl[n]) * jj) * lv[n][1];
                cph[n] = cis(k[0] * rc[n][0] + k[1] * rc[n][1]);
            }
            for (int i = 0; i < 3; ++i) {
                int64_t ie = fe[3 * f + i];
                int64_t ib = ebf[ie - 1];
                if (ib == 0) continue;
                cplx cs[2] = {0, 0};
                for (int n = 0; n < 3; ++n) {
                    double zc[2] = {-lv[n][1], lv[n][0]};
                    for (int d = 0; d < 2; ++d) {
                        cplx cj = mk(0.0, r[i][d]);
                        cplx c3t = rmul(j0k[n], cadd(mk(zc[d], 0), rmul(zl[n], csub(ct1[n][d], cj))));
                        cs[d] = cadd(cs[d], cmul(cph[n], csub(c3t, mk(rt2[n][d], 0))));
                    }
                }
                cplx w = cdivr(ff[eci[ie - 1]], denom);
                double sg = (bff[2 * (ib - 1)] - 1 == f) ? 1.0 : -1.0;
                for (int d = 0; d < 2; ++d) {
                    cplx t = cmul(cs[d], w);
                    ft[2 * (ib - 1) + d] = sg > 0 ? cadd(ft[2 * (ib - 1) + d], t) : csub(ft[2 * (ib - 1) + d], t);
                }
            }
        }
    }
}
