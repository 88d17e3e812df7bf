/*
 * hw_oracle2d.c -- CPU restatement of the HAWASSI 2D flat-bottom RHS and its
 * gsl_odeiv2 rkf45 stepping (TEST INFRASTRUCTURE ONLY, see hw_oracle2d.h).
 *
 * Every transform is the full complex 2D DFT the reference runs through FFTW
 * (fftw_plan_dft_2d, unnormalised); the symmetrisation before each inverse
 * transform, the real parts taken after it, the complex intermediate of
 * fun_adjust and the order of the pointwise products follow the reference's
 * statements one by one.
 */
#include "hw_oracle2d.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static const double GRAV = 9.80665;   /* 2d/var_initialization.h:246 */
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

void or_fft(int n, const double* re_in, const double* im_in, double* re_out, double* im_out, int sign);
void or_cspline_coeffs(int n, const double* x, const double* y, double* c_out);
double or_cspline_eval(int n, const double* x, const double* y, const double* c, double t);

static char g_err2[512];
const char* or2d_last_error(void) { return g_err2; }
static void set_err2(const char* fmt, ...) {
    va_list ap; va_start(ap, fmt); vsnprintf(g_err2, sizeof g_err2, fmt, ap); va_end(ap);
}

typedef struct { double re, im; } cx;

struct or2d_ctx {
    int nx, ny, n, model, prop, nt;
    double cpeak, eps_abs, eps_rel;
    double *kx, *ky, *c2d, *l2d, *aal, *charac, *chiadj, *newgam, *skewgam;
    double *tsig, *sig, *sigskew, *csig, *csigskew;   /* spline second-derivative coefficients */
    int var;                                           /* varying bottom (two reference depths) */
    double *gmin, *gplus, *cmin, *cplus, *omin, *oplus;
    double *gmid, *cmid, *omid;                        /* three reference depths, NULL: two */
    int nk;                                            /* K reference depths (0: min/plus/mid tables) */
    double *gk, *ck, *ok;                              /* [K][n] weights, C^2, Omega^2 */
    double* wallchar;                                  /* NULL: no wall */
    int refl_one;                                      /* flat bottom, refl_coef == 1 */
    double *gwx, *gwy;                                 /* fun_gradient(wallchar) (refl_one) */
    struct brk2* brk;                                  /* kinematic breaking, NULL: off */
    long long rhs_calls, acc, rej;
    /* rkf45 work vectors */
    double *k1, *k2, *k3, *k4, *k5, *k6, *ytmp, *y0, *yerr, *dydt_in, *dydt_out;
};

struct brk2;
static struct brk2* brk_create(const or2d_tables* tb);
static void fun_gradient2(const double* f, int Nx, int Ny, double dx, double dy, double* gx, double* gy);
static void brk_destroy(struct brk2* b);

static double* dup(const double* a, size_t n) {
    double* p = (double*)malloc(sizeof(double) * n);
    memcpy(p, a, sizeof(double) * n);
    return p;
}

/* ------------------------------------------------------------------------ */
/* 2D DFT = 1D transforms over rows, then over columns (FFTW's 2D result).   */
/* ------------------------------------------------------------------------ */
static void fft2(int nx, int ny, cx* a, int sign) {
    int m = nx > ny ? nx : ny;
    double *ri = malloc(sizeof(double) * m), *ii = malloc(sizeof(double) * m);
    double *ro = malloc(sizeof(double) * m), *io = malloc(sizeof(double) * m);
    for (int i = 0; i < ny; i++) {
        for (int j = 0; j < nx; j++) { ri[j] = a[i * nx + j].re; ii[j] = a[i * nx + j].im; }
        or_fft(nx, ri, ii, ro, io, sign);
        for (int j = 0; j < nx; j++) { a[i * nx + j].re = ro[j]; a[i * nx + j].im = io[j]; }
    }
    for (int j = 0; j < nx; j++) {
        for (int i = 0; i < ny; i++) { ri[i] = a[i * nx + j].re; ii[i] = a[i * nx + j].im; }
        or_fft(ny, ri, ii, ro, io, sign);
        for (int i = 0; i < ny; i++) { a[i * nx + j].re = ro[i]; a[i * nx + j].im = io[i]; }
    }
    free(ri); free(ii); free(ro); free(io);
}

void or2d_fft(int nx, int ny, const double* re_in, const double* im_in, double* re_out, double* im_out, int sign) {
    int n = nx * ny;
    cx* a = malloc(sizeof(cx) * n);
    for (int q = 0; q < n; q++) { a[q].re = re_in[q]; a[q].im = im_in ? im_in[q] : 0.0; }
    fft2(nx, ny, a, sign);
    for (int q = 0; q < n; q++) { re_out[q] = a[q].re; im_out[q] = a[q].im; }
    free(a);
}

/* fftwcomplex_2d_sym (2d/functions1.c:492-521), called there with (Nxy, Nt) =
 * (Nx, Ny): the right half of every row is overwritten by the conjugate mirror
 * of the left half, column 0 below row Ny/2 by the mirror of its upper half, and
 * the four self-conjugate points lose their imaginary parts.  Column Nx/2 is left
 * as it is (rows other than 0 and Ny/2). */
static void sym2(cx* a, int Nxy, int Nt) {
    a[0].im = 0;
    a[0 * Nxy + (Nxy / 2)].im = 0;
    a[Nt / 2 * Nxy].im = 0;
    a[Nt / 2 * Nxy + (Nxy / 2)].im = 0;
    for (int j = 1; j < Nxy / 2; j++) {
        a[Nxy - j].re = a[j].re;
        a[Nxy - j].im = -a[j].im;
        a[Nt / 2 * Nxy + Nxy - j].re = a[Nt / 2 * Nxy + j].re;
        a[Nt / 2 * Nxy + Nxy - j].im = -a[Nt / 2 * Nxy + j].im;
    }
    for (int i = 1; i < Nt / 2; i++) {
        a[(Nt - i) * Nxy].re = a[i * Nxy].re;
        a[(Nt - i) * Nxy].im = -a[i * Nxy].im;
    }
    int it = 1;
    for (int i = 1; i < Nt; i++) {
        int iy = 1;
        for (int j = Nxy / 2 + 1; j < Nxy; j++) {
            a[i * Nxy + j].re = a[(Nt - it) * Nxy + Nxy / 2 - iy].re;
            a[i * Nxy + j].im = -a[(Nt - it) * Nxy + Nxy / 2 - iy].im;
            iy++;
        }
        it++;
    }
}

void or2d_sym(int nx, int ny, double* re, double* im) {
    int n = nx * ny;
    cx* a = malloc(sizeof(cx) * n);
    for (int q = 0; q < n; q++) { a[q].re = re[q]; a[q].im = im[q]; }
    sym2(a, nx, ny);
    for (int q = 0; q < n; q++) { re[q] = a[q].re; im[q] = a[q].im; }
    free(a);
}

/* ------------------------------------------------------------------------ */
or2d_ctx* or2d_create(const or2d_tables* tb, double eps_abs, double eps_rel) {
    if (!tb || tb->nx < 4 || tb->ny < 4 || (tb->nx & 1) || (tb->ny & 1)) {
        set_err2("or2d_create: grid must be even and at least 4x4");
        return NULL;
    }
    if (tb->model < 1 || tb->model > 3) { set_err2("or2d_create: model must be 1 (HS1), 2 (HS2) or 3 (HS3)"); return NULL; }
    or2d_ctx* c = calloc(1, sizeof(or2d_ctx));
    c->nx = tb->nx; c->ny = tb->ny; c->n = tb->nx * tb->ny;
    c->model = tb->model; c->prop = tb->propagation; c->cpeak = tb->cpeak;
    c->eps_abs = eps_abs > 0 ? eps_abs : 1e-3;
    c->eps_rel = eps_rel > 0 ? eps_rel : 1e-2;
    size_t n = (size_t)c->n;
    c->kx = dup(tb->kx, c->nx); c->ky = dup(tb->ky, c->ny);
    c->c2d = dup(tb->c2d, n); c->l2d = dup(tb->l2d, n); c->aal = dup(tb->aal, n);
    c->charac = dup(tb->charac, n); c->chiadj = dup(tb->chiadj, n);
    c->nt = (tb->sig && tb->newgam && tb->tsig) ? tb->nt : 0;
    if (c->nt > 0) {
        c->newgam = dup(tb->newgam, n);
        c->skewgam = tb->skewgam ? dup(tb->skewgam, n) : calloc(n, sizeof(double));
        c->tsig = dup(tb->tsig, c->nt);
        c->sig = dup(tb->sig, n / c->nx * c->nt);
        c->sigskew = tb->sigskew ? dup(tb->sigskew, (size_t)c->ny * c->nt) : calloc((size_t)c->ny * c->nt, sizeof(double));
        c->csig = malloc(sizeof(double) * (size_t)c->ny * c->nt);
        c->csigskew = malloc(sizeof(double) * (size_t)c->ny * c->nt);
        for (int i = 0; i < c->ny; i++) {
            or_cspline_coeffs(c->nt, c->tsig, c->sig + (size_t)i * c->nt, c->csig + (size_t)i * c->nt);
            or_cspline_coeffs(c->nt, c->tsig, c->sigskew + (size_t)i * c->nt, c->csigskew + (size_t)i * c->nt);
        }
    }
    if (tb->gam_min && tb->gam_plus && tb->csq_min && tb->csq_plus && tb->om2_min && tb->om2_plus) {
        c->var = 1;
        c->gmin = dup(tb->gam_min, n); c->gplus = dup(tb->gam_plus, n);
        c->cmin = dup(tb->csq_min, n); c->cplus = dup(tb->csq_plus, n);
        c->omin = dup(tb->om2_min, n); c->oplus = dup(tb->om2_plus, n);
        if (tb->gam_mid || tb->csq_mid || tb->om2_mid) {
            if (!(tb->gam_mid && tb->csq_mid && tb->om2_mid)) {
                set_err2("or2d_create: three reference depths need gam_mid, csq_mid and om2_mid"); free(c); return NULL;
            }
            c->gmid = dup(tb->gam_mid, n); c->cmid = dup(tb->csq_mid, n); c->omid = dup(tb->om2_mid, n);
        }
    }
    if (tb->nrefk) {
        if (tb->nrefk < 2 || tb->nrefk > 16 || !tb->gam_k || !tb->csq_k || !tb->om2_k) {
            set_err2("or2d_create: K reference depths need 2 <= K <= 16 and gam_k, csq_k, om2_k"); free(c); return NULL;
        }
        c->var = 1;
        c->nk = tb->nrefk;
        c->gk = dup(tb->gam_k, (size_t)c->nk * n);
        c->ck = dup(tb->csq_k, (size_t)c->nk * n);
        c->ok = dup(tb->om2_k, (size_t)c->nk * n);
    }
    if (tb->wallchar) {
        c->wallchar = dup(tb->wallchar, n);
        if (!c->var && tb->refl_coef == 1) {
            if (!(tb->dx > 0) || !(tb->dy > 0)) { set_err2("or2d_create: walls with refl_coef 1 need dx, dy"); free(c); return NULL; }
            c->refl_one = 1;
            c->gwx = malloc(sizeof(double) * n); c->gwy = malloc(sizeof(double) * n);
            fun_gradient2(c->wallchar, c->nx, c->ny, tb->dx, tb->dy, c->gwx, c->gwy);   /* 2d/functions.c:741 */
        }
    }
    if (tb->breaking) {
        if (c->model == 1) { set_err2("or2d_create: breaking is restated for the HS2 and HS3 RHS only"); free(c); return NULL; }
        if (!tb->bathy || !tb->brchar || !tb->x || !tb->y) { set_err2("or2d_create: breaking tables missing"); free(c); return NULL; }
        c->brk = brk_create(tb);
    }
    return c;
}

/* the rkf45 work vectors, allocated by the first evolve_apply (an RHS-only
 * context, as the CPU baseline's threads use, needs none) */
static void ensure_rk(or2d_ctx* c) {
    if (c->k1) return;
    size_t d = 6 * (size_t)c->n;
    double** w[] = {&c->k1, &c->k2, &c->k3, &c->k4, &c->k5, &c->k6, &c->ytmp, &c->y0, &c->yerr, &c->dydt_in, &c->dydt_out};
    for (size_t q = 0; q < sizeof w / sizeof w[0]; q++) *w[q] = calloc(d, sizeof(double));
}

void or2d_destroy(or2d_ctx* c) {
    if (!c) return;
    double* f[] = {c->kx, c->ky, c->c2d, c->l2d, c->aal, c->charac, c->chiadj, c->newgam, c->skewgam, c->tsig,
                   c->sig, c->sigskew, c->csig, c->csigskew, c->k1, c->k2, c->k3, c->k4, c->k5, c->k6, c->ytmp,
                   c->y0, c->yerr, c->dydt_in, c->dydt_out, c->gmin, c->gplus, c->cmin, c->cplus, c->omin,
                   c->oplus, c->wallchar, c->gwx, c->gwy, c->gmid, c->cmid, c->omid, c->gk, c->ck, c->ok};
    for (size_t q = 0; q < sizeof f / sizeof f[0]; q++) free(f[q]);
    brk_destroy(c->brk);
    free(c);
}

void or2d_stats(const or2d_ctx* c, long long* r, long long* a, long long* j) {
    if (r) *r = c->rhs_calls;
    if (a) *a = c->acc;
    if (j) *j = c->rej;
}

/* ------------------------------------------------------------------------ */
/* fun_adjust (2d/fun_odesolver.c:810-833): symmetrise Ahat in place, complex
 * inverse transform, multiply both parts by ChiAdj/(Nx*Ny), forward transform. */
static void fun_adjust(const or2d_ctx* c, cx* AChi_hat, cx* Ahat) {
    int Nx = c->nx, Ny = c->ny, n = c->n;
    cx* A = malloc(sizeof(cx) * n);
    sym2(Ahat, Nx, Ny);
    memcpy(A, Ahat, sizeof(cx) * n);
    fft2(Nx, Ny, A, +1);
    for (int i = 0; i < Ny; i++)
        for (int j = 0; j < Nx; j++) {
            AChi_hat[i * Nx + j].re = (A[i * Nx + j].re * c->chiadj[i * Nx + j] / (Nx * Ny));
            AChi_hat[i * Nx + j].im = (A[i * Nx + j].im * c->chiadj[i * Nx + j] / (Nx * Ny));
        }
    fft2(Nx, Ny, AChi_hat, -1);
    free(A);
}

/* fun_source (2d/fun_odesolver.c:886-983), vertical influx line: one signal per
 * row, Source[i][j] = INsig_t[i] newGam[j][i] (twice that for Bi), SkewSource =
 * -/+ INsig_skew_t[i] SkewGam[j][i] for Uni+/Uni- (0 for Bi); Source_hat is the
 * sum of the two forward transforms. */
static void fun_source(const or2d_ctx* c, double t, cx* Source_hat) {
    int Nx = c->nx, Ny = c->ny, n = c->n;
    if (c->nt <= 0) { memset(Source_hat, 0, sizeof(cx) * n); return; }
    double* ins = malloc(sizeof(double) * Ny);
    double* inss = malloc(sizeof(double) * Ny);
    for (int j = 0; j < Ny; j++) {
        ins[j] = or_cspline_eval(c->nt, c->tsig, c->sig + (size_t)j * c->nt, c->csig + (size_t)j * c->nt, t);
        inss[j] = or_cspline_eval(c->nt, c->tsig, c->sigskew + (size_t)j * c->nt, c->csigskew + (size_t)j * c->nt, t);
    }
    cx* S0 = malloc(sizeof(cx) * n);
    cx* SS = malloc(sizeof(cx) * n);
    for (int i = 0; i < Ny; i++)
        for (int j = 0; j < Nx; j++) {
            double src, skew;
            if (c->prop == 0) { src = ins[i] * c->newgam[i * Nx + j]; skew = -1 * inss[i] * c->skewgam[i * Nx + j]; }
            else if (c->prop == 1) { src = ins[i] * c->newgam[i * Nx + j]; skew = 1 * inss[i] * c->skewgam[i * Nx + j]; }
            else { src = 2 * ins[i] * c->newgam[i * Nx + j]; skew = 0; }
            S0[i * Nx + j].re = src; S0[i * Nx + j].im = 0;
            SS[i * Nx + j].re = skew; SS[i * Nx + j].im = 0;
        }
    fft2(Nx, Ny, S0, -1);
    fft2(Nx, Ny, SS, -1);
    for (int q = 0; q < n; q++) {
        Source_hat[q].re = S0[q].re + SS[q].re;
        Source_hat[q].im = S0[q].im + SS[q].im;
    }
    free(ins); free(inss); free(S0); free(SS);
}


/* HSSgen_2depth (2d/fun_odesolver.c:500-586): with phi the unnormalised physical
 * field (its real part used) and phihat its spectrum,
 * result = [F(gam_min Re F^-1 S(Op_min phihat)) + Op_min F(gam_min phi)
 *           + F(gam_plus Re F^-1 S(Op_plus phihat)) + Op_plus F(gam_plus phi)] / 2 */
/* HSSgen_3depth (2d/fun_odesolver.c:588-697): the two-depth operator with the middle
 * depth's round trip and spectral term between the outer ones' */
static void hssgen_3depth(const or2d_ctx* c, const cx* phi, const cx* phihat, const double* Om, const double* Oc,
                          const double* Op, cx* result) {
    const int Nx = c->nx, Ny = c->ny, n = c->n;
    const double factIFFT = (double)Nx * Ny;
    const double* O[3] = {Om, Oc, Op};
    const double* G[3] = {c->gmin, c->gmid, c->gplus};
    cx *L0[3], *g[3], *gL[3];
    for (int d = 0; d < 3; d++) {
        L0[d] = malloc(sizeof(cx) * n);
        for (int q = 0; q < n; q++) { L0[d][q].re = O[d][q] * phihat[q].re; L0[d][q].im = O[d][q] * phihat[q].im; }
        sym2(L0[d], Nx, Ny);
        fft2(Nx, Ny, L0[d], +1);
    }
    for (int d = 0; d < 3; d++) {
        g[d] = malloc(sizeof(cx) * n); gL[d] = malloc(sizeof(cx) * n);
        for (int q = 0; q < n; q++) {
            g[d][q].re = G[d][q] * phi[q].re / factIFFT; g[d][q].im = 0;
            gL[d][q].re = G[d][q] * L0[d][q].re / (Nx * Ny); gL[d][q].im = 0;
        }
    }
    for (int d = 0; d < 3; d++) fft2(Nx, Ny, g[d], -1);
    for (int d = 0; d < 3; d++) fft2(Nx, Ny, gL[d], -1);
    for (int q = 0; q < n; q++) {
        result[q].re = (gL[0][q].re + Om[q] * g[0][q].re + gL[1][q].re + Oc[q] * g[1][q].re + gL[2][q].re
                        + Op[q] * g[2][q].re) / 2;
        result[q].im = (gL[0][q].im + Om[q] * g[0][q].im + gL[1][q].im + Oc[q] * g[1][q].im + gL[2][q].im
                        + Op[q] * g[2][q].im) / 2;
    }
    for (int d = 0; d < 3; d++) { free(L0[d]); free(g[d]); free(gL[d]); }
}

/* The K-reference-depth operator (no counterpart in the reference): HSSgen_3depth's
 * sum over K depths, result = 1/2 sum_j [F(gam_j Re F^-1 S(O_j phihat)) + O_j F(gam_j phi)],
 * summed in the same order (j ascending, round-trip term then spectral term); with K = 2
 * and K = 3 and the same tables it is HSSgen_2depth / HSSgen_3depth bit for bit.
 * O = c->ck (C^2) or c->ok (Omega^2), [K][n]. */
static void hssgen_k(const or2d_ctx* c, const cx* phi, const cx* phihat, const double* O, cx* result) {
    const int Nx = c->nx, Ny = c->ny, n = c->n, K = c->nk;
    const double factIFFT = (double)Nx * Ny;
    cx* L0 = malloc(sizeof(cx) * n);
    cx* g = malloc(sizeof(cx) * n);
    cx* gL = malloc(sizeof(cx) * n);
    for (int q = 0; q < n; q++) { result[q].re = 0; result[q].im = 0; }
    for (int d = 0; d < K; d++) {
        const double* Od = O + (size_t)d * n;
        const double* Gd = c->gk + (size_t)d * n;
        for (int q = 0; q < n; q++) { L0[q].re = Od[q] * phihat[q].re; L0[q].im = Od[q] * phihat[q].im; }
        sym2(L0, Nx, Ny);
        fft2(Nx, Ny, L0, +1);
        for (int q = 0; q < n; q++) {
            g[q].re = Gd[q] * phi[q].re / factIFFT; g[q].im = 0;
            gL[q].re = Gd[q] * L0[q].re / (Nx * Ny); gL[q].im = 0;
        }
        fft2(Nx, Ny, g, -1);
        fft2(Nx, Ny, gL, -1);
        for (int q = 0; q < n; q++) {
            result[q].re = result[q].re + gL[q].re + Od[q] * g[q].re;
            result[q].im = result[q].im + gL[q].im + Od[q] * g[q].im;
        }
    }
    for (int q = 0; q < n; q++) { result[q].re /= 2; result[q].im /= 2; }
    free(L0); free(g); free(gL);
}

static void hssgen_2depth(const or2d_ctx* c, const cx* phi, const cx* phihat, const double* Om, const double* Op,
                          cx* result) {
    const int Nx = c->nx, Ny = c->ny, n = c->n;
    const double factIFFT = (double)Nx * Ny;
    cx *L0m = malloc(sizeof(cx) * n), *L0p = malloc(sizeof(cx) * n);
    for (int q = 0; q < n; q++) {
        L0m[q].re = Om[q] * phihat[q].re; L0m[q].im = Om[q] * phihat[q].im;
        L0p[q].re = Op[q] * phihat[q].re; L0p[q].im = Op[q] * phihat[q].im;
    }
    sym2(L0m, Nx, Ny); sym2(L0p, Nx, Ny);
    fft2(Nx, Ny, L0m, +1); fft2(Nx, Ny, L0p, +1);
    cx *gm = malloc(sizeof(cx) * n), *gp = malloc(sizeof(cx) * n);
    cx *gmL = malloc(sizeof(cx) * n), *gpL = malloc(sizeof(cx) * n);
    for (int q = 0; q < n; q++) {
        gm[q].re = c->gmin[q] * phi[q].re / factIFFT; gm[q].im = 0;
        gp[q].re = c->gplus[q] * phi[q].re / factIFFT; gp[q].im = 0;
        gmL[q].re = c->gmin[q] * L0m[q].re / (Nx * Ny); gmL[q].im = 0;
        gpL[q].re = c->gplus[q] * L0p[q].re / (Nx * Ny); gpL[q].im = 0;
    }
    fft2(Nx, Ny, gm, -1); fft2(Nx, Ny, gp, -1); fft2(Nx, Ny, gmL, -1); fft2(Nx, Ny, gpL, -1);
    for (int q = 0; q < n; q++) {
        result[q].re = (gmL[q].re + Om[q] * gm[q].re + gpL[q].re + Op[q] * gp[q].re) / 2;
        result[q].im = (gmL[q].im + Om[q] * gm[q].im + gpL[q].im + Op[q] * gp[q].im) / 2;
    }
    free(L0m); free(L0p); free(gm); free(gp); free(gmL); free(gpL);
}

/* ------------------------------------------------------------------------ */
/* Kinematic breaking of the 2D model: parambreak, breaking_process and its   */
/* helpers (2d/breaking.c:1-733) and fun_sbreaking (2d/fun_odesolver.c:      */
/* 985-1019).  The crest records keep the reference's fields and its use of  */
/* slots (CB, CBNew, CBPrev with NB in slot 0; the continuing crests' break  */
/* nodes and every crest's nodes written to CBPrev slots counted separately);*/
/* node lists grow as needed where the reference's are 100 entries long.     */
/* ------------------------------------------------------------------------ */
typedef struct { int x, y; } v2i;
typedef struct {
    int xindex, yindex, xNow, yNow, kwadran, NB;
    double Ucrest, time, theta;
    v2i* nodes; int nnode, cap;          /* break nodes (B > 0) of a continuing crest */
    v2i* nodes_prev; int nnode_prev, cap_prev;   /* every node inside the crest's sector */
} crest2;

struct brk2 {
    int nx, ny, n;
    double *bathy, *pbchar, *x, *y;
    double dx, dy, max_eta_init, tstar, rsearch, kbc, tc, delb, cur_u, t0, dt_out;
    double tprev;
    int flagbr, iterbdt;
    double *B, *U, *etah, *work;         /* B and the per-call physical fields */
    cx *sbx, *sby;                        /* Sb_xhat, Sb_yhat (persist between calls) */
    crest2 *CB, *CBNew, *CBPrev;
    int capCB, capNew, capPrev;
    v2i *bn, *bnp;                        /* Break_nodes, Break_nodes_prev */
    int nbreak_nodes, nbreak_prev;
    /* breaking.dat records */
    double* log_t; int* log_cnt; int nrec, caprec;
    v2i* log_nodes; long long nlog, caplog;
};

static struct brk2* brk_create(const or2d_tables* tb) {
    struct brk2* b = calloc(1, sizeof(struct brk2));
    b->nx = tb->nx; b->ny = tb->ny; b->n = tb->nx * tb->ny;
    size_t n = (size_t)b->n;
    b->bathy = dup(tb->bathy, n); b->pbchar = dup(tb->brchar, n);
    b->x = dup(tb->x, b->nx); b->y = dup(tb->y, b->ny);
    b->dx = tb->dx; b->dy = tb->dy;
    b->max_eta_init = tb->max_eta_init; b->tstar = tb->tstar; b->rsearch = tb->rsearch;
    b->kbc = tb->kbc; b->tc = tb->tc; b->delb = tb->delb; b->cur_u = tb->cur_u;
    b->t0 = tb->t0; b->dt_out = tb->dt_out;
    b->tprev = tb->t0;                    /* tprev = dominfo.t[0] (2d/main.c:120) */
    b->B = calloc(n, sizeof(double)); b->U = calloc(n, sizeof(double));
    b->etah = calloc(n, sizeof(double)); b->work = calloc(4 * n, sizeof(double));
    b->sbx = calloc(n, sizeof(cx)); b->sby = calloc(n, sizeof(cx));
    b->bn = malloc(sizeof(v2i) * n); b->bnp = malloc(sizeof(v2i) * n);
    return b;
}

static void crest_free(crest2* a, int cap) {
    for (int i = 0; i < cap; i++) { free(a[i].nodes); free(a[i].nodes_prev); }
    free(a);
}

static void brk_destroy(struct brk2* b) {
    if (!b) return;
    free(b->bathy); free(b->pbchar); free(b->x); free(b->y);
    free(b->B); free(b->U); free(b->etah); free(b->work); free(b->sbx); free(b->sby);
    crest_free(b->CB, b->capCB); crest_free(b->CBNew, b->capNew); crest_free(b->CBPrev, b->capPrev);
    free(b->bn); free(b->bnp); free(b->log_t); free(b->log_cnt); free(b->log_nodes);
    free(b);
}

static crest2* crest_reserve(crest2* a, int* cap, int need) {
    if (need <= *cap) return a;
    int nc = *cap ? *cap : 16;
    while (nc < need) nc *= 2;
    a = realloc(a, sizeof(crest2) * nc);
    memset(a + *cap, 0, sizeof(crest2) * (nc - *cap));
    *cap = nc;
    return a;
}

/* copy of the scalar fields (the reference's field-by-field copies) */
static void crest_copy(crest2* d, const crest2* s) {
    d->xindex = s->xindex; d->yindex = s->yindex; d->xNow = s->xNow; d->yNow = s->yNow;
    d->Ucrest = s->Ucrest; d->theta = s->theta; d->time = s->time; d->NB = s->NB; d->kwadran = s->kwadran;
}

static int fun_sign2(double v) { return v < 0 ? -1 : 1; }   /* 2d/functions1.c:170 */

/* fun_kwadran (2d/breaking.c:199-213) */
static int fun_kwadran(double ux, double uy) {
    if ((ux >= 0) && (uy >= 0)) return 1;
    else if ((ux < 0) && (uy >= 0)) return 2;
    else if ((ux < 0) && (uy < 0)) return 3;
    return 4;
}

/* fun_exact_Cp1d_val (2d/functions.c:70-80) */
static double exact_cp(double k, double D, double U) {
    if (k == 0) return sqrt(GRAV * D) + U;
    return (fun_sign2(k) * sqrt(GRAV * k * tanh(k * D)) + k * U) / k;
}

/* gradient2D (2d/functions1.c:868-885) at one point: one-sided at the edges */
static double grad_x_at(const double* a, int nx, int i, int j, double dx) {
    if (j == 0) return (a[i * nx + 1] - a[i * nx]) / dx;
    if (j == nx - 1) return (a[i * nx + nx - 1] - a[i * nx + nx - 2]) / dx;
    return (a[i * nx + j + 1] - a[i * nx + j - 1]) / (2 * dx);
}
static double grad_y_at(const double* a, int nx, int ny, int i, int j, double dy) {
    if (i == 0) return (a[nx + j] - a[j]) / dy;
    if (i == ny - 1) return (a[(ny - 1) * nx + j] - a[(ny - 2) * nx + j]) / dy;
    return (a[(i + 1) * nx + j] - a[(i - 1) * nx + j]) / (2 * dy);
}

/* fun_peaks (2d/breaking.c:56-136), called with (ROWS, COLS) = (Nx, Ny): "row"
 * is the x index, "col" the y index; interior points first (x outer), then the
 * x = 0 edge, the x = Nx-1 edge, the y = 0 edge and the y = Ny-1 edge. */
static int fun_peaks(const struct brk2* b, const double* A, int* pk) {
    const int Nx = b->nx, Ny = b->ny;
    const double thr = b->max_eta_init;
    int np = 0;
#define AT(yy, xx) A[(yy) * Nx + (xx)]
    for (int row = 1; row < Nx - 1; row++)
        for (int col = 1; col < Ny - 1; col++) {
            int cnt = 0;
            for (int i = -1; i < 2; i++)
                for (int j = -1; j < 2; j++) cnt += (AT(col + i, row + j) - AT(col, row) <= 0.001) ? 1 : 0;
            if (cnt == 9 && AT(col, row) > thr) { pk[2 * np] = row; pk[2 * np + 1] = col; np++; }
        }
    for (int e = 0; e < 4; e++) {
        const int along_x = e >= 2;                 /* y edges run along x */
        const int len = along_x ? Nx : Ny;
        for (int m = 1; m < len - 1; m++) {
            int row, col, i0, i1, j0, j1;
            if (e == 0) { row = 0; col = m; i0 = -1; i1 = 2; j0 = 0; j1 = 2; }
            else if (e == 1) { row = Nx - 1; col = m; i0 = -1; i1 = 2; j0 = -1; j1 = 1; }
            else if (e == 2) { col = 0; row = m; i0 = 0; i1 = 2; j0 = -1; j1 = 2; }
            else { col = Ny - 1; row = m; i0 = -1; i1 = 1; j0 = -1; j1 = 2; }
            int cnt = 0;
            for (int i = i0; i < i1; i++)
                for (int j = j0; j < j1; j++) cnt += (AT(col + i, row + j) - AT(col, row) <= 0.001) ? 1 : 0;
            if (cnt == 6 && AT(col, row) > thr) { pk[2 * np] = row; pk[2 * np + 1] = col; np++; }
        }
    }
#undef AT
    return np;
}

/* breaking_criterion (2d/breaking.c:215-326): candidates into CB, NB in CB[0] */
static void brk_criterion(struct brk2* b, double t, const double* Zhat, const double* kx, const double* ky,
                          const cx* gpx, const cx* gpy) {
    const int Nx = b->nx, Ny = b->ny, n = b->n;
    double* chk = b->work;
    for (int q = 0; q < n; q++) chk[q] = b->etah[q] * b->pbchar[q];
    double mx = chk[0];
    for (int q = 0; q < n; q++) mx = (mx > chk[q] ? mx : chk[q]);
    if (!(mx > b->max_eta_init)) return;
    int* pk = malloc(sizeof(int) * 2 * (size_t)n);
    const int npk = fun_peaks(b, chk, pk);
    if (npk == 0) { free(pk); return; }
    /* HilbEta: Re = Im(eta^) sign(kx + ky), Im = -Re(eta^) sign, symmetrised, inverse */
    cx* H = malloc(sizeof(cx) * n);
    for (int i = 0; i < Ny; i++)
        for (int j = 0; j < Nx; j++) {
            const int q = i * Nx + j;
            const int s = fun_sign2(kx[j] + ky[i]);
            H[q].re = Zhat[n + q] * s;
            H[q].im = -Zhat[q] * s;
        }
    sym2(H, Nx, Ny);
    fft2(Nx, Ny, H, +1);
    double* Hr = b->work + n;
    for (int q = 0; q < n; q++) Hr[q] = H[q].re / (Nx * Ny);
    free(H);
    int it = 0;
    for (int p = 0; p < npk; p++) {
        const int ix = pk[2 * p], iy = pk[2 * p + 1], q = iy * Nx + ix;
        const double e = b->etah[q], h = Hr[q];
        const double gxH = grad_x_at(Hr, Nx, iy, ix, b->dx), gyH = grad_y_at(Hr, Nx, Ny, iy, ix, b->dy);
        const double gxE = grad_x_at(b->etah, Nx, iy, ix, b->dx), gyE = grad_y_at(b->etah, Nx, Ny, iy, ix, b->dy);
        const double Kx = (e * gxH - h * gxE) / (pow(e, 2) + pow(h, 2));
        const double Ky = (e * gyH - h * gyE) / (pow(e, 2) + pow(h, 2));
        const double Kk = sqrt(pow(Kx, 2) + pow(Ky, 2));
        const double Cc = exact_cp(Kk, -b->bathy[q] + e, b->cur_u);
        if (fabs(b->U[q]) >= (b->kbc * fabs(Cc))) {
            b->CB = crest_reserve(b->CB, &b->capCB, it + 1);
            crest2* r = &b->CB[it];
            r->xindex = ix; r->yindex = iy; r->xNow = ix; r->yNow = iy;
            r->Ucrest = fabs(b->U[q]); r->time = t;
            r->theta = fabs(atan(gpy[q].re / gpx[q].re));
            r->kwadran = fun_kwadran(gpx[q].re, gpy[q].re);
            it++;
        }
    }
    free(pk);
    if (b->capCB > 0) b->CB[0].NB = it;
}

/* fun_check_crest (2d/breaking.c:328-349) */
static int check_crest(const struct brk2* b, int k, int ncbprev) {
    const int idx = b->CB[k].xindex, idy = b->CB[k].yindex;
    for (int l = 0; l < ncbprev; l++)
        if (b->CBPrev[l].xindex == idx && b->CBPrev[l].yindex == idy) return 0;
    for (int l = 0; l < ncbprev; l++)
        for (int m = 0; m < b->CBPrev[l].nnode; m++)
            if (b->CBPrev[l].nodes[m].x == idx && b->CBPrev[l].nodes[m].y == idy) return 0;
    return 1;
}

/* funBr_Char (2d/breaking.c:351-441) at one point: inside the search disc and the
 * 160-degree sector of the crest's quadrant */
static int crest_char(const struct brk2* b, const crest2* r, int i, int j) {
    const double xp = b->x[r->xNow], yp = b->y[r->yNow];
    const double xc = b->x[j] - xp, yc = b->y[i] - yp;
    if (!((pow(xc, 2) + pow(yc, 2)) <= pow(b->rsearch, 2))) return 0;
    const double spread = 80.0, theta = r->theta;
    double alpha, beta;
    if (r->kwadran == 1 || r->kwadran == 3) {
        alpha = theta - spread * M_PI / 180.0;
        beta = (spread * M_PI / 180.0 + theta) - M_PI / 2.0;
    } else {
        alpha = spread * M_PI / 180.0 - theta;
        beta = (M_PI / 2.0 - theta) - (spread * M_PI / 180.0);
    }
    const double XXr = (b->x[j] - xp) * cos(alpha) + (b->y[i] - yp) * sin(alpha);
    const double YYr = (b->y[i] - yp) * cos(beta) - (b->x[j] - xp) * sin(beta);
    switch (r->kwadran) {
        case 1: if ((XXr < 0) || (YYr < 0)) return 0; break;
        case 2: if ((XXr > 0) || (YYr < 0)) return 0; break;
        case 3: if ((XXr > 0) || (YYr > 0)) return 0; break;
        default: if ((XXr < 0) || (YYr > 0)) return 0; break;
    }
    return 1;
}

/* funBr_find_peak_loc + idx_max_matrix (2d/breaking.c:443-454, 2d/functions1.c:248-262) */
static void find_peak_loc(const struct brk2* b, const crest2* r, int* ix, int* iy) {
    const int Nx = b->nx, Ny = b->ny;
    double temp = b->etah[0] * crest_char(b, r, 0, 0) * b->pbchar[0];
    *ix = -1; *iy = -1;
    for (int i = 0; i < Ny; i++)
        for (int j = 0; j < Nx; j++) {
            const double v = b->etah[i * Nx + j] * crest_char(b, r, i, j) * b->pbchar[i * Nx + j];
            if (v > temp) { temp = v; *ix = j; *iy = i; }
        }
}

/* funBr_BreakNodes_char (2d/breaking.c:456-503) */
static void break_nodes(struct brk2* b, const crest2* r, double Ustar, double UF) {
    const int Nx = b->nx, Ny = b->ny;
    int id = 0, idp = 0;
    for (int i = 0; i < Ny; i++)
        for (int j = 0; j < Nx; j++) {
            const int q = i * Nx + j;
            double ch = crest_char(b, r, i, j);
            if ((b->U[q] < UF) || (b->etah[q] < 0)) ch = 0;
            ch = ch * b->pbchar[q];
            if (ch == 1) {
                b->bnp[idp].x = j; b->bnp[idp].y = i; idp++;
                if (b->B[q] == 0) {
                    if (b->U[q] >= (2 * Ustar)) b->B[q] = 1;
                    else if (b->U[q] <= Ustar) b->B[q] = 0;
                    else b->B[q] = ((b->U[q] / Ustar) - 1);
                    if (b->B[q] > 0) { b->bn[id].x = j; b->bn[id].y = i; id++; }
                }
            }
        }
    b->nbreak_nodes = id;
    b->nbreak_prev = idp;
}

static void set_nodes(v2i** dst, int* cnt, int* cap, const v2i* src, int m) {
    if (m > *cap) { *dst = realloc(*dst, sizeof(v2i) * m); *cap = m; }
    memcpy(*dst, src, sizeof(v2i) * m);
    *cnt = m;
}

/* breaking_process (2d/breaking.c:505-733) */
static void brk_process(or2d_ctx* c, double t, const double* Zhat, const cx* eta, const cx* u, const cx* v) {
    struct brk2* b = c->brk;
    const int n = c->n;
    const double fact = (double)c->nx * c->ny;
    for (int q = 0; q < n; q++) {
        b->etah[q] = eta[q].re / fact;
        b->U[q] = sqrt(pow(u[q].re / fact, 2) + pow(v[q].re / fact, 2));
    }
    b->CB = crest_reserve(b->CB, &b->capCB, 1);
    b->CB[0].NB = 0;
    memset(b->B, 0, sizeof(double) * n);
    brk_criterion(b, t, Zhat, c->kx, c->ky, u, v);
    const int NCB = b->CB[0].NB;
    if ((NCB > 0) && (b->flagbr == 0)) {
        b->flagbr = 1;
        b->CBNew = crest_reserve(b->CBNew, &b->capNew, NCB);
        for (int j = 0; j < NCB; j++) crest_copy(&b->CBNew[j], &b->CB[j]);
    } else if ((NCB == 0) && (b->flagbr == 2)) {
        const int ncp = b->CBPrev[0].NB;
        b->CBNew = crest_reserve(b->CBNew, &b->capNew, ncp > 0 ? ncp : 1);
        for (int j = 0; j < ncp; j++) crest_copy(&b->CBNew[j], &b->CBPrev[j]);
        b->CBNew[0].NB = ncp;
    } else if ((NCB > 0) && (b->flagbr == 2)) {
        const int ncp = b->CBPrev[0].NB;
        b->CBNew = crest_reserve(b->CBNew, &b->capNew, ncp + NCB);
        for (int j = 0; j < ncp; j++) crest_copy(&b->CBNew[j], &b->CBPrev[j]);
        int add = 0;
        for (int k = 0; k < NCB; k++)
            if (check_crest(b, k, ncp) == 1) {
                crest2* d = &b->CBNew[ncp + add];
                const crest2* s = &b->CB[k];
                d->xindex = s->xindex; d->yindex = s->yindex; d->xNow = s->xNow; d->yNow = s->yNow;
                d->Ucrest = s->Ucrest; d->time = s->time; d->theta = s->theta; d->kwadran = s->kwadran;
                add++;
            }
        b->CBNew[0].NB = ncp + add;
    }
    if ((b->flagbr == 1) || (b->flagbr == 2)) {
        const int ncnow = b->CBNew[0].NB;
        b->CBPrev = crest_reserve(b->CBPrev, &b->capPrev, ncnow > 0 ? ncnow : 1);
        b->CBPrev[0].NB = 0;
        int* term = calloc(ncnow > 0 ? ncnow : 1, sizeof(int));
        int itpp = 0, itp = 0;
        for (int lx = 0; lx < ncnow; lx++) {
            crest2* r = &b->CBNew[lx];
            term[lx] = 0;
            if (b->flagbr == 1) {
                r->xNow = r->xindex;
                r->yNow = r->yindex;
            } else {
                int mx, my;
                find_peak_loc(b, r, &mx, &my);
                if (mx < 0) { term[lx] = 1; continue; }
                r->xNow = mx;
                r->yNow = my;
                const int q = my * c->nx + mx;
                r->theta = fabs(atan(v[q].re / u[q].re));
                r->kwadran = fun_kwadran(u[q].re, v[q].re);
            }
            const double tbreak = r->time, UI = r->Ucrest, UF = b->tc * UI;
            double Ustar;
            if ((t - tbreak) >= b->tstar) Ustar = UF;
            else if (((t - tbreak) >= 0) && (t - tbreak) < b->tstar) Ustar = UI + ((t - tbreak) / b->tstar) * (UF - UI);
            else Ustar = UI;
            break_nodes(b, r, Ustar, UF);
            if (b->nbreak_prev > 0) {
                crest2* d = &b->CBPrev[itpp];
                set_nodes(&d->nodes_prev, &d->nnode_prev, &d->cap_prev, b->bnp, b->nbreak_prev);
                itpp++;
            }
            if (b->nbreak_nodes == 0) {
                term[lx] = 1;
            } else {
                term[lx] = 0;
                crest2* d = &b->CBPrev[itp];
                set_nodes(&d->nodes, &d->nnode, &d->cap, b->bn, b->nbreak_nodes);
                d->xindex = r->xindex; d->yindex = r->yindex; d->xNow = r->xNow; d->yNow = r->yNow;
                d->Ucrest = r->Ucrest; d->time = r->time; d->theta = r->theta; d->kwadran = r->kwadran;
                itp++;
            }
            b->CBPrev[0].NB = itp;
        }
        for (int lx = 0; lx < ncnow; lx++) {
            if (term[lx] == 0) { b->flagbr = 2; break; }
            else b->flagbr = 0;
        }
        if ((t > b->t0 + b->iterbdt * b->dt_out) && (itpp > 0)) {
            long long m = 0;
            for (int lx = 0; lx < itpp; lx++) m += b->CBPrev[lx].nnode_prev;
            if (b->nrec + 1 > b->caprec) {
                b->caprec = b->caprec ? 2 * b->caprec : 64;
                b->log_t = realloc(b->log_t, sizeof(double) * b->caprec);
                b->log_cnt = realloc(b->log_cnt, sizeof(int) * b->caprec);
            }
            if (b->nlog + m > b->caplog) {
                while (b->nlog + m > b->caplog) b->caplog = b->caplog ? 2 * b->caplog : 4096;
                b->log_nodes = realloc(b->log_nodes, sizeof(v2i) * b->caplog);
            }
            b->log_t[b->nrec] = t;
            b->log_cnt[b->nrec] = (int)m;
            for (int lx = 0; lx < itpp; lx++) {
                memcpy(b->log_nodes + b->nlog, b->CBPrev[lx].nodes_prev, sizeof(v2i) * b->CBPrev[lx].nnode_prev);
                b->nlog += b->CBPrev[lx].nnode_prev;
            }
            b->nrec++;
        }
        free(term);
    }
    if (t > b->t0 + b->iterbdt * b->dt_out) b->iterbdt = b->iterbdt + 1;
}

/* fun_gradient (2d/functions.c:392-460): periodic forward and backward
 * differences, the forward ones clipped to <= 0, the backward ones to >= 0, summed */
static void fun_gradient2(const double* f, int Nx, int Ny, double dx, double dy, double* gx, double* gy) {
    for (int i = 0; i < Ny; i++)
        for (int j = 0; j < Nx; j++) {
            const int q = i * Nx + j;
            double Fx = (j < Nx - 1) ? (f[q + 1] - f[q]) / dx : (f[i * Nx] - f[q]) / dx;
            double Fy = (i < Ny - 1) ? (f[q + Nx] - f[q]) / dy : (f[j] - f[q]) / dy;
            double Bx = (j > 0) ? (f[q] - f[q - 1]) / dx : (f[q] - f[i * Nx + Nx - 1]) / dx;
            double By = (i > 0) ? (f[q] - f[q - Nx]) / dy : (f[q] - f[(Ny - 1) * Nx + j]) / dy;
            if (Fx > 0) Fx = 0;
            if (Fy > 0) Fy = 0;
            if (Bx < 0) Bx = 0;
            if (By < 0) By = 0;
            gx[q] = Fx + Bx;
            gy[q] = Fy + By;
        }
}

/* fun_sbreaking (2d/fun_odesolver.c:985-1019); delphiH_hat is symmetrised in
 * place (ifftw_2d_c2r, 2d/functions1.c:523-559), which the RHS's assembly then sees */
static void brk_force(or2d_ctx* c, const cx* eta, cx* dphi) {
    struct brk2* b = c->brk;
    const int Nx = c->nx, Ny = c->ny, n = c->n;
    const double fact = (double)Nx * Ny;
    sym2(dphi, Nx, Ny);
    cx* d = malloc(sizeof(cx) * n);
    memcpy(d, dphi, sizeof(cx) * n);
    fft2(Nx, Ny, d, +1);
    double* flux = b->work;
    double* gx = b->work + n;
    double* gy = b->work + 2 * n;
    for (int q = 0; q < n; q++) {
        const double dp = d[q].re / (Nx * Ny);
        flux[q] = -b->B[q] * pow(b->delb, 2) * (eta[q].re / fact - b->bathy[q]) * pow(dp, 2);
    }
    fun_gradient2(flux, Nx, Ny, b->dx, b->dy, gx, gy);
    for (int q = 0; q < n; q++) {
        const double hq = eta[q].re / fact - b->bathy[q];
        b->sbx[q].re = gx[q] / hq; b->sbx[q].im = 0;
        b->sby[q].re = gy[q] / hq; b->sby[q].im = 0;
    }
    fft2(Nx, Ny, b->sbx, -1);
    fft2(Nx, Ny, b->sby, -1);
    free(d);
}

void or2d_set_tprev(or2d_ctx* c, double tprev) {
    if (c && c->brk) c->brk->tprev = tprev;
}

int or2d_brk_fields(const or2d_ctx* c, double* B, double* sbx, double* sby, int* flagbr, int* ncrest) {
    if (!c || !c->brk) return -1;
    const struct brk2* b = c->brk;
    if (B) memcpy(B, b->B, sizeof(double) * b->n);
    if (sbx) memcpy(sbx, b->sbx, sizeof(cx) * b->n);
    if (sby) memcpy(sby, b->sby, sizeof(cx) * b->n);
    if (flagbr) *flagbr = b->flagbr;
    if (ncrest) *ncrest = (b->flagbr == 2 && b->capPrev > 0) ? b->CBPrev[0].NB : 0;
    return 0;
}

int or2d_brk_log(const or2d_ctx* c, double* times, int* cnt, int* nodes, int cap_rec, int cap_nodes) {
    if (!c || !c->brk) return -1;
    const struct brk2* b = c->brk;
    long long off = 0;
    for (int r = 0; r < b->nrec && r < cap_rec; r++) {
        if (times) times[r] = b->log_t[r];
        if (cnt) cnt[r] = b->log_cnt[r];
        for (int m = 0; m < b->log_cnt[r]; m++, off++)
            if (nodes && off < cap_nodes) { nodes[2 * off] = b->log_nodes[off].x; nodes[2 * off + 1] = b->log_nodes[off].y; }
    }
    return b->nrec;
}

long long or2d_brk_log_nodes(const or2d_ctx* c) { return (c && c->brk) ? c->brk->nlog : -1; }

/* rhs_AB2_2DB_uv (2d/fun_odesolver.c:4542-4626) with fun_termshat_AB1_2DB_uv
 * (:2874-2960) and fun_termshat_AB2_2DB_uv (:3327-3510), ninterp = 2; walls enter
 * through dominfo.wallchar in the H2 products (:3416-3430); kinematic breaking
 * (breaking_process, fun_sbreaking) when the tables ask for it; no friction or
 * coupling. */
static int rhs_2db(or2d_ctx* c, double t, const double* Zhat, double* dt_Zhat) {
    const int Nx = c->nx, Ny = c->ny, n = c->n;
    const double factIFFT = (double)Nx * Ny;
    const double* kx = c->kx;
    const double* ky = c->ky;
    c->rhs_calls++;
    /* AB1: symmetrised copies, inverse transforms, HSS of u^ and v^ with Csqr */
    cx *eta_hat = malloc(sizeof(cx) * n), *u_hat = malloc(sizeof(cx) * n), *v_hat = malloc(sizeof(cx) * n);
    for (int q = 0; q < n; q++) {
        eta_hat[q].re = Zhat[q]; eta_hat[q].im = Zhat[n + q];
        u_hat[q].re = Zhat[2 * n + q]; u_hat[q].im = Zhat[3 * n + q];
        v_hat[q].re = Zhat[4 * n + q]; v_hat[q].im = Zhat[5 * n + q];
    }
    sym2(eta_hat, Nx, Ny); sym2(u_hat, Nx, Ny); sym2(v_hat, Nx, Ny);
    cx *eta = malloc(sizeof(cx) * n), *u = malloc(sizeof(cx) * n), *v = malloc(sizeof(cx) * n);
    memcpy(eta, eta_hat, sizeof(cx) * n); memcpy(u, u_hat, sizeof(cx) * n); memcpy(v, v_hat, sizeof(cx) * n);
    fft2(Nx, Ny, eta, +1); fft2(Nx, Ny, u, +1); fft2(Nx, Ny, v, +1);
    cx *Csqr_uhat = malloc(sizeof(cx) * n), *Csqr_vhat = malloc(sizeof(cx) * n);
    if (c->nk) {
        hssgen_k(c, u, u_hat, c->ck, Csqr_uhat);
        hssgen_k(c, v, v_hat, c->ck, Csqr_vhat);
    } else if (c->gmid) {   /* ninterp = 3 (2d/fun_odesolver.c:2917-2920) */
        hssgen_3depth(c, u, u_hat, c->cmin, c->cmid, c->cplus, Csqr_uhat);
        hssgen_3depth(c, v, v_hat, c->cmin, c->cmid, c->cplus, Csqr_vhat);
    } else {
        hssgen_2depth(c, u, u_hat, c->cmin, c->cplus, Csqr_uhat);
        hssgen_2depth(c, v, v_hat, c->cmin, c->cplus, Csqr_vhat);
    }
    const double sevenC = 7 * c->cpeak;
    cx *dampeta = malloc(sizeof(cx) * n), *dampu = malloc(sizeof(cx) * n), *dampv = malloc(sizeof(cx) * n);
    cx *deluH1 = malloc(sizeof(cx) * n), *delvH1 = malloc(sizeof(cx) * n);
    for (int i = 0; i < Ny; i++)
        for (int j = 0; j < Nx; j++) {
            const int q = i * Nx + j;
            const double ch = c->charac[q];
            dampeta[q].re = sevenC * ch * eta[q].re / factIFFT; dampeta[q].im = 0;
            dampu[q].re = sevenC * ch * u[q].re / factIFFT; dampu[q].im = 0;
            dampv[q].re = sevenC * ch * v[q].re / factIFFT; dampv[q].im = 0;
            deluH1[q].re = Csqr_uhat[q].im / GRAV * kx[j];
            deluH1[q].im = -Csqr_uhat[q].re / GRAV * kx[j];
            delvH1[q].re = Csqr_vhat[q].im / GRAV * ky[i];
            delvH1[q].im = -Csqr_vhat[q].re / GRAV * ky[i];
        }
    fft2(Nx, Ny, dampeta, -1); fft2(Nx, Ny, dampu, -1); fft2(Nx, Ny, dampv, -1);
    free(eta_hat); free(u_hat); free(v_hat); free(Csqr_uhat); free(Csqr_vhat);

    if (c->model == 1) {
        /* rhs_AB1_2DB_uv (2d/fun_odesolver.c:4350-4402): the linear model */
        cx* Source_hat = malloc(sizeof(cx) * n);
        fun_source(c, t, Source_hat);
        for (int i = 0; i < Ny; i++)
            for (int j = 0; j < Nx; j++) {
                const int q = i * Nx + j;
                const double a = c->aal[q];
                dt_Zhat[q] = (Source_hat[q].re + deluH1[q].re + delvH1[q].re - dampeta[q].re) * a;
                dt_Zhat[n + q] = (Source_hat[q].im + deluH1[q].im + delvH1[q].im - dampeta[q].im) * a;
                dt_Zhat[2 * n + q] = (GRAV * kx[j] * Zhat[n + q] - dampu[q].re) * a;
                dt_Zhat[3 * n + q] = (-GRAV * kx[j] * Zhat[q] - dampu[q].im) * a;
                dt_Zhat[4 * n + q] = (GRAV * ky[i] * Zhat[n + q] - dampv[q].re) * a;
                dt_Zhat[5 * n + q] = (-GRAV * ky[i] * Zhat[q] - dampv[q].im) * a;
            }
        cx* fr1[] = {eta, u, v, dampeta, dampu, dampv, deluH1, delvH1, Source_hat};
        for (size_t q = 0; q < sizeof fr1 / sizeof fr1[0]; q++) free(fr1[q]);
        for (int q = 0; q < 6 * n; q++)
            if (!isfinite(dt_Zhat[q])) return 1;
        return 0;
    }

    /* AB2: the physical fields again (same transforms as AB1), M0 u = delu H1 */
    cx *M0u = malloc(sizeof(cx) * n), *M0v = malloc(sizeof(cx) * n), *Lphi = malloc(sizeof(cx) * n);
    for (int q = 0; q < n; q++) {
        M0u[q] = deluH1[q];
        M0v[q] = delvH1[q];
        Lphi[q].re = deluH1[q].re + delvH1[q].re;
        Lphi[q].im = deluH1[q].im + delvH1[q].im;
    }
    sym2(M0u, Nx, Ny); sym2(M0v, Nx, Ny); sym2(Lphi, Nx, Ny);
    fft2(Nx, Ny, M0u, +1); fft2(Nx, Ny, M0v, +1); fft2(Nx, Ny, Lphi, +1);
    const double f2 = pow(factIFFT, 2);
    cx *etaM0u = malloc(sizeof(cx) * n), *eta_u = malloc(sizeof(cx) * n), *etaM0v = malloc(sizeof(cx) * n);
    cx *eta_v = malloc(sizeof(cx) * n), *deletaH2 = malloc(sizeof(cx) * n);
    for (int q = 0; q < n; q++) {
        const double wallchar = c->wallchar ? c->wallchar[q] : 1.0;
        etaM0u[q].re = eta[q].re * M0u[q].re / f2 * wallchar; etaM0u[q].im = 0;
        eta_u[q].re = eta[q].re * u[q].re / f2 * wallchar; eta_u[q].im = 0;
        etaM0v[q].re = eta[q].re * M0v[q].re / f2 * wallchar; etaM0v[q].im = 0;
        eta_v[q].re = eta[q].re * v[q].re / f2 * wallchar; eta_v[q].im = 0;
        deletaH2[q].re = 0.5 * ((pow(u[q].re, 2) + pow(v[q].re, 2)) - pow(Lphi[q].re, 2)) / f2 * wallchar;
        deletaH2[q].im = 0;
    }
    cx *etaM0uhat = malloc(sizeof(cx) * n), *etaM0vhat = malloc(sizeof(cx) * n);
    memcpy(etaM0uhat, etaM0u, sizeof(cx) * n); memcpy(etaM0vhat, etaM0v, sizeof(cx) * n);
    fft2(Nx, Ny, etaM0uhat, -1); fft2(Nx, Ny, eta_u, -1); fft2(Nx, Ny, etaM0vhat, -1);
    fft2(Nx, Ny, eta_v, -1); fft2(Nx, Ny, deletaH2, -1);
    for (int q = 0; q < n; q++) {   /* "for operator": back to the unnormalised scale HSSgen divides out */
        etaM0u[q].re = etaM0u[q].re * factIFFT;
        etaM0v[q].re = etaM0v[q].re * factIFFT;
    }
    cx *LetaM0u = malloc(sizeof(cx) * n), *LetaM0v = malloc(sizeof(cx) * n);
    if (c->nk) {
        hssgen_k(c, etaM0u, etaM0uhat, c->ok, LetaM0u);
        hssgen_k(c, etaM0v, etaM0vhat, c->ok, LetaM0v);
    } else if (c->gmid) {   /* ninterp = 3 (:3463-3466) */
        hssgen_3depth(c, etaM0u, etaM0uhat, c->omin, c->omid, c->oplus, LetaM0u);
        hssgen_3depth(c, etaM0v, etaM0vhat, c->omin, c->omid, c->oplus, LetaM0v);
    } else {
        hssgen_2depth(c, etaM0u, etaM0uhat, c->omin, c->oplus, LetaM0u);
        hssgen_2depth(c, etaM0v, etaM0vhat, c->omin, c->oplus, LetaM0v);
    }
    cx *ikx = malloc(sizeof(cx) * n), *iky = malloc(sizeof(cx) * n);
    cx *delu = malloc(sizeof(cx) * n), *delv = malloc(sizeof(cx) * n);
    for (int i = 0; i < Ny; i++)
        for (int j = 0; j < Nx; j++) {
            const int q = i * Nx + j;
            ikx[q].re = -kx[j] * deletaH2[q].im; ikx[q].im = kx[j] * deletaH2[q].re;
            iky[q].re = -ky[i] * deletaH2[q].im; iky[q].im = ky[i] * deletaH2[q].re;
            delu[q].re = kx[j] * eta_u[q].im - LetaM0u[q].re / GRAV;
            delu[q].im = -kx[j] * eta_u[q].re - LetaM0u[q].im / GRAV;
            delv[q].re = ky[i] * eta_v[q].im - LetaM0v[q].re / GRAV;
            delv[q].im = -ky[i] * eta_v[q].re - LetaM0v[q].im / GRAV;
        }
    cx *deluH2adj = malloc(sizeof(cx) * n), *delvH2adj = malloc(sizeof(cx) * n);
    cx *ikxH2adj = malloc(sizeof(cx) * n), *ikyH2adj = malloc(sizeof(cx) * n);
    fun_adjust(c, deluH2adj, delu);
    fun_adjust(c, delvH2adj, delv);
    fun_adjust(c, ikxH2adj, ikx);
    fun_adjust(c, ikyH2adj, iky);

    /* HS3: the cubic terms of fun_termshat_AB3_2DB_uv (2d/fun_odesolver.c:4104-4296),
     * the flat bottom's with L applied as HSS(.; Om2dSq) / g, the physical products
     * fed to HSS at the unnormalised scale; each adjusted on its own and added after the
     * H2 terms (rhs_AB3_2DB_uv, :4776-4829) */
    cx *deluH3adj = NULL, *delvH3adj = NULL, *ikxH3adj = NULL, *ikyH3adj = NULL;
    if (c->model == 3) {
        const double f3 = pow(factIFFT, 3);
        cx *LMu = malloc(sizeof(cx) * n), *LMv = malloc(sizeof(cx) * n), *LetaLphi = malloc(sizeof(cx) * n);
        cx *divgradphi = malloc(sizeof(cx) * n), *dxu = malloc(sizeof(cx) * n), *dyv = malloc(sizeof(cx) * n);
        cx *eta2M0u = malloc(sizeof(cx) * n), *eta2M0v = malloc(sizeof(cx) * n);
        for (int i = 0; i < Ny; i++)
            for (int j = 0; j < Nx; j++) {
                const int q = i * Nx + j;
                const double wallchar = c->wallchar ? c->wallchar[q] : 1.0;
                LMu[q].re = LetaM0u[q].re / GRAV; LMu[q].im = LetaM0u[q].im / GRAV;
                LMv[q].re = LetaM0v[q].re / GRAV; LMv[q].im = LetaM0v[q].im / GRAV;
                LetaLphi[q].re = LMu[q].re + LMv[q].re; LetaLphi[q].im = LMu[q].im + LMv[q].im;
                divgradphi[q].re = -kx[j] * Zhat[3 * n + q] - ky[i] * Zhat[5 * n + q];
                divgradphi[q].im = kx[j] * Zhat[2 * n + q] + ky[i] * Zhat[4 * n + q];
                eta2M0u[q].re = pow(eta[q].re, 2) * M0u[q].re / f3 * wallchar; eta2M0u[q].im = 0;
                eta2M0v[q].re = pow(eta[q].re, 2) * M0v[q].re / f3 * wallchar; eta2M0v[q].im = 0;
                dxu[q].re = -kx[j] * Zhat[3 * n + q]; dxu[q].im = kx[j] * Zhat[2 * n + q];
                dyv[q].re = -ky[i] * Zhat[5 * n + q]; dyv[q].im = ky[i] * Zhat[4 * n + q];
            }
        sym2(LMu, Nx, Ny); sym2(LMv, Nx, Ny); sym2(divgradphi, Nx, Ny);
        sym2(LetaLphi, Nx, Ny); sym2(dxu, Nx, Ny); sym2(dyv, Nx, Ny);
        fft2(Nx, Ny, LMu, +1); fft2(Nx, Ny, LMv, +1); fft2(Nx, Ny, divgradphi, +1);
        fft2(Nx, Ny, eta2M0u, -1); fft2(Nx, Ny, eta2M0v, -1);
        fft2(Nx, Ny, LetaLphi, +1); fft2(Nx, Ny, dxu, +1); fft2(Nx, Ny, dyv, +1);
        /* physical cubic products p[0..3] = eta L(eta M0u), eta L(eta M0v), eta^2 dx u,
         * eta^2 dy v; deletaH3 */
        cx *p[4], *ph[4], *deletaH3 = malloc(sizeof(cx) * n);
        for (int k = 0; k < 4; k++) { p[k] = malloc(sizeof(cx) * n); ph[k] = malloc(sizeof(cx) * n); }
        for (int q = 0; q < n; q++) {
            const double wallchar = c->wallchar ? c->wallchar[q] : 1.0;
            p[0][q].re = eta[q].re / factIFFT * LMu[q].re / factIFFT; p[0][q].im = 0;
            p[1][q].re = eta[q].re / factIFFT * LMv[q].re / factIFFT; p[1][q].im = 0;
            p[2][q].re = pow(eta[q].re, 2) * dxu[q].re / f3 * wallchar; p[2][q].im = 0;
            p[3][q].re = pow(eta[q].re, 2) * dyv[q].re / f3 * wallchar; p[3][q].im = 0;
            deletaH3[q].re = (Lphi[q].re / factIFFT * eta[q].re / factIFFT * divgradphi[q].re / factIFFT
                              + Lphi[q].re / factIFFT * LetaLphi[q].re / factIFFT);
            deletaH3[q].im = 0;
        }
        for (int k = 0; k < 4; k++) { memcpy(ph[k], p[k], sizeof(cx) * n); fft2(Nx, Ny, ph[k], -1); }
        fft2(Nx, Ny, deletaH3, -1);
        for (int k = 0; k < 4; k++)
            for (int q = 0; q < n; q++) p[k][q].re = p[k][q].re * factIFFT;   /* "for operator" */
        cx* Lp[4];
        for (int k = 0; k < 4; k++) {
            Lp[k] = malloc(sizeof(cx) * n);
            if (c->nk) hssgen_k(c, p[k], ph[k], c->ok, Lp[k]);
            else if (c->gmid) hssgen_3depth(c, p[k], ph[k], c->omin, c->omid, c->oplus, Lp[k]);
            else hssgen_2depth(c, p[k], ph[k], c->omin, c->oplus, Lp[k]);
        }
        cx *ikx3 = malloc(sizeof(cx) * n), *iky3 = malloc(sizeof(cx) * n);
        cx *delu3 = malloc(sizeof(cx) * n), *delv3 = malloc(sizeof(cx) * n);
        for (int i = 0; i < Ny; i++)
            for (int j = 0; j < Nx; j++) {
                const int q = i * Nx + j;
                ikx3[q].re = -kx[j] * deletaH3[q].im; ikx3[q].im = kx[j] * deletaH3[q].re;
                iky3[q].re = -ky[i] * deletaH3[q].im; iky3[q].im = ky[i] * deletaH3[q].re;
                delu3[q].re = Lp[0][q].re / GRAV + 0.5 * Lp[2][q].re / GRAV - 0.5 * (pow(kx[j], 2) * eta2M0u[q].re);
                delu3[q].im = Lp[0][q].im / GRAV + 0.5 * Lp[2][q].im / GRAV - 0.5 * (pow(kx[j], 2) * eta2M0u[q].im);
                delv3[q].re = Lp[1][q].re / GRAV + 0.5 * Lp[3][q].re / GRAV - 0.5 * (pow(ky[i], 2) * eta2M0v[q].re);
                delv3[q].im = Lp[1][q].im / GRAV + 0.5 * Lp[3][q].im / GRAV - 0.5 * (pow(ky[i], 2) * eta2M0v[q].im);
            }
        deluH3adj = malloc(sizeof(cx) * n); delvH3adj = malloc(sizeof(cx) * n);
        ikxH3adj = malloc(sizeof(cx) * n); ikyH3adj = malloc(sizeof(cx) * n);
        fun_adjust(c, deluH3adj, delu3);
        fun_adjust(c, delvH3adj, delv3);
        fun_adjust(c, ikxH3adj, ikx3);
        fun_adjust(c, ikyH3adj, iky3);
        for (int k = 0; k < 4; k++) { free(p[k]); free(ph[k]); free(Lp[k]); }
        cx* f3r[] = {LMu, LMv, LetaLphi, divgradphi, dxu, dyv, eta2M0u, eta2M0v, deletaH3, ikx3, iky3, delu3, delv3};
        for (size_t q = 0; q < sizeof f3r / sizeof f3r[0]; q++) free(f3r[q]);
    }
    cx* Source_hat = malloc(sizeof(cx) * n);
    fun_source(c, t, Source_hat);
    cx* dphi = malloc(sizeof(cx) * n);   /* delphiH_hat (2d/fun_odesolver.c:4564-4570) */
    for (int q = 0; q < n; q++) {
        dphi[q].re = deluH1[q].re + delvH1[q].re + deluH2adj[q].re + delvH2adj[q].re;
        dphi[q].im = deluH1[q].im + delvH1[q].im + deluH2adj[q].im + delvH2adj[q].im;
        if (c->model == 3) {
            dphi[q].re = deluH1[q].re + delvH1[q].re + deluH2adj[q].re + delvH2adj[q].re + deluH3adj[q].re
                         + delvH3adj[q].re;
            dphi[q].im = deluH1[q].im + delvH1[q].im + deluH2adj[q].im + delvH2adj[q].im + deluH3adj[q].im
                         + delvH3adj[q].im;
        }
    }
    /* breaking (:4578-4584): B cleared on every call, the update only past tprev;
     * Sb_xhat / Sb_yhat keep their last values otherwise */
    static const cx zero = {0.0, 0.0};
    if (c->brk) {
        memset(c->brk->B, 0, sizeof(double) * n);
        if (c->brk->tprev < t) {
            brk_process(c, t, Zhat, eta, u, v);
            brk_force(c, eta, dphi);
        }
    }
    for (int i = 0; i < Ny; i++)
        for (int j = 0; j < Nx; j++) {
            const int q = i * Nx + j;
            const double a = c->aal[q];
            const cx sbx = c->brk ? c->brk->sbx[q] : zero, sby = c->brk ? c->brk->sby[q] : zero;
            dt_Zhat[q] = (Source_hat[q].re + dphi[q].re - dampeta[q].re) * a;
            dt_Zhat[n + q] = (Source_hat[q].im + dphi[q].im - dampeta[q].im) * a;
            if (c->model == 3) {
                const cx jx = ikxH3adj[q], jy = ikyH3adj[q];
                dt_Zhat[2 * n + q] = (GRAV * kx[j] * Zhat[n + q] + sbx.re - ikxH2adj[q].re - jx.re - dampu[q].re) * a;
                dt_Zhat[3 * n + q] = (-GRAV * kx[j] * Zhat[q] + sbx.im - ikxH2adj[q].im - jx.im - dampu[q].im) * a;
                dt_Zhat[4 * n + q] = (GRAV * ky[i] * Zhat[n + q] + sby.re - ikyH2adj[q].re - jy.re - dampv[q].re) * a;
                dt_Zhat[5 * n + q] = (-GRAV * ky[i] * Zhat[q] + sby.im - ikyH2adj[q].im - jy.im - dampv[q].im) * a;
                continue;
            }
            dt_Zhat[2 * n + q] = (GRAV * kx[j] * Zhat[n + q] + sbx.re - ikxH2adj[q].re - dampu[q].re) * a;
            dt_Zhat[3 * n + q] = (-GRAV * kx[j] * Zhat[q] + sbx.im - ikxH2adj[q].im - dampu[q].im) * a;
            dt_Zhat[4 * n + q] = (GRAV * ky[i] * Zhat[n + q] + sby.re - ikyH2adj[q].re - dampv[q].re) * a;
            dt_Zhat[5 * n + q] = (-GRAV * ky[i] * Zhat[q] + sby.im - ikyH2adj[q].im - dampv[q].im) * a;
        }
    cx* fr[] = {eta, u, v, dampeta, dampu, dampv, deluH1, delvH1, M0u, M0v, Lphi, etaM0u, eta_u, etaM0v, eta_v,
                deletaH2, etaM0uhat, etaM0vhat, LetaM0u, LetaM0v, ikx, iky, delu, delv, deluH2adj, delvH2adj,
                ikxH2adj, ikyH2adj, Source_hat, dphi, deluH3adj, delvH3adj, ikxH3adj, ikyH3adj};
    for (size_t q = 0; q < sizeof fr / sizeof fr[0]; q++) free(fr[q]);
    for (int q = 0; q < 6 * n; q++)
        if (!isfinite(dt_Zhat[q])) return 1;
    return 0;
}

/* rhs_AB1_2DF_uv / rhs_AB2_2DF_uv (2d/fun_odesolver.c:4404-4540) with the term
 * functions fun_delphiH1hat (no wall, :2270-2283), fun_termshat_AB1_2DF_uv
 * (:2962-3027) and fun_termshat_AB2_2DF_uv (:3136-3325), kinematic breaking when the
 * tables ask for it (HS2), walls through fun_delphiH1hat's refl_coef < 1 branch
 * and the H2 products' wallchar; no friction or coupling. */
int or2d_rhs(or2d_ctx* c, double t, const double* Zhat, double* dt_Zhat) {
    if (c->var) return rhs_2db(c, t, Zhat, dt_Zhat);
    const int Nx = c->nx, Ny = c->ny, n = c->n;
    const double factIFFT = (double)Nx * Ny;
    const double* kx = c->kx;
    const double* ky = c->ky;
    c->rhs_calls++;
    cx* delphiH1hat = malloc(sizeof(cx) * n);
    for (int i = 0; i < Ny; i++)
        for (int j = 0; j < Nx; j++) {
            const int q = i * Nx + j;
            const double c2 = pow(c->c2d[q], 2);
            cx du = {c2 / GRAV * Zhat[2 * n + q], c2 / GRAV * Zhat[3 * n + q]};
            cx dv = {c2 / GRAV * Zhat[4 * n + q], c2 / GRAV * Zhat[5 * n + q]};
            delphiH1hat[q].re = kx[j] * du.im + ky[i] * dv.im;
            delphiH1hat[q].im = -kx[j] * du.re - ky[i] * dv.re;
        }
    if (c->wallchar && c->refl_one) {
        /* fun_delphiH1hat's branch for refl_coef == 1 (2d/fun_odesolver.c:2105-2170):
         * Flux = Re F^-1 S(C^2/g u^) / N (both components), divC2u from the symmetrised
         * spectra, delphiH1^ = F(divC2u wallchar) - F(Flux . grad wallchar) */
        cx *A = malloc(sizeof(cx) * n), *B = malloc(sizeof(cx) * n), *D = malloc(sizeof(cx) * n);
        for (int q = 0; q < n; q++) {
            const double c2 = pow(c->c2d[q], 2);
            A[q].re = c2 * Zhat[2 * n + q] / GRAV; A[q].im = c2 * Zhat[3 * n + q] / GRAV;
            B[q].re = c2 * Zhat[4 * n + q] / GRAV; B[q].im = c2 * Zhat[5 * n + q] / GRAV;
        }
        sym2(A, Nx, Ny); sym2(B, Nx, Ny);   /* ifftw_2d_c2r symmetrises its input in place */
        for (int i = 0; i < Ny; i++)
            for (int j = 0; j < Nx; j++) {
                const int q = i * Nx + j;
                D[q].re = -(-kx[j] * A[q].im - ky[i] * B[q].im);
                D[q].im = -(kx[j] * A[q].re + ky[i] * B[q].re);
            }
        sym2(D, Nx, Ny);
        fft2(Nx, Ny, A, +1); fft2(Nx, Ny, B, +1); fft2(Nx, Ny, D, +1);
        cx *W = malloc(sizeof(cx) * n), *F = malloc(sizeof(cx) * n);
        for (int q = 0; q < n; q++) {
            const double fx = A[q].re / (Nx * Ny), fy = B[q].re / (Nx * Ny), dv = D[q].re / (Nx * Ny);
            W[q].re = dv * c->wallchar[q]; W[q].im = 0;
            F[q].re = fx * c->gwx[q] + fy * c->gwy[q]; F[q].im = 0;
        }
        fft2(Nx, Ny, W, -1); fft2(Nx, Ny, F, -1);
        for (int q = 0; q < n; q++) {
            delphiH1hat[q].re = W[q].re - F[q].re;
            delphiH1hat[q].im = W[q].im - F[q].im;
        }
        free(A); free(B); free(D); free(W); free(F);
    } else if (c->wallchar) {
        /* fun_delphiH1hat's wall branch for refl_coef < 1 (2d/fun_odesolver.c:2172-2219):
         * C u^, C v^ to physical space (symmetrised, real part over N), times wallchar,
         * back (r2c), times C/g, then -i (kx . + ky .) */
        cx *Cu = malloc(sizeof(cx) * n), *Cv = malloc(sizeof(cx) * n);
        for (int q = 0; q < n; q++) {
            Cu[q].re = (c->c2d[q]) * Zhat[2 * n + q]; Cu[q].im = (c->c2d[q]) * Zhat[3 * n + q];
            Cv[q].re = (c->c2d[q]) * Zhat[4 * n + q]; Cv[q].im = (c->c2d[q]) * Zhat[5 * n + q];
        }
        sym2(Cu, Nx, Ny); sym2(Cv, Nx, Ny);
        fft2(Nx, Ny, Cu, +1); fft2(Nx, Ny, Cv, +1);
        for (int q = 0; q < n; q++) {
            Cu[q].re = Cu[q].re / (Nx * Ny) * c->wallchar[q]; Cu[q].im = 0;
            Cv[q].re = Cv[q].re / (Nx * Ny) * c->wallchar[q]; Cv[q].im = 0;
        }
        fft2(Nx, Ny, Cu, -1); fft2(Nx, Ny, Cv, -1);
        for (int i = 0; i < Ny; i++)
            for (int j = 0; j < Nx; j++) {
                const int q = i * Nx + j;
                cx du = {(c->c2d[q]) / GRAV * Cu[q].re, (c->c2d[q]) / GRAV * Cu[q].im};
                cx dv = {(c->c2d[q]) / GRAV * Cv[q].re, (c->c2d[q]) / GRAV * Cv[q].im};
                delphiH1hat[q].re = kx[j] * du.im + ky[i] * dv.im;
                delphiH1hat[q].im = -kx[j] * du.re - ky[i] * dv.re;
            }
        free(Cu); free(Cv);
    }

    /* spectra of the state, copies symmetrised before the inverse transforms */
    cx *eta = malloc(sizeof(cx) * n), *u = malloc(sizeof(cx) * n), *v = malloc(sizeof(cx) * n);
    cx *Lphi = NULL, *M0u = NULL, *M0v = NULL;
    for (int q = 0; q < n; q++) {
        eta[q].re = Zhat[q]; eta[q].im = Zhat[n + q];
        u[q].re = Zhat[2 * n + q]; u[q].im = Zhat[3 * n + q];
        v[q].re = Zhat[4 * n + q]; v[q].im = Zhat[5 * n + q];
    }
    if (c->model >= 2) {
        Lphi = malloc(sizeof(cx) * n); M0u = malloc(sizeof(cx) * n); M0v = malloc(sizeof(cx) * n);
        for (int i = 0; i < Ny; i++)
            for (int j = 0; j < Nx; j++) {
                const int q = i * Nx + j;
                const double c2 = pow(c->c2d[q], 2);
                M0u[q].re = c2 / GRAV * kx[j] * Zhat[3 * n + q];
                M0u[q].im = -c2 / GRAV * kx[j] * Zhat[2 * n + q];
                M0v[q].re = c2 / GRAV * ky[i] * Zhat[5 * n + q];
                M0v[q].im = -c2 / GRAV * ky[i] * Zhat[4 * n + q];
                Lphi[q].re = M0u[q].re + M0v[q].re;
                Lphi[q].im = M0u[q].im + M0v[q].im;
            }
    }
    sym2(eta, Nx, Ny); sym2(u, Nx, Ny); sym2(v, Nx, Ny);
    fft2(Nx, Ny, eta, +1); fft2(Nx, Ny, u, +1); fft2(Nx, Ny, v, +1);
    if (c->model >= 2) {
        sym2(Lphi, Nx, Ny); sym2(M0u, Nx, Ny); sym2(M0v, Nx, Ny);
        fft2(Nx, Ny, Lphi, +1); fft2(Nx, Ny, M0u, +1); fft2(Nx, Ny, M0v, +1);
    }

    /* physical products */
    const double sevenC = 7 * c->cpeak;
    cx *dampeta = malloc(sizeof(cx) * n), *dampu = malloc(sizeof(cx) * n), *dampv = malloc(sizeof(cx) * n);
    cx *etaM0u = NULL, *eta_u = NULL, *etaM0v = NULL, *eta_v = NULL, *deletaH2 = NULL;
    if (c->model >= 2) {
        etaM0u = malloc(sizeof(cx) * n); eta_u = malloc(sizeof(cx) * n);
        etaM0v = malloc(sizeof(cx) * n); eta_v = malloc(sizeof(cx) * n); deletaH2 = malloc(sizeof(cx) * n);
    }
    const double f2 = pow(factIFFT, 2);
    for (int q = 0; q < n; q++) {
        const double ch = c->charac[q];
        dampeta[q].re = sevenC * ch * eta[q].re / factIFFT; dampeta[q].im = 0;
        dampu[q].re = sevenC * ch * u[q].re / factIFFT; dampu[q].im = 0;
        dampv[q].re = sevenC * ch * v[q].re / factIFFT; dampv[q].im = 0;
        if (c->model >= 2) {
            const double wallchar = c->wallchar ? c->wallchar[q] : 1.0;   /* :3239-3249 */
            etaM0u[q].re = eta[q].re * M0u[q].re / f2 * wallchar; etaM0u[q].im = 0;
            eta_u[q].re = eta[q].re * u[q].re / f2 * wallchar; eta_u[q].im = 0;
            etaM0v[q].re = eta[q].re * M0v[q].re / f2 * wallchar; etaM0v[q].im = 0;
            eta_v[q].re = eta[q].re * v[q].re / f2 * wallchar; eta_v[q].im = 0;
            deletaH2[q].re = 0.5 * ((pow(u[q].re, 2) + pow(v[q].re, 2)) - pow(Lphi[q].re, 2)) / f2 * wallchar;
            deletaH2[q].im = 0;
        }
    }
    fft2(Nx, Ny, dampeta, -1); fft2(Nx, Ny, dampu, -1); fft2(Nx, Ny, dampv, -1);

    cx *ikxH2adj = NULL, *ikyH2adj = NULL, *deluH2adj = NULL, *delvH2adj = NULL;
    if (c->model >= 2) {
        fft2(Nx, Ny, etaM0u, -1); fft2(Nx, Ny, eta_u, -1); fft2(Nx, Ny, etaM0v, -1);
        fft2(Nx, Ny, eta_v, -1); fft2(Nx, Ny, deletaH2, -1);
        cx *ikx = malloc(sizeof(cx) * n), *iky = malloc(sizeof(cx) * n);
        cx *delu = malloc(sizeof(cx) * n), *delv = malloc(sizeof(cx) * n);
        for (int i = 0; i < Ny; i++)
            for (int j = 0; j < Nx; j++) {
                const int q = i * Nx + j;
                ikx[q].re = -kx[j] * deletaH2[q].im;
                ikx[q].im = kx[j] * deletaH2[q].re;
                iky[q].re = -ky[i] * deletaH2[q].im;
                iky[q].im = ky[i] * deletaH2[q].re;
                cx Lu = {c->l2d[q] * etaM0u[q].re, c->l2d[q] * etaM0u[q].im};
                cx Lv = {c->l2d[q] * etaM0v[q].re, c->l2d[q] * etaM0v[q].im};
                delu[q].re = -Lu.re + kx[j] * eta_u[q].im;
                delu[q].im = -Lu.im - kx[j] * eta_u[q].re;
                delv[q].re = -Lv.re + ky[i] * eta_v[q].im;
                delv[q].im = -Lv.im - ky[i] * eta_v[q].re;
            }
        deluH2adj = malloc(sizeof(cx) * n); delvH2adj = malloc(sizeof(cx) * n);
        ikxH2adj = malloc(sizeof(cx) * n); ikyH2adj = malloc(sizeof(cx) * n);
        fun_adjust(c, deluH2adj, delu);
        fun_adjust(c, delvH2adj, delv);
        fun_adjust(c, ikxH2adj, ikx);
        fun_adjust(c, ikyH2adj, iky);
        free(ikx); free(iky); free(delu); free(delv);
    }

    /* HS3: the cubic terms of fun_termshat_AB3_2DF_uv (2d/fun_odesolver.c:3685-3851),
     * each adjusted on its own (:3848-3851) and added after the H2 terms (:4670-4725) */
    cx *deluH3adj = NULL, *delvH3adj = NULL, *ikxH3adj = NULL, *ikyH3adj = NULL;
    if (c->model == 3) {
        const double f3 = pow(factIFFT, 3);
        cx *LetaM0u = malloc(sizeof(cx) * n), *LetaM0v = malloc(sizeof(cx) * n), *LetaLphi = malloc(sizeof(cx) * n);
        cx *divgradphi = malloc(sizeof(cx) * n), *dxu = malloc(sizeof(cx) * n), *dyv = malloc(sizeof(cx) * n);
        cx *eta2M0u = malloc(sizeof(cx) * n), *eta2M0v = malloc(sizeof(cx) * n);
        for (int i = 0; i < Ny; i++)
            for (int j = 0; j < Nx; j++) {
                const int q = i * Nx + j;
                const double L = c->l2d[q], wallchar = c->wallchar ? c->wallchar[q] : 1.0;
                LetaM0u[q].re = L * etaM0u[q].re; LetaM0u[q].im = L * etaM0u[q].im;
                LetaM0v[q].re = L * etaM0v[q].re; LetaM0v[q].im = L * etaM0v[q].im;
                LetaLphi[q].re = LetaM0u[q].re + LetaM0v[q].re;
                LetaLphi[q].im = LetaM0u[q].im + LetaM0v[q].im;
                divgradphi[q].re = -kx[j] * Zhat[3 * n + q] - ky[i] * Zhat[5 * n + q];
                divgradphi[q].im = kx[j] * Zhat[2 * n + q] + ky[i] * Zhat[4 * n + q];
                eta2M0u[q].re = pow(eta[q].re, 2) * M0u[q].re / f3 * wallchar; eta2M0u[q].im = 0;
                eta2M0v[q].re = pow(eta[q].re, 2) * M0v[q].re / f3 * wallchar; eta2M0v[q].im = 0;
                dxu[q].re = -kx[j] * Zhat[3 * n + q]; dxu[q].im = kx[j] * Zhat[2 * n + q];
                dyv[q].re = -ky[i] * Zhat[5 * n + q]; dyv[q].im = ky[i] * Zhat[4 * n + q];
            }
        sym2(LetaM0u, Nx, Ny); sym2(LetaM0v, Nx, Ny); sym2(divgradphi, Nx, Ny);
        sym2(LetaLphi, Nx, Ny); sym2(dxu, Nx, Ny); sym2(dyv, Nx, Ny);
        fft2(Nx, Ny, LetaM0u, +1); fft2(Nx, Ny, LetaM0v, +1); fft2(Nx, Ny, divgradphi, +1);
        fft2(Nx, Ny, eta2M0u, -1); fft2(Nx, Ny, eta2M0v, -1);
        fft2(Nx, Ny, LetaLphi, +1); fft2(Nx, Ny, dxu, +1); fft2(Nx, Ny, dyv, +1);
        cx *etaLetaM0u = malloc(sizeof(cx) * n), *etaLetaM0v = malloc(sizeof(cx) * n);
        cx *eta2dxu = malloc(sizeof(cx) * n), *eta2dyv = malloc(sizeof(cx) * n), *deletaH3 = malloc(sizeof(cx) * n);
        for (int q = 0; q < n; q++) {
            const double wallchar = c->wallchar ? c->wallchar[q] : 1.0;
            etaLetaM0u[q].re = eta[q].re / factIFFT * LetaM0u[q].re / factIFFT; etaLetaM0u[q].im = 0;
            etaLetaM0v[q].re = eta[q].re / factIFFT * LetaM0v[q].re / factIFFT; etaLetaM0v[q].im = 0;
            eta2dxu[q].re = pow(eta[q].re, 2) * dxu[q].re / f3 * wallchar; eta2dxu[q].im = 0;
            eta2dyv[q].re = pow(eta[q].re, 2) * dyv[q].re / f3 * wallchar; eta2dyv[q].im = 0;
            deletaH3[q].re = (Lphi[q].re / factIFFT * eta[q].re / factIFFT * divgradphi[q].re / factIFFT
                              + Lphi[q].re / factIFFT * LetaLphi[q].re / factIFFT);
            deletaH3[q].im = 0;
        }
        fft2(Nx, Ny, etaLetaM0u, -1); fft2(Nx, Ny, etaLetaM0v, -1); fft2(Nx, Ny, eta2dxu, -1);
        fft2(Nx, Ny, eta2dyv, -1); fft2(Nx, Ny, deletaH3, -1);
        cx *ikx = malloc(sizeof(cx) * n), *iky = malloc(sizeof(cx) * n);
        cx *delu = malloc(sizeof(cx) * n), *delv = malloc(sizeof(cx) * n);
        for (int i = 0; i < Ny; i++)
            for (int j = 0; j < Nx; j++) {
                const int q = i * Nx + j;
                const double L = c->l2d[q];
                ikx[q].re = -kx[j] * deletaH3[q].im; ikx[q].im = kx[j] * deletaH3[q].re;
                iky[q].re = -ky[i] * deletaH3[q].im; iky[q].im = ky[i] * deletaH3[q].re;
                delu[q].re = L * etaLetaM0u[q].re + 0.5 * L * eta2dxu[q].re - 0.5 * (pow(kx[j], 2) * eta2M0u[q].re);
                delu[q].im = L * etaLetaM0u[q].im + 0.5 * L * eta2dxu[q].im - 0.5 * (pow(kx[j], 2) * eta2M0u[q].im);
                delv[q].re = L * etaLetaM0v[q].re + 0.5 * L * eta2dyv[q].re - 0.5 * (pow(ky[i], 2) * eta2M0v[q].re);
                delv[q].im = L * etaLetaM0v[q].im + 0.5 * L * eta2dyv[q].im - 0.5 * (pow(ky[i], 2) * eta2M0v[q].im);
            }
        deluH3adj = malloc(sizeof(cx) * n); delvH3adj = malloc(sizeof(cx) * n);
        ikxH3adj = malloc(sizeof(cx) * n); ikyH3adj = malloc(sizeof(cx) * n);
        fun_adjust(c, deluH3adj, delu);
        fun_adjust(c, delvH3adj, delv);
        fun_adjust(c, ikxH3adj, ikx);
        fun_adjust(c, ikyH3adj, iky);
        free(ikx); free(iky); free(delu); free(delv);
        free(LetaM0u); free(LetaM0v); free(LetaLphi); free(divgradphi); free(dxu); free(dyv);
        free(eta2M0u); free(eta2M0v); free(etaLetaM0u); free(etaLetaM0v); free(eta2dxu); free(eta2dyv);
        free(deletaH3);
    }

    cx* Source_hat = malloc(sizeof(cx) * n);
    fun_source(c, t, Source_hat);

    cx* dphi = malloc(sizeof(cx) * n);   /* delphiH_hat (2d/fun_odesolver.c:4480-4486) */
    for (int q = 0; q < n; q++) {
        dphi[q] = delphiH1hat[q];
        if (c->model >= 2) {
            dphi[q].re = delphiH1hat[q].re + deluH2adj[q].re + delvH2adj[q].re;
            dphi[q].im = delphiH1hat[q].im + deluH2adj[q].im + delvH2adj[q].im;
        }
        if (c->model == 3) {
            dphi[q].re = delphiH1hat[q].re + deluH2adj[q].re + delvH2adj[q].re + deluH3adj[q].re + delvH3adj[q].re;
            dphi[q].im = delphiH1hat[q].im + deluH2adj[q].im + delvH2adj[q].im + deluH3adj[q].im + delvH3adj[q].im;
        }
    }
    /* breaking (:4494-4502), as in the varying-bottom RHS */
    static const cx zero = {0.0, 0.0};
    if (c->brk) {
        memset(c->brk->B, 0, sizeof(double) * n);
        if (c->brk->tprev < t) {
            brk_process(c, t, Zhat, eta, u, v);
            brk_force(c, eta, dphi);
        }
    }
    for (int i = 0; i < Ny; i++)
        for (int j = 0; j < Nx; j++) {
            const int q = i * Nx + j;
            const double a = c->aal[q];
            cx ix = {0, 0}, iy = {0, 0};
            if (c->model >= 2) {
                ix = ikxH2adj[q];
                iy = ikyH2adj[q];
            }
            const cx sbx = c->brk ? c->brk->sbx[q] : zero, sby = c->brk ? c->brk->sby[q] : zero;
            dt_Zhat[q] = (Source_hat[q].re + dphi[q].re - dampeta[q].re) * a;
            dt_Zhat[n + q] = (Source_hat[q].im + dphi[q].im - dampeta[q].im) * a;
            if (c->model == 3) {   /* rhs_AB3_2DF_uv (:4703-4725) */
                const cx jx = ikxH3adj[q], jy = ikyH3adj[q];
                dt_Zhat[2 * n + q] = (GRAV * kx[j] * Zhat[n + q] + sbx.re - ix.re - jx.re - dampu[q].re) * a;
                dt_Zhat[3 * n + q] = (-GRAV * kx[j] * Zhat[q] + sbx.im - ix.im - jx.im - dampu[q].im) * a;
                dt_Zhat[4 * n + q] = (GRAV * ky[i] * Zhat[n + q] + sby.re - iy.re - jy.re - dampv[q].re) * a;
                dt_Zhat[5 * n + q] = (-GRAV * ky[i] * Zhat[q] + sby.im - iy.im - jy.im - dampv[q].im) * a;
                continue;
            }
            dt_Zhat[2 * n + q] = (GRAV * kx[j] * Zhat[n + q] + sbx.re - ix.re - dampu[q].re) * a;
            dt_Zhat[3 * n + q] = (-GRAV * kx[j] * Zhat[q] + sbx.im - ix.im - dampu[q].im) * a;
            dt_Zhat[4 * n + q] = (GRAV * ky[i] * Zhat[n + q] + sby.re - iy.re - dampv[q].re) * a;
            dt_Zhat[5 * n + q] = (-GRAV * ky[i] * Zhat[q] + sby.im - iy.im - dampv[q].im) * a;
        }
    free(dphi);

    free(delphiH1hat); free(eta); free(u); free(v); free(Lphi); free(M0u); free(M0v);
    free(dampeta); free(dampu); free(dampv); free(etaM0u); free(eta_u); free(etaM0v); free(eta_v);
    free(deletaH2); free(ikxH2adj); free(ikyH2adj); free(deluH2adj); free(delvH2adj); free(Source_hat);
    free(deluH3adj); free(delvH3adj); free(ikxH3adj); free(ikyH3adj);
    for (int q = 0; q < 6 * n; q++)
        if (!isfinite(dt_Zhat[q])) return 1;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* gsl_odeiv2 rkf45 (Fehlberg tableau, 5th-order solution propagated),
 * control_y (a_y = 1, a_dydt = 0, safety 0.9) and evolve_apply (dydt_in at
 * every call, final-step clipping, retry on an effective decrease), as called
 * at 2d/fun_odesolver.c:2567-2647.                                          */
/* ------------------------------------------------------------------------ */
static const double ah[] = {1.0 / 4.0, 3.0 / 8.0, 12.0 / 13.0, 1.0, 1.0 / 2.0};
static const double b3[] = {3.0 / 32.0, 9.0 / 32.0};
static const double b4[] = {1932.0 / 2197.0, -7200.0 / 2197.0, 7296.0 / 2197.0};
static const double b5[] = {8341.0 / 4104.0, -32832.0 / 4104.0, 29440.0 / 4104.0, -845.0 / 4104.0};
static const double b6[] = {-6080.0 / 20520.0, 41040.0 / 20520.0, -28352.0 / 20520.0, 9295.0 / 20520.0, -5643.0 / 20520.0};
static const double c1 = 902880.0 / 7618050.0, c3 = 3953664.0 / 7618050.0, c4 = 3855735.0 / 7618050.0,
                    c5 = -1371249.0 / 7618050.0, c6 = 277020.0 / 7618050.0;
static const double ec[] = {0.0, 1.0 / 360.0, 0.0, -128.0 / 4275.0, -2197.0 / 75240.0, 1.0 / 50.0, 2.0 / 55.0};

static int rkf45_apply(or2d_ctx* c, double t, double h, double* y, double* yerr, const double* dydt_in, double* dydt_out) {
    const int dim = 6 * c->n;
    double *k1 = c->k1, *k2 = c->k2, *k3 = c->k3, *k4 = c->k4, *k5 = c->k5, *k6 = c->k6, *ytmp = c->ytmp;
    memcpy(k1, dydt_in, sizeof(double) * dim);
    for (int i = 0; i < dim; i++) ytmp[i] = y[i] + ah[0] * h * k1[i];
    if (or2d_rhs(c, t + ah[0] * h, ytmp, k2)) return 1;
    for (int i = 0; i < dim; i++) ytmp[i] = y[i] + h * (b3[0] * k1[i] + b3[1] * k2[i]);
    if (or2d_rhs(c, t + ah[1] * h, ytmp, k3)) return 1;
    for (int i = 0; i < dim; i++) ytmp[i] = y[i] + h * (b4[0] * k1[i] + b4[1] * k2[i] + b4[2] * k3[i]);
    if (or2d_rhs(c, t + ah[2] * h, ytmp, k4)) return 1;
    for (int i = 0; i < dim; i++) ytmp[i] = y[i] + h * (b5[0] * k1[i] + b5[1] * k2[i] + b5[2] * k3[i] + b5[3] * k4[i]);
    if (or2d_rhs(c, t + ah[3] * h, ytmp, k5)) return 1;
    for (int i = 0; i < dim; i++)
        ytmp[i] = y[i] + h * (b6[0] * k1[i] + b6[1] * k2[i] + b6[2] * k3[i] + b6[3] * k4[i] + b6[4] * k5[i]);
    if (or2d_rhs(c, t + ah[4] * h, ytmp, k6)) return 1;
    for (int i = 0; i < dim; i++) {
        const double di = c1 * k1[i] + c3 * k3[i] + c4 * k4[i] + c5 * k5[i] + c6 * k6[i];
        y[i] += h * di;
    }
    if (or2d_rhs(c, t + h, y, dydt_out)) return 1;
    for (int i = 0; i < dim; i++)
        yerr[i] = h * (ec[1] * k1[i] + ec[3] * k3[i] + ec[4] * k4[i] + ec[5] * k5[i] + ec[6] * k6[i]);
    return 0;
}

/* std_control_hadjust: -1 decrease, +1 increase, 0 keep */
static int hadjust(const or2d_ctx* c, const double* y, const double* yerr, double* h) {
    const int dim = 6 * c->n;
    const double S = 0.9, ord = 5.0;
    const double h_old = *h;
    double rmax = 2.2250738585072014e-308;
    for (int i = 0; i < dim; i++) {
        const double D0 = c->eps_rel * (1.0 * fabs(y[i])) + c->eps_abs;
        const double r = fabs(yerr[i]) / fabs(D0);
        rmax = r > rmax ? r : rmax;
    }
    if (rmax > 1.1) {
        double r = S / pow(rmax, 1.0 / ord);
        if (r < 0.2) r = 0.2;
        *h = r * h_old;
        return -1;
    } else if (rmax < 0.5) {
        double r = S / pow(rmax, 1.0 / (ord + 1.0));
        if (r > 5.0) r = 5.0;
        if (r < 1.0) r = 1.0;
        *h = r * h_old;
        return 1;
    }
    return 0;
}

int or2d_evolve_apply(or2d_ctx* c, double* t, double t1, double* h, double* y) {
    ensure_rk(c);
    const int dim = 6 * c->n;
    const double t0 = *t;
    double h0 = *h;
    const double dt = t1 - t0;
    if ((dt < 0.0 && h0 > 0.0) || (dt > 0.0 && h0 < 0.0)) { set_err2("step direction"); return 1; }
    memcpy(c->y0, y, sizeof(double) * dim);
    if (c->brk) c->brk->tprev = t0;   /* tprev = t after every evolve_apply (2d/fun_odesolver.c:2646) */
    if (or2d_rhs(c, t0, y, c->dydt_in)) { set_err2("non-finite RHS"); return 1; }
    for (int attempt = 0; attempt < 1000; attempt++) {
        int final_step = 0;
        if ((dt >= 0.0 && h0 > dt) || (dt < 0.0 && h0 < dt)) { h0 = dt; final_step = 1; }
        if (rkf45_apply(c, t0, h0, y, c->yerr, c->dydt_in, c->dydt_out)) {
            memcpy(y, c->y0, sizeof(double) * dim);
            set_err2("non-finite RHS");
            return 1;
        }
        *t = final_step ? t1 : t0 + h0;
        const double h_old = h0;
        const int adj = hadjust(c, y, c->yerr, &h0);
        if (adj == -1) {
            const double t_curr = *t, t_next = (*t) + h0;
            if (fabs(h0) < fabs(h_old) && t_next != t_curr) {
                memcpy(y, c->y0, sizeof(double) * dim);
                c->rej++;
                continue;
            }
            h0 = h_old;
        }
        c->acc++;
        *h = h0;
        if (c->brk) c->brk->tprev = *t;
        return 0;
    }
    set_err2("too many rejected steps");
    return 1;
}

int or2d_run_to(or2d_ctx* c, double* t, double t1, double* h, double* y) {
    while (*t < t1) {
        int s = or2d_evolve_apply(c, t, t1, h, y);
        if (s) return s;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Output stage of ode_solver_uv                                             */
/* ------------------------------------------------------------------------ */

/* ifftw_2d_c2r (2d/functions1.c:523-557) on a copy of one spectrum */
static void c2r2(int nx, int ny, const double* re, const double* im, double* out) {
    int n = nx * ny;
    cx* a = malloc(sizeof(cx) * n);
    for (int q = 0; q < n; q++) { a[q].re = re[q]; a[q].im = im[q]; }
    sym2(a, nx, ny);
    fft2(nx, ny, a, +1);
    for (int q = 0; q < n; q++) out[q] = a[q].re / (nx * ny);
    free(a);
}

void or2d_fields(int nx, int ny, const double* y, double* eta, double* u, double* v) {
    int n = nx * ny;
    double* dst[3] = {eta, u, v};
    for (int f = 0; f < 3; f++)
        if (dst[f]) c2r2(nx, ny, y + 2 * f * n, y + (2 * f + 1) * n, dst[f]);
}

static FILE* open_named(const char* dir, const char* name, const char* mode) {
    char path[1024];
    snprintf(path, sizeof path, "%s%s", dir, name);
    return fopen(path, mode);
}

/* print_xt (2d/fun_odesolver.c:2532-2563) */
static void print_xt2(FILE* fpc, const or2d_outputs* o, int nx, int ny, int ntpart, const double* th) {
    double NX = (double)nx, NT = (double)ntpart, NY = (double)ny;
    fwrite(&NX, sizeof(double), 1, fpc);
    fwrite(o->x, sizeof(double), nx, fpc);
    fwrite(&NY, sizeof(double), 1, fpc);
    fwrite(o->y, sizeof(double), ny, fpc);
    fwrite(&NT, sizeof(double), 1, fpc);
    fwrite(th, sizeof(double), ntpart, fpc);
    fwrite(&o->hs, sizeof(double), 1, fpc);
    fwrite(&o->kp, sizeof(double), 1, fpc);
    fwrite(&o->wp, sizeof(double), 1, fpc);
    fwrite(o->kx, sizeof(double), nx, fpc);
    fwrite(o->ky, sizeof(double), ny, fpc);
    for (int kk = 0; kk < ny; kk++) fwrite(o->bathy + (size_t)kk * nx, sizeof(double), nx, fpc);
    for (int kk = 0; kk < ny; kk++) fwrite(o->cfsa + (size_t)kk * nx, sizeof(double), nx, fpc);
    if (o->chiadjphi)
        for (int kk = 0; kk < ny; kk++) fwrite(o->chiadjphi + (size_t)kk * nx, sizeof(double), nx, fpc);
}

int or2d_run_outputs(or2d_ctx* c, double* t, double* h, double* y, const or2d_outputs* o) {
    const int nx = c->nx, ny = c->ny, n = c->n, ng = o->ngauge;
    if (o->nt < 1 || o->npartition < 1 || o->nt / o->npartition < 1) { set_err2("npartition"); return -1; }
    const int ntpart = o->nt / o->npartition;   /* 2d/fun_odesolver.c:2582 */
    int* ix = malloc(sizeof(int) * (ng > 0 ? ng : 1));
    int* iy = malloc(sizeof(int) * (ng > 0 ? ng : 1));
    for (int j = 0; j < ng; j++) {   /* index_gauge, 2d/functions.c:774-781 */
        ix[j] = (int)round((o->xgauge[j] - o->x[0]) / o->dx);
        iy[j] = (int)round((o->ygauge[j] - o->y[0]) / o->dy);
        if (ix[j] >= nx || iy[j] >= ny || ix[j] < 0 || iy[j] < 0) {
            set_err2("Gauges are outside of the domain!");
            free(ix); free(iy);
            return -1;
        }
    }
    double* eta = malloc(sizeof(double) * n);
    double* u = malloc(sizeof(double) * n);
    double* v = malloc(sizeof(double) * n);
    FILE *fg1 = NULL, *fg2 = NULL, *fg3 = NULL, *feta = NULL, *fu = NULL, *fv = NULL;
    if (ng > 0) {
        fg1 = open_named(o->outdir, "Hawassi_eta_gauge.dat", "wb");
        fg2 = open_named(o->outdir, "Hawassi_u_gauge.dat", "wb");
        fg3 = open_named(o->outdir, "Hawassi_v_gauge.dat", "wb");
    }
    int ipart = 1, ret = o->nt;
    for (int i = 0; i < o->nt; i++) {
        double ti = o->tout[i];
        while (*t < ti) {
            if (or2d_evolve_apply(c, t, ti, h, y)) { ret = -1; goto done; }
        }
        or2d_fields(nx, ny, y, eta, u, v);
        if ((i % ntpart) == 0) {
            char s1[64];
            if (feta) { fclose(feta); fclose(fu); fclose(fv); }
            snprintf(s1, sizeof s1, "Hawassi_eta_%02d.dat", ipart); feta = open_named(o->outdir, s1, "wb");
            snprintf(s1, sizeof s1, "Hawassi_u_%02d.dat", ipart); fu = open_named(o->outdir, s1, "wb");
            snprintf(s1, sizeof s1, "Hawassi_v_%02d.dat", ipart); fv = open_named(o->outdir, s1, "wb");
            if (i == 0) {
                double* th = malloc(sizeof(double) * ntpart);
                for (int j = 0; j < ntpart; j++) th[j] = (i + j) * o->dt;
                snprintf(s1, sizeof s1, "Constant_%02d.dat", ipart);
                FILE* fcon = open_named(o->outdir, s1, "wb");
                print_xt2(fcon, o, nx, ny, ntpart, th);
                fclose(fcon);
                free(th);
            }
            ipart++;
        }
        for (int kk = 0; kk < ny; kk++)
            for (int ll = 0; ll < nx; ll++) {
                float fe = (float)eta[kk * nx + ll];
                fwrite(&fe, sizeof(float), 1, feta);
            }
        fflush(feta);
        if (o->uv_every_sample || (i % ntpart) == 0) {
            for (int kk = 0; kk < ny; kk++)
                for (int ll = 0; ll < nx; ll++) {
                    float fu1 = (float)u[kk * nx + ll], fv1 = (float)v[kk * nx + ll];
                    fwrite(&fu1, sizeof(float), 1, fu);
                    fwrite(&fv1, sizeof(float), 1, fv);
                }
            fflush(fu);
            fflush(fv);
        }
        if (ng > 0) {   /* print_data_gauges_uv, 2d/fun_odesolver.c:427-476 */
            FILE* g[3] = {fg1, fg2, fg3};
            const double* fld[3] = {eta, u, v};
            if (i == 0) {
                for (int f = 0; f < 3; f++) {
                    fprintf(g[f], "0 ");
                    for (int j = 0; j < ng; j++) fprintf(g[f], "%f ", o->x[ix[j]]);
                    fprintf(g[f], "\n");
                }
                for (int f = 0; f < 3; f++) {
                    fprintf(g[f], "0 ");
                    for (int j = 0; j < ng; j++) fprintf(g[f], "%f ", o->y[iy[j]]);
                    fprintf(g[f], "\n");
                }
            }
            for (int f = 0; f < 3; f++) fprintf(g[f], "%f ", *t);
            for (int j = 0; j < ng; j++)
                for (int f = 0; f < 3; f++) fprintf(g[f], "%f ", fld[f][iy[j] * nx + ix[j]]);
            for (int f = 0; f < 3; f++) { fprintf(g[f], "\n"); fflush(g[f]); }
        }
        /* fun_max2darray's running comparison (2d/functions1.c:130-139), then the
         * NaN test of 2d/fun_odesolver.c:2819-2823 */
        double mx = eta[0];
        for (int q = 0; q < n; q++) mx = (mx > eta[q] ? mx : eta[q]);
        if (isnan(mx)) { set_err2("Time stepping failed at t=%fs.", *t); ret = -1; goto done; }
    }
    if (c->brk) {   /* breaking.dat lines (2d/breaking.c:712-720) */
        int nrec = or2d_brk_log(c, NULL, NULL, NULL, 0, 0);
        long long nn = or2d_brk_log_nodes(c);
        double* tr = malloc(sizeof(double) * (nrec > 0 ? nrec : 1));
        int* cnt = malloc(sizeof(int) * (nrec > 0 ? nrec : 1));
        int* nodes = malloc(sizeof(int) * 2 * (nn > 0 ? nn : 1));
        or2d_brk_log(c, tr, cnt, nodes, nrec, (int)nn);
        FILE* fb = open_named(o->outdir, "breaking.dat", "w");
        long long k = 0;
        for (int r = 0; r < nrec; r++) {
            fprintf(fb, "%lf ", tr[r]);
            for (int j = 0; j < cnt[r]; j++, k++) fprintf(fb, " %d %d ", nodes[2 * k], nodes[2 * k + 1]);
            fprintf(fb, "\n");
        }
        fclose(fb);
        free(tr); free(cnt); free(nodes);
    }
done:
    if (feta) { fclose(feta); fclose(fu); fclose(fv); }
    if (fg1) { fclose(fg1); fclose(fg2); fclose(fg3); }
    free(eta); free(u); free(v); free(ix); free(iy);
    return ret;
}

/* ------------------------------------------------------------------------ */
/* The directional JONSWAP influx (jonswap_influx, 2d/functions.c:2226-2446) */
/* ------------------------------------------------------------------------ */
static double kappa_exact(double w, double d) {   /* w^2 = g k tanh(k d), Newton to convergence */
    double k = w / sqrt(GRAV * d);
    for (int it = 0; it < 60; it++) {
        double th = tanh(k * d);
        k = k - (GRAV * k * th - w * w) / (GRAV * th + GRAV * k * d * (1 - th * th));
    }
    return k;
}

void or2d_jonswap_components(int nt, const double* t, double Hs, double Tp, double gamma, double s, double depth,
                             const double* rn, const double* ru, double* a, double* w, double* k, double* theta,
                             double* phi) {
    const int Nhalf = nt / 2;
    /* freqspace (2d/functions.c:1810-1832) of the time span, its first Nt/2 entries */
    const double len = t[nt - 1] - t[0];
    const double dom = 2 * M_PI / len, fmin = -0.5 * 2 * M_PI / (len / (nt - 1));
    const double fmax = (nt / 2) * 2 == nt ? -fmin - dom : -fmin;
    const double du = (fmax - fmin) / (nt - 1);
    double* ww = malloc(sizeof(double) * (size_t)nt);
    for (int i = 0; i < nt / 2; i++) ww[i] = fmin + (nt / 2 + i) * du;
    for (int i = nt / 2, n = 0; i < nt; i++, n++) ww[i] = fmin + n * du;
    ww[0] = 1e-10;
    /* fun_jonswap (2d/functions.c:2226-2307, no SPcorrection.dat) */
    const double omgp = 2 * M_PI / Tp, fp = omgp / (2 * M_PI), alpha = 0.0081;
    double* JS = calloc((size_t)Nhalf, sizeof(double));
    for (int i = 1; i < Nhalf; i++) {
        double sig = ww[i] <= omgp ? 0.07 : 0.09;
        double f = ww[i] / (2 * M_PI);
        double gp = exp(-0.5 * pow(((f / fp - 1) / sig), 2));
        JS[i] = alpha * pow(GRAV, 2) * pow((2 * M_PI), (-4)) * pow(f, (-5)) * exp(-(5.0 / 4.0) * pow((f / fp), (-4))) *
                pow(gamma, gp);
    }
    double m0 = 0;   /* trapz (2d/functions1.c:236) */
    for (int i = 0; i < Nhalf; i++) m0 += (i == 0 || i == Nhalf - 1) ? JS[i] / 2 : JS[i];
    m0 *= ww[1] - ww[0];
    const double domg = ww[1] - ww[0];
    /* directions: the cos^2s inverse CDF at the given uniforms */
    double* th = malloc(sizeof(double) * (size_t)Nhalf);
    const double ds = M_PI / (Nhalf - 1);
    for (int j = 0; j < Nhalf; j++) th[j] = -M_PI / 2.0 + j * ds;
    if (s > 0) {
        const double coef = tgamma(s + 1.0) / (sqrt(M_PI) * tgamma(s + 0.5));
        double* cdf = malloc(sizeof(double) * (size_t)Nhalf);
        double total = 0;
        for (int j = 0; j < Nhalf; j++) { total = total + coef * pow(cos(th[j]), 2 * s); cdf[j] = total; }
        for (int j = 0; j < Nhalf; j++) cdf[j] = cdf[j] / cdf[Nhalf - 1] + exp(-12.0) / M_PI * th[j];
        double* cc = malloc(sizeof(double) * (size_t)Nhalf);
        or_cspline_coeffs(Nhalf, cdf, th, cc);
        for (int j = 0; j < Nhalf; j++) theta[j] = or_cspline_eval(Nhalf, cdf, th, cc, rn[j]);
        free(cdf); free(cc);
    } else {
        for (int j = 0; j < Nhalf; j++) theta[j] = 0.0;
    }
    for (int j = 0; j < Nhalf; j++) {
        const double js = (pow(Hs, 2) / 16) * JS[j] / m0;
        a[j] = sqrt(2 * js * domg);
        w[j] = ww[j];
        k[j] = kappa_exact(ww[j], depth);
        phi[j] = 2 * M_PI * ru[j];
    }
    free(ww); free(JS); free(th);
}

void or2d_directional_signal(int nt, const double* t, int nlines, const double* y, double y0, int nc,
                             const double* a, const double* w, const double* k, const double* theta,
                             const double* phi, double mdir, const double* ramp_t, const double* ramp_y,
                             double* eta, double* skew) {
    for (int j = 0; j < nlines; j++)
        for (int i = 0; i < nt; i++) {
            double sc = 0, ss = 0;
            for (int c = 0; c < nc; c++) {
                const double ph = -w[c] * t[i] + phi[c] + k[c] * sin(theta[c] + mdir) * (y[j] - y0);
                sc += a[c] * cos(ph);
                ss += a[c] * sin(ph);
            }
            const double r = ramp_t[i] * ramp_y[j];
            eta[(size_t)j * nt + i] = sc * r;
            skew[(size_t)j * nt + i] = ss * r;
        }
}
