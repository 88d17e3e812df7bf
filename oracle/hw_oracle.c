/*
 * hw_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY) for the HAWASSI 1D hot
 * path: deck parsing and table set-up, the pseudo-spectral Hamiltonian RHS
 * (HS1/HS2/HS3, flat and varying bathymetry), kinematic breaking, influx
 * source, damping, aliasing, and the GSL-style RKF45 evolve loop.
 *
 * It restates the reference C code (paths relative to the reference project,
 * cited per function) in plain C without globals, and restates the published
 * algorithms of the third-party libraries the reference links but does not
 * ship: FFTW3's c2c DFT definition, GSL's rkf45 stepper (Fehlberg tableau),
 * GSL's standard step-size control (control_y_new) and legacy
 * gsl_odeiv_evolve_apply, GSL's natural cubic spline (cspline) with bsearch
 * accelerator, and GSL's Newton fdf root solver with gsl_root_test_delta.
 *
 * Neutralised reference defects (arithmetic unchanged):
 *   - the per-call leak of `force` (1d/rhs.c:213-214);
 *   - srand(time(0)) for jonswap phases is replaced by a seeded splitmix64
 *     stream and phase[0] (read uninitialised, 1d/influx_lib.c:301-305) is 0;
 *   - define_forcing on wavename = zero evaluates no spline (the reference
 *     evaluates a never-initialised spline there, 1d/rhs.c:662).
 * Out of scope (rejected with an error): wall, friction, wind, coupling,
 * runup (negative depth), HS4.
 */
#define _GNU_SOURCE
#include "hw_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static const double G = 9.80665;   /* 1d/header.h:27 */
static const double DELB = 1.2;    /* 1d/header.h:29 */
#define PI (4.0 * atan(1.0))       /* 1d/header.h:28 */

static char g_err[512];
const char* or_last_error(void) { return g_err; }
static void set_err(const char* fmt, ...) {
    va_list ap; va_start(ap, fmt); vsnprintf(g_err, sizeof g_err, fmt, ap); va_end(ap);
}

typedef struct { double re, im; } cpx;

/* ------------------------------------------------------------------------ */
/* FFT: DFT with FFTW's sign convention, X[k] = sum_n x[n] exp(sign*2*pi*i*n*k/N),
 * sign = -1 forward, +1 backward, unnormalised (FFTW3 fftw_plan_dft_1d).  Any
 * correct FFT reproduces FFTW's values to rounding; power-of-two sizes use an
 * iterative radix-2 transform, others a recursive mixed-radix one.          */
/* ------------------------------------------------------------------------ */
typedef struct { int n; cpx* w; int* rev; } fftplan;

static void plan_free(fftplan* p) { free(p->w); free(p->rev); p->w = NULL; p->rev = NULL; p->n = 0; }

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void plan_make(fftplan* p, int n) {
    p->n = n;
    p->w = (cpx*)malloc(sizeof(cpx) * (size_t)n);
    for (int j = 0; j < n; j++) {
        double a = 2.0 * PI * (double)j / (double)n;
        p->w[j].re = cos(a); p->w[j].im = sin(a);   /* exp(+i 2 pi j / n) */
    }
    p->rev = NULL;
    if (is_pow2(n)) {
        int lg = 0; while ((1 << lg) < n) lg++;
        p->rev = (int*)malloc(sizeof(int) * (size_t)n);
        for (int j = 0; j < n; j++) {
            int r = 0; for (int b = 0; b < lg; b++) if (j & (1 << b)) r |= 1 << (lg - 1 - b);
            p->rev[j] = r;
        }
    }
}

static void fft_exec(const fftplan* p, const cpx* in, cpx* out, int sign);
static void plan_make(fftplan* p, int n);
/* Bluestein: X[k] = c[k] sum_n (x[n] c[n]) b[k-n], c[n] = e^{s i pi n^2/N}, b[m] = conj-chirp */
static void bluestein(const cpx* in, int stride, cpx* out, int n, int sign) {
    int M = 1; while (M < 2 * n - 1) M <<= 1;
    fftplan pm; plan_make(&pm, M);
    cpx* ch = (cpx*)malloc(sizeof(cpx) * (size_t)n);
    for (int j = 0; j < n; j++) {
        long long q = ((long long)j * j) % (2LL * n);
        double a = PI * (double)q / (double)n;
        ch[j].re = cos(a); ch[j].im = sign > 0 ? sin(a) : -sin(a);
    }
    cpx* A = (cpx*)calloc((size_t)M, sizeof(cpx));
    cpx* Bv = (cpx*)calloc((size_t)M, sizeof(cpx));
    for (int j = 0; j < n; j++) {
        cpx x = in[(size_t)j * stride];
        A[j].re = x.re * ch[j].re - x.im * ch[j].im;
        A[j].im = x.re * ch[j].im + x.im * ch[j].re;
    }
    for (int j = 0; j < n; j++) {
        Bv[j].re = ch[j].re; Bv[j].im = -ch[j].im;
        if (j) { Bv[M - j].re = ch[j].re; Bv[M - j].im = -ch[j].im; }
    }
    fft_exec(&pm, A, A, -1); fft_exec(&pm, Bv, Bv, -1);
    for (int j = 0; j < M; j++) {
        double r = A[j].re * Bv[j].re - A[j].im * Bv[j].im;
        double i = A[j].re * Bv[j].im + A[j].im * Bv[j].re;
        A[j].re = r; A[j].im = i;
    }
    fft_exec(&pm, A, A, +1);
    for (int k = 0; k < n; k++) {
        double r = A[k].re / M, i = A[k].im / M;
        out[k].re = r * ch[k].re - i * ch[k].im;
        out[k].im = r * ch[k].im + i * ch[k].re;
    }
    free(ch); free(A); free(Bv);
    free(pm.w); free(pm.rev);
}

/* recursive mixed radix: out[k] = sum_r W^(r k) FFT_m(in[r::p])[k mod m] */
static void fft_rec(const cpx* in, int stride, cpx* out, int n, int sign, const cpx* wN, int N) {
    if (n == 1) { out[0] = in[0]; return; }
    int p = 0;
    for (int f = 2; f * f <= n; f++) if (n % f == 0) { p = f; break; }
    if (p == 0 && n > 64) { /* large prime: Bluestein chirp-z over a power-of-two FFT */
        bluestein(in, stride, out, n, sign);
        return;
    }
    if (p == 0) { /* small prime: direct DFT */
        for (int k = 0; k < n; k++) {
            double sr = 0, si = 0;
            for (int j = 0; j < n; j++) {
                long long e = ((long long)j * k) % n;
                const cpx w = wN[(e * (N / n)) % N];
                double wi = sign > 0 ? w.im : -w.im;
                const cpx x = in[(size_t)j * stride];
                sr += x.re * w.re - x.im * wi;
                si += x.re * wi + x.im * w.re;
            }
            out[k].re = sr; out[k].im = si;
        }
        return;
    }
    int m = n / p;
    cpx* sub = (cpx*)malloc(sizeof(cpx) * (size_t)n);
    for (int r = 0; r < p; r++) fft_rec(in + (size_t)r * stride, stride * p, sub + (size_t)r * m, m, sign, wN, N);
    for (int k = 0; k < n; k++) {
        double sr = 0, si = 0;
        int km = k % m;
        for (int r = 0; r < p; r++) {
            long long e = ((long long)r * k) % n;
            const cpx w = wN[(e * (N / n)) % N];
            double wi = sign > 0 ? w.im : -w.im;
            const cpx x = sub[(size_t)r * m + km];
            sr += x.re * w.re - x.im * wi;
            si += x.re * wi + x.im * w.re;
        }
        out[k].re = sr; out[k].im = si;
    }
    free(sub);
}

static void fft_exec(const fftplan* p, const cpx* in, cpx* out, int sign) {
    int n = p->n;
    if (p->rev) {
        cpx* a = out;
        if (in == out) {
            cpx* tmp = (cpx*)malloc(sizeof(cpx) * (size_t)n);
            memcpy(tmp, in, sizeof(cpx) * (size_t)n);
            for (int j = 0; j < n; j++) a[p->rev[j]] = tmp[j];
            free(tmp);
        } else {
            for (int j = 0; j < n; j++) a[p->rev[j]] = in[j];
        }
        for (int len = 2; len <= n; len <<= 1) {
            int half = len >> 1, step = n / len;
            for (int s = 0; s < n; s += len) {
                for (int j = 0; j < half; j++) {
                    cpx w = p->w[j * step];
                    double wi = sign > 0 ? w.im : -w.im;
                    cpx u = a[s + j], v = a[s + j + half];
                    double tr = v.re * w.re - v.im * wi;
                    double ti = v.re * wi + v.im * w.re;
                    a[s + j].re = u.re + tr; a[s + j].im = u.im + ti;
                    a[s + j + half].re = u.re - tr; a[s + j + half].im = u.im - ti;
                }
            }
        }
    } else {
        cpx* tmp = (cpx*)malloc(sizeof(cpx) * (size_t)n);
        fft_rec(in, 1, tmp, n, sign, p->w, n);
        memcpy(out, tmp, sizeof(cpx) * (size_t)n);
        free(tmp);
    }
}

void or_fft(int n, const double* re_in, const double* im_in, double* re_out, double* im_out, int sign) {
    fftplan p; plan_make(&p, n);
    cpx* a = (cpx*)malloc(sizeof(cpx) * (size_t)n);
    for (int j = 0; j < n; j++) { a[j].re = re_in[j]; a[j].im = im_in ? im_in[j] : 0.0; }
    fft_exec(&p, a, a, sign);
    for (int j = 0; j < n; j++) { re_out[j] = a[j].re; im_out[j] = a[j].im; }
    free(a); plan_free(&p);
}

/* one-shot transforms with a temporary plan (1d/functions.c:1059-1118,1663-1719) */
static void fft_any(int n, const cpx* in, cpx* out, int sign) {
    fftplan p; plan_make(&p, n); fft_exec(&p, in, out, sign); plan_free(&p);
}
/* fft_real_complex (1d/functions.c:1690) */
static void fft_real_complex(const double* in, cpx* out, int n) {
    cpx* a = (cpx*)malloc(sizeof(cpx) * (size_t)n);
    for (int i = 0; i < n; i++) { a[i].re = in[i]; a[i].im = 0; }
    fft_any(n, a, out, -1); free(a);
}
/* ifft_complex_real (1d/functions.c:1663): real part of the backward DFT over N */
static void ifft_complex_real(const cpx* in, double* out, int n) {
    cpx* b = (cpx*)malloc(sizeof(cpx) * (size_t)n);
    fft_any(n, in, b, +1);
    for (int i = 0; i < n; i++) out[i] = b[i].re / n;
    free(b);
}
/* ifft_real_real (1d/functions.c:1438) */
static void ifft_real_real(const double* in, double* out, int n) {
    cpx* a = (cpx*)malloc(sizeof(cpx) * (size_t)n);
    cpx* b = (cpx*)malloc(sizeof(cpx) * (size_t)n);
    for (int i = 0; i < n; i++) { a[i].re = in[i]; a[i].im = 0; }
    fft_any(n, a, b, +1);
    for (int i = 0; i < n; i++) out[i] = b[i].re / n;   /* ifft_1d divides Re and Im by N */
    free(a); free(b);
}

/* ------------------------------------------------------------------------ */
/* GSL natural cubic spline (gsl_interp_cspline) + bsearch accelerator.     */
/* ------------------------------------------------------------------------ */
typedef struct { int n; double *x, *y, *c; } cspline;

static void cspline_free(cspline* s) { free(s->x); free(s->y); free(s->c); memset(s, 0, sizeof *s); }

/* GSL's symmetric tridiagonal solve (LDL^T) */
static void solve_symm_tridiag(const double* diag, const double* off, const double* b, double* x, int N) {
    double* gamma = (double*)malloc(sizeof(double) * (size_t)N);
    double* alpha = (double*)malloc(sizeof(double) * (size_t)N);
    double* c = (double*)malloc(sizeof(double) * (size_t)N);
    double* z = (double*)malloc(sizeof(double) * (size_t)N);
    alpha[0] = diag[0];
    gamma[0] = (N > 1) ? off[0] / alpha[0] : 0.0;
    for (int i = 1; i < N - 1; i++) {
        alpha[i] = diag[i] - off[i - 1] * gamma[i - 1];
        gamma[i] = off[i] / alpha[i];
    }
    if (N > 1) alpha[N - 1] = diag[N - 1] - off[N - 2] * gamma[N - 2];
    z[0] = b[0];
    for (int i = 1; i < N; i++) z[i] = b[i] - gamma[i - 1] * z[i - 1];
    for (int i = 0; i < N; i++) c[i] = z[i] / alpha[i];
    x[N - 1] = c[N - 1];
    if (N >= 2) for (int i = N - 2; i >= 0; i--) x[i] = c[i] - gamma[i] * x[i + 1];
    free(gamma); free(alpha); free(c); free(z);
}

static void cspline_init(cspline* s, const double* x, const double* y, int n) {
    s->n = n;
    s->x = (double*)malloc(sizeof(double) * (size_t)n); memcpy(s->x, x, sizeof(double) * (size_t)n);
    s->y = (double*)malloc(sizeof(double) * (size_t)n); memcpy(s->y, y, sizeof(double) * (size_t)n);
    s->c = (double*)calloc((size_t)n, sizeof(double));
    int sys = n - 2;
    if (sys <= 0) return;
    double* diag = (double*)malloc(sizeof(double) * (size_t)sys);
    double* off = (double*)malloc(sizeof(double) * (size_t)sys);
    double* g = (double*)malloc(sizeof(double) * (size_t)sys);
    for (int i = 0; i < sys; i++) {
        double h_i = x[i + 1] - x[i], h_ip1 = x[i + 2] - x[i + 1];
        double yd_i = y[i + 1] - y[i], yd_ip1 = y[i + 2] - y[i + 1];
        double g_i = (h_i != 0.0) ? 1.0 / h_i : 0.0;
        double g_ip1 = (h_ip1 != 0.0) ? 1.0 / h_ip1 : 0.0;
        off[i] = h_ip1;
        diag[i] = 2.0 * (h_ip1 + h_i);
        g[i] = 3.0 * (yd_ip1 * g_ip1 - yd_i * g_i);
    }
    if (sys == 1) s->c[1] = g[0] / diag[0];
    else solve_symm_tridiag(diag, off, g, s->c + 1, sys);
    free(diag); free(off); free(g);
}

static int bsearch_idx(const double* xa, double x, int lo, int hi) {
    while (hi > lo + 1) { int i = (hi + lo) / 2; if (xa[i] > x) hi = i; else lo = i; }
    return lo;
}

static double cspline_eval(const cspline* s, double x) {
    if (x < s->x[0] || x > s->x[s->n - 1]) return NAN;   /* GSL_EDOM */
    int i = bsearch_idx(s->x, x, 0, s->n - 1);
    double x_lo = s->x[i], x_hi = s->x[i + 1];
    double y_lo = s->y[i], y_hi = s->y[i + 1];
    double h = x_hi - x_lo, dy = y_hi - y_lo, delx = x - x_lo;
    double c_i = s->c[i], c_ip1 = s->c[i + 1];
    double b_i = dy / h - h * (c_ip1 + 2.0 * c_i) / 3.0;
    double d_i = (c_ip1 - c_i) / (3.0 * h);
    return y_lo + delx * (b_i + delx * (c_i + delx * d_i));
}

/* exported for the 2D restatement (hw_oracle2d.c), which evaluates the same
 * GSL natural spline on each influx-line signal */
void or_cspline_coeffs(int n, const double* x, const double* y, double* c_out) {
    cspline s; cspline_init(&s, x, y, n);
    memcpy(c_out, s.c, sizeof(double) * (size_t)n);
    cspline_free(&s);
}
double or_cspline_eval(int n, const double* x, const double* y, const double* c, double t) {
    cspline s; s.n = n; s.x = (double*)x; s.y = (double*)y; s.c = (double*)c;
    return cspline_eval(&s, t);
}

/* ------------------------------------------------------------------------ */
/* Exact dispersion (dispersion = "exact", 1d/main.cc:31)                   */
/* ------------------------------------------------------------------------ */
static double sgn(double v) { return v < 0 ? -1.0 : 1.0; }
/* omega_i (1d/functions.c:1397) */
static double omega_i(double k, double d) { return k == 0 ? 0.0 : sgn(k) * sqrt(G * k * tanh(d * k)); }
/* phase_velocity_i (1d/functions.c:1415) */
static double phase_velocity_i(double k, double d) { return k == 0 ? sqrt(G * d) : sgn(k) * sqrt(G * k * tanh(d * k)) / k; }
/* group_velocity_i (1d/functions.c:1361) */
static double group_velocity_i(double k, double d) {
    if (k == 0) return sqrt(G * d);
    double th = tanh(d * k);
    return sgn(k) * sqrt(G) / 2 / sqrt(k * th) * (th + k * (1 - pow(th, 2)) * d);
}
/* invers_omega (1d/functions.c:984-1020): GSL Newton fdf from x=0,
 * stop when gsl_root_test_delta(x, x0, 0, 1e-3) succeeds. */
static double invers_omega(double w, double d) {
    double x = 0.0, value = 0.0;
    double root = x;
    double f = w - omega_i(root, d), df = -group_velocity_i(root, d);
    int iter = 0, status;
    do {
        iter++;
        if (df == 0.0) break;                           /* GSL_EZERODIV */
        double root_new = root - f / df;
        root = root_new;
        f = w - omega_i(root, d); df = -group_velocity_i(root, d);
        double x0 = x;
        x = root;
        double tol = 0.0 + 1e-3 * fabs(x);
        status = (fabs(x - x0) < tol || x == x0) ? 0 : 1;
        if (status == 0) value = x;
    } while (status == 1 && iter < 1000);
    return value;
}

/* ------------------------------------------------------------------------ */
/* Context                                                                  */
/* ------------------------------------------------------------------------ */
typedef struct {
    int Bindex, BindexNow; double Ucrest; int DirProp; double Bposition, Btime; int Bcount;
} CB;   /* 1d/header.h:48-56 */

struct or_ctx {
    /* deck (1d/read_input.c, 1d/influx_lib.c) */
    char wavename[64], initial[64], bath[64], dynmodel[64], breaking[64], friction[64],
         influxing[64], propagation[64], kinematic[64], wall[64], coupling[64], rampbool[64],
         cut_temp[64], mid_temp[64], min_z[64], max_z[64], dir_force[256];
    double depthflat, adjcoef, parKBC, parTC, parTchar, xinterv1, xinterv2, nTramp;
    double Xwall, refl_coef, x_cpl[2], alpha_corr;
    int ngauge, npartition, nsurf, ndeep, walltype;
    double T0, Tend, dt, Tp, Hs, gamJS, lenT, omgp;
    int Nt;
    double Xstart, Xend, Xinflux, dx, dampL, dampR, length;
    int Nx, n, idx_inf, cutfracwn, model;   /* model: 1,2,3 */
    int flat;                               /* bath == flat */
    double mid[2];
    int nref;

    /* influx */
    double *wave_t, *wave_eta, *ttrace;
    double nu_peak, kp, Tp_peak, lambda_p, Hs_in, MaxEtaInit, depthinf;
    double *ww, *spinflux, *insig, *insig_skew, *kom, *GVom;
    cpx* insig_hat;
    cspline sp_in, sp_skew;
    int has_influx;

    /* domain */
    double *x, *k, *depth, *dampchar, *dampcoef, *spatgamX, *Ug, *aal, *ChiAdj, *gauge;
    cpx *gamX, *gamX_skew;
    double Cpeak, CpLeft, CpRight;
    double *temp_wave, *temp_u;

    /* operators */
    double *Csqr, *L, *M0im;
    double *Csq_min, *Csq_mid, *Csq_plus, *gam_min, *gam_mid, *gam_plus;
    double *CsqK, *gamK;   /* K > 3 reference depths: [K][Nx] */

    /* breaking (1d/header.h:79-83,106-109) */
    int brk;
    double KBC, TC, Tstar; int xbstart, xbend, xbendL, xbstartR, lenIF, ILL, IFF;
    CB *CrestBreak, *CrestBreakNew, *CrestBreakPrev;
    int *ID_Node_end, *Break_nodes;
    double* B;
    int flag, ITERbdt, ITERbn;
    char* blog; size_t blog_len, blog_cap;

    /* rhs state */
    double* dy;
    cpx* Rb_hat;
    fftplan plan;

    /* stepper */
    double eps_abs, eps_rel, h0, t_stop;
    double *y0, *yerr, *dydt_in, *dydt_out, *k1, *k2, *k3, *k4, *k5, *k6, *ytmp;
    long long rhs_calls, accepted, rejected;
    unsigned long long seed;
    char outdir[512];
    int write_fields;

    /* kinematics (read_kinematics, 1d/functions.c:3555-3669) */
    int kin, kin_i1, kin_i2, kin_nx, kin_nz;
    double *kin_z, kin_maxD, kin_minD, kin_maxEta, kin_minEta;
};
static int kin_setup(or_ctx* c);

static void blog_append(or_ctx* c, const char* fmt, ...) {
    char buf[256]; va_list ap;
    for (;;) {
        size_t room = c->blog_cap - c->blog_len;
        va_start(ap, fmt);
        int w = vsnprintf(c->blog + c->blog_len, room, fmt, ap);
        va_end(ap);
        if (w >= 0 && (size_t)w < room) { c->blog_len += (size_t)w; return; }
        c->blog_cap = c->blog_cap * 2 + 4096;
        c->blog = (char*)realloc(c->blog, c->blog_cap);
        (void)buf;
    }
}

/* ------------------------------------------------------------------------ */
/* Deck parsing: the same positional stdio reads as 1d/read_input.c:1-60 and
 * 1d/influx_lib.c:1-109 (the input.txt format itself).                     */
/* ------------------------------------------------------------------------ */
static int read_input_file(or_ctx* c, const char* dir) {
    char path[1024], line[128];
    snprintf(path, sizeof path, "%s/input.txt", dir);
    FILE* f = fopen(path, "r");
    if (!f) { set_err("cannot open %s", path); return -1; }
    int r = 0;
    if (!fgets(line, sizeof line, f)) r = -1;
    if (fscanf(f, "%*s %*s %63s \n", c->wavename) != 1) r = -1;
    if (fscanf(f, "%*s %*s %63s \n", c->initial) != 1) r = -1;
    rewind(f);
    for (int i = 0; i < 18; i++) if (!fgets(line, sizeof line, f)) r = -1;
    if (fscanf(f, "%*s %*s %63s \n %*s %*s %lf \n %*s %*s %lf \n", c->bath, &c->depthflat, &c->adjcoef) != 3) r = -1;
    rewind(f);
    for (int i = 0; i < 23; i++) if (!fgets(line, sizeof line, f)) r = -1;
    if (fscanf(f, "%*s %*s %63s \n", c->dynmodel) != 1) r = -1;
    if (fscanf(f, "%*s %*s %63s \n", c->breaking) != 1) r = -1;
    if (fscanf(f, "%*s %*s %63s \n", c->friction) != 1) r = -1;
    if (fscanf(f, "%*s %*s %63s \n", c->influxing) != 1) r = -1;
    if (fscanf(f, "%*s %*s %63s \n", c->propagation) != 1) r = -1;
    if (fscanf(f, "%*s %*s %63s \n", c->kinematic) != 1) r = -1;
    if (fscanf(f, "%*s %*s %d \n", &c->ngauge) != 1) r = -1;
    if (fscanf(f, "%*s %*s %d \n", &c->npartition) != 1) r = -1;
    if (r) { fclose(f); set_err("malformed input.txt (header blocks)"); return -1; }
    /* optional blocks: a failed conversion keeps the zero default, like the reference globals */
    if (fgets(line, sizeof line, f)) {
        if (fscanf(f, "%*s %*s %lf \n %*s %*s %lf %lf \n", &c->parKBC, &c->parTC, &c->parTchar) < 0) {}
    }
    if (fgets(line, sizeof line, f)) {
        if (fscanf(f, "%*s %*s %lf \n %*s %*s %lf \n", &c->xinterv1, &c->xinterv2) < 0) {}
        if (fscanf(f, "%*s %*s %d \n %*s %*s %d \n", &c->nsurf, &c->ndeep) < 0) {}
    }
    if (fgets(line, sizeof line, f)) {
        if (fscanf(f, "%*s %*s %63s \n", c->cut_temp) < 0) {}
        if (fscanf(f, "%*s %*s %63s \n", c->mid_temp) < 0) {}
        if (fscanf(f, "%*s %*s %63s \n", c->min_z) < 0) {}
        if (fscanf(f, "%*s %*s %63s \n", c->max_z) < 0) {}
        if (fscanf(f, "%*s %*s %63s %lf", c->rampbool, &c->nTramp) < 0) {}
        if (fscanf(f, "%*s %*s %63s \n", c->wall) < 0) {}
        if (fscanf(f, "%*s %*s %d %lf %lf\n", &c->walltype, &c->Xwall, &c->refl_coef) < 0) {}
    }
    if (fgets(line, sizeof line, f)) {
        if (fscanf(f, "%*s %*s %63s %255s\n %*s %*s %lf %lf\n", c->coupling, c->dir_force, &c->x_cpl[0], &c->x_cpl[1]) < 0) {}
        if (fscanf(f, "%*s %*s %lf\n", &c->alpha_corr) < 0) {}
    }
    fclose(f);
    return 0;
}

/* splitmix64 uniform in [0,1): the seeded stand-in for rand()/RAND_MAX */
static double sm64_uniform(unsigned long long* s) {
    unsigned long long z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

/* freqspace (1d/functions.c:1173-1197): the reference's wavenumber grid */
static void freqspace(double* fs, double len, int N) {
    double delta = 2 * PI / len;
    double fmin = -0.5 * 2 * PI / (len / (N - 1));
    double fmax = ((N / 2) * 2 == N) ? -fmin - delta : -fmin;
    double d = (fmax - fmin) / (N - 1);
    for (int i = 0; i < N / 2; i++) fs[i] = fmin + (N / 2 + i) * d;
    int Ni = 0;
    for (int i = N / 2; i < N; i++) { fs[i] = fmin + Ni * d; Ni++; }
}

static double trapz(const double* x, const double* a, int N) {   /* 1d/functions.c:1822 */
    double s = 0.0;
    for (int i = 0; i < N; i++) s += (i == 0 || i == N - 1) ? a[i] / 2 : a[i];
    return s * (x[1] - x[0]);
}
static void cumtrapz(const double* in, int n, double dt, double* out) {   /* 1d/functions.c:1841 */
    double t = 0; out[0] = t;
    for (int i = 1; i < n; i++) { t = t + 0.5 * dt * (in[i - 1] + in[i]); out[i] = t; }
}
static double mean_array(const double* a, int n) { double s = 0; for (int i = 0; i < n; i++) s += a[i]; return s / n; }
static double var_array(const double* a, int n, double m) { double v = 0; for (int i = 0; i < n; i++) v += pow(a[i] - m, 2); return v / n; }
static int closest(const double* a, double ref, int N) {   /* 1d/functions.c:1761 */
    int idx = 0; double mn = 10 * (a[N / 2] - a[N / 2 - 1]);
    for (int i = 0; i < N; i++) if (fabs(a[i] - ref) < mn) { mn = fabs(a[i] - ref); idx = i; }
    return idx;
}
static double search_max_val(const double* a, int n) { double t = a[0]; for (int i = 0; i < n; i++) if (a[i] > t) t = a[i]; return t; }
static double search_min_val(const double* a, int n) { double t = a[0]; for (int i = 0; i < n; i++) if (a[i] < t) t = a[i]; return t; }
/* search_max (1d/functions.c:1271): first half only, >= keeps the last maximum */
static void search_max_half(const double* a, int n, double* mx, int* idx) {
    double t = a[0];
    for (int i = 0; i < n / 2; i++) if (a[i] >= t) { t = a[i]; *idx = i; }
    *mx = t;
}
static int primeFactors_bad(int number) {   /* 1d/functions.c:3671: 1 if largest prime factor > 13 */
    while (number % 2 == 0) number /= 2;
    for (int i = 3; i <= sqrt(number); i += 2) while (number % i == 0) number /= i;
    return number > 13 ? 1 : 0;
}
static void circshift(double* a, int shift, int N) {   /* 1d/functions.c:1231 (same result, O(N)) */
    if (N <= 0) return;
    int s = ((shift % N) + N) % N;
    if (s == 0) return;
    double* t = (double*)malloc(sizeof(double) * (size_t)N);
    for (int j = 0; j < N; j++) t[(j + s) % N] = a[j];
    memcpy(a, t, sizeof(double) * (size_t)N); free(t);
}
/* cf (1d/x_space.c:1-16) */
static double* cf(const double* xi, double Xi, double del, int Nx) {
    double* r = (double*)malloc(sizeof(double) * (size_t)Nx);
    for (int j = 0; j < Nx; j++) {
        if (xi[j] < Xi) r[j] = 0;
        else if (xi[j] == Xi) r[j] = 0.5 * fmax((xi[j] - (Xi + del)) / fabs(xi[j] - (Xi + del)), (1 - cos((xi[j] - Xi) * PI / del)) / 2);
        else r[j] = fmax((xi[j] - (Xi + del)) / fabs(xi[j] - (Xi + del)), (1 - cos((xi[j] - Xi) * PI / del)) / 2);
    }
    return r;
}
/* dampzone (1d/functions.c:1331) */
static void dampzone(or_ctx* c, double Bleft, double Bright) {
    for (int i = 0; i < c->Nx; i++) {
        double xi = c->x[i];
        double hR0 = Bright - xi < 0 ? -1 : 1;
        double hR1 = 1 + ((Bright + c->dampR - xi) < 0 ? -1 : 1);
        double hR2 = (1 + cos(PI * (xi - Bright) / c->dampR)) / 2;
        double mR = hR1 < hR2 ? hR1 : hR2;
        double hhR = hR0 > mR ? hR0 : mR;
        double hL0 = 1 + ((xi - Bleft + c->dampL) < 0 ? -1 : 1);
        double hL1 = (xi - Bleft) < 0 ? -1 : 1;
        double hL2 = (1 - cos(PI * (xi - Bleft + c->dampL) / c->dampL)) / 2;
        double mL = hL1 > hL2 ? hL1 : hL2;
        double hhL = hL0 < mL ? hL0 : mL;
        c->dampchar[i] = 1 - (hhR * hhL);
    }
}

/* fun_jonswap (1d/influx_lib.c:243), including its integer exponent 5/4 == 1 */
static double* fun_jonswap(const double* omg, double omgp, double gamJS, double Hs, int Nt) {
    int Nomg = Nt / 2;
    double* sigma = (double*)malloc(sizeof(double) * (size_t)Nomg);
    double* JS = (double*)calloc((size_t)Nomg, sizeof(double));
    double* out = (double*)malloc(sizeof(double) * (size_t)Nomg);
    for (int i = 0; i < Nomg; i++) sigma[i] = omg[i] <= omgp ? 0.07 : 0.09;
    double alpha = 0.0081, f_p = omgp / (2 * PI);
    for (int i = 1; i < Nomg; i++) {
        double f = omg[i] / (2 * PI);
        double gp = exp(-0.5 * pow(((f / f_p - 1) / sigma[i]), 2));
        JS[i] = alpha * pow(G, 2) * pow((2 * PI), (-4)) * pow(f, (-5)) * exp(-(5 / 4) * pow((f / f_p), (-4))) * pow(gamJS, gp);
    }
    /* JS[0] is uninitialised heap in the reference; it is 0 here */
    double m0 = trapz(omg, JS, Nomg);
    for (int i = 0; i < Nomg; i++) out[i] = (pow(Hs, 2) / 16) * JS[i] / m0;
    free(sigma); free(JS);
    return out;
}

/* jonswap_influx (1d/influx_lib.c:289) with seeded phases: the JONSWAP spectrum on
 * Nt/2 lines (fun_jonswap), random phases (the reference's off-by-one kept: line
 * i+1 takes phase[i], phase[0] = 0), the inverse transform, the start/end ramps and
 * the normalisation to Hs / (4 sqrt(variance)). */
static void jonswap_synth(double T0, double lenT, double dt, double Tp, double Hs, double gamJS, double nTramp,
                          unsigned long long seed, int Nt, double* eta) {
    const double omgp = 2 * PI / Tp;
    double* omsig = (double*)malloc(sizeof(double) * (size_t)Nt);
    freqspace(omsig, lenT, Nt);
    double* JS = fun_jonswap(omsig, omgp, gamJS, Hs, Nt);
    double* phase = (double*)calloc((size_t)(Nt / 2 + 1), sizeof(double));
    cpx* rh = (cpx*)calloc((size_t)Nt, sizeof(cpx));
    unsigned long long s = seed;
    for (int i = 0; i < Nt / 2; i++) {
        phase[i + 1] = 2 * PI * sm64_uniform(&s);
        rh[i + 1].re = (sqrt(JS[i]) * cos(phase[i])) / dt * 2 * pow(PI, 2);
        rh[i + 1].im = -(sqrt(JS[i]) * sin(phase[i])) / dt * 2 * pow(PI, 2);
        rh[Nt - 1 - i].re = rh[i + 1].re;
        rh[Nt - 1 - i].im = -rh[i + 1].im;
    }
    rh[0].re = 0; rh[0].im = 0;
    double* raw = (double*)malloc(sizeof(double) * (size_t)Nt);
    ifft_complex_real(rh, raw, Nt);
    double* ramp = (double*)malloc(sizeof(double) * (size_t)Nt);
    for (int j = 0; j < Nt; j++) {
        double tin = T0 + j * dt;
        double A = ((tin - T0) - nTramp * Tp);
        double B1 = A / fabs(A);
        double B2 = (1 - cos((tin - T0) * PI / nTramp / Tp)) / 2;
        ramp[j] = B1 > B2 ? B1 : B2;
    }
    double* ins = (double*)malloc(sizeof(double) * (size_t)Nt);
    for (int j = 0; j < Nt; j++) ins[j] = ramp[j] * raw[j] * ramp[Nt - 1 - j];
    double v = var_array(ins, Nt, mean_array(ins, Nt));
    for (int j = 0; j < Nt; j++) eta[j] = ins[j] * Hs / (4 * sqrt(v));
    free(omsig); free(JS); free(phase); free(rh); free(raw); free(ramp); free(ins);
}

int or_jonswap_signal(double T0, double Tend, double dt, double Tp, double Hs, double gamma, double nTramp,
                      unsigned long long seed, double* eta_out, int cap) {
    const double lenT = Tend - T0;
    const int Nt = (int)((lenT) / dt + 1);
    if (Nt < 4) return -1;
    if (eta_out && cap >= Nt) jonswap_synth(T0, lenT, dt, Tp, Hs, gamma, nTramp, seed, Nt, eta_out);
    return Nt;
}

/* influxlib (1d/influx_lib.c:1-109) + harmonic/jonswap synthesis */
static int influxlib(or_ctx* c, const char* dir) {
    char path[1024], line[256];
    snprintf(path, sizeof path, "%s/input.txt", dir);
    FILE* f = fopen(path, "r");
    if (!f) { set_err("cannot open %s", path); return -1; }
    int known = 0;
    if (!strcmp(c->wavename, "harmonic") || !strcmp(c->wavename, "jonswap") || !strcmp(c->wavename, "zero")) {
        for (int i = 0; i < 5; i++) if (!fgets(line, sizeof line, f)) break;
        if (fscanf(f, "%*s %*s %lf \n %*s %*s %lf \n %*s %*s %lf\n", &c->T0, &c->Tend, &c->dt) != 3 ||
            fscanf(f, "%*s %*s %lf \n %*s %*s %lf \n %*s %*s %lf\n", &c->Tp, &c->Hs, &c->gamJS) != 3) {
            fclose(f); set_err("malformed time/spectrum block in input.txt"); return -1;
        }
        rewind(f);
        c->lenT = c->Tend - c->T0;
        c->Nt = (int)((c->lenT) / c->dt + 1);
        c->omgp = 2 * PI / c->Tp;
        known = 1;
    }
    if (!strcmp(c->wavename, "zero")) {
        c->n = c->Nt;
        c->wave_t = (double*)malloc(sizeof(double) * (size_t)c->n);
        c->wave_eta = (double*)calloc((size_t)c->n, sizeof(double));
        for (int i = 0; i < c->n; i++) c->wave_t[i] = c->T0 + c->dt * i;
    } else if (!strcmp(c->wavename, "user_defined")) {
        known = 1;
        char ip[1024]; snprintf(ip, sizeof ip, "%s/influx.dat", dir);
        FILE* fi = fopen(ip, "r");
        if (!fi) { fclose(f); set_err("cannot open influx file %s", ip); return -1; }
        int cap = 1024, cnt = 0; double tt, ss;
        c->wave_t = (double*)malloc(sizeof(double) * (size_t)cap);
        c->wave_eta = (double*)malloc(sizeof(double) * (size_t)cap);
        while (fscanf(fi, "%lf %lf", &tt, &ss) == 2) {
            if (cnt == cap) { cap *= 2; c->wave_t = (double*)realloc(c->wave_t, sizeof(double) * (size_t)cap); c->wave_eta = (double*)realloc(c->wave_eta, sizeof(double) * (size_t)cap); }
            c->wave_t[cnt] = tt; c->wave_eta[cnt] = ss; cnt++;
        }
        fclose(fi);
        c->n = cnt;
        if (cnt < 2) { fclose(f); set_err("influx.dat holds fewer than 2 samples"); return -1; }
    } else if (!strcmp(c->wavename, "harmonic")) {
        /* harmonic_influx (1d/influx_lib.c:217) */
        int cap = 1024, i = 0; double t = c->T0, amp = 0.5 * c->Hs;
        c->wave_t = (double*)malloc(sizeof(double) * (size_t)cap);
        c->wave_eta = (double*)malloc(sizeof(double) * (size_t)cap);
        while (t <= c->Tend) {
            t = c->T0 + i * c->dt;
            double r1 = ((t - 4 * c->Tp) < 0 ? -1 : 1);
            double r2 = (1 - cos(t * PI / 4 / c->Tp)) / 2;
            double ramp = r1 > r2 ? r1 : r2;
            if (i == cap) { cap *= 2; c->wave_t = (double*)realloc(c->wave_t, sizeof(double) * (size_t)cap); c->wave_eta = (double*)realloc(c->wave_eta, sizeof(double) * (size_t)cap); }
            c->wave_t[i] = t; c->wave_eta[i] = amp * ramp * (sin(t * 2 * PI / c->Tp));
            i++;
        }
        c->n = i;
    } else if (!strcmp(c->wavename, "jonswap")) {
        c->n = c->Nt;
        c->wave_t = (double*)malloc(sizeof(double) * (size_t)c->Nt);
        c->wave_eta = (double*)malloc(sizeof(double) * (size_t)c->Nt);
        jonswap_synth(c->T0, c->lenT, c->dt, c->Tp, c->Hs, c->gamJS, c->nTramp, c->seed, c->Nt, c->wave_eta);
        for (int j = 0; j < c->Nt; j++) c->wave_t[j] = c->T0 + j * c->dt;
    }
    if (!known) { fclose(f); set_err("unsupported wavename '%s'", c->wavename); return -1; }
    for (int i = 0; i < 13; i++) if (!fgets(line, sizeof line, f)) break;
    if (fscanf(f, "%*s %*s %lf \n %*s %*s %lf \n %*s %*s %lf\n", &c->Xstart, &c->Xend, &c->Xinflux) != 3 ||
        fscanf(f, "%*s %*s %lf \n %*s %*s %lf %lf\n ", &c->dx, &c->dampL, &c->dampR) != 3) {
        fclose(f); set_err("malformed &SPATIAL block in input.txt"); return -1;
    }
    fclose(f);
    if (!strcmp(c->dynmodel, "HS1")) c->cutfracwn = 2;
    else if (!strcmp(c->dynmodel, "HS2")) c->cutfracwn = 4;
    else if (!strcmp(c->dynmodel, "HS3")) c->cutfracwn = 6;
    else if (!strcmp(c->dynmodel, "HS4")) c->cutfracwn = 8;
    c->length = c->Xend - c->Xstart;
    c->Nx = (int)((c->length / c->dx) + 1);
    if (c->Nx % 2 != 0) c->Nx = c->Nx - 1;
    if (c->Nx < 4) { set_err("grid too small (Nx=%d)", c->Nx); return -1; }
    c->x = (double*)malloc(sizeof(double) * (size_t)c->Nx);
    c->dx = c->length / (c->Nx - 1);
    for (int i = 0; i < c->Nx; i++) c->x[i] = c->Xstart + c->dx * i;
    c->idx_inf = closest(c->x, c->Xinflux, c->Nx);
    c->Xinflux = c->x[c->idx_inf];
    return 0;
}

static int read_vector_file(const char* dir, const char* name, double* out, int n) {
    char p[1024]; snprintf(p, sizeof p, "%s/%s", dir, name);
    FILE* f = fopen(p, "r");
    if (!f) { set_err("cannot open %s", p); return -1; }
    for (int j = 0; j < n; j++) if (fscanf(f, "%lf \n", &out[j]) != 1) { fclose(f); set_err("%s: short file", p); return -1; }
    fclose(f);
    return 0;
}

/* nsqrspec + set_influx (1d/functions.c:1256-1269,1320-1329) */
static void set_influx(or_ctx* c) {
    int n = c->n;
    cpx* sig = (cpx*)malloc(sizeof(cpx) * (size_t)n);
    cpx* shat = (cpx*)malloc(sizeof(cpx) * (size_t)n);
    for (int i = 0; i < n; i++) { sig[i].re = c->wave_eta[i]; sig[i].im = 0; }
    fft_any(n, sig, shat, -1);
    double* sq = (double*)malloc(sizeof(double) * (size_t)n);
    double sum = 0;
    for (int i = 0; i < n; i++) {
        double a = sqrt(pow(shat[i].re, 2) + pow(shat[i].im, 2));
        sq[i] = a * a;
    }
    for (int i = 0; i < n; i++) sum += sq[i];
    for (int i = 0; i < n; i++) c->spinflux[i] = sqrt(sq[i] / sum);
    freqspace(c->ww, c->wave_t[n - 1] - c->wave_t[0], n);
    double mx; int idx = 0;
    search_max_half(c->spinflux, n, &mx, &idx);
    c->nu_peak = fabs(c->ww[idx]);
    free(sig); free(shat); free(sq);
}

/* modified_influx (1d/functions.c:1968-2042) */
static void modified_influx(or_ctx* c) {
    int n = c->n;
    for (int j = 0; j < n; j++) c->insig[j] = c->wave_eta[j];
    if (!strcmp(c->wavename, "user_defined")) {
        double* ramp = (double*)malloc(sizeof(double) * (size_t)n);
        for (int j = 0; j < n; j++) {
            double A = ((c->ttrace[j] - c->ttrace[0]) - c->nTramp * c->Tp_peak);
            double B1 = A / fabs(A);
            double B2 = (1 - cos((c->ttrace[j] - c->ttrace[0]) * PI / c->nTramp / c->Tp_peak)) / 2;
            ramp[j] = B1 > B2 ? B1 : B2;
        }
        for (int j = 0; j < n; j++) c->insig[j] = ramp[j] * c->insig[j] * ramp[n - 1 - j];
        free(ramp);
    }
    cumtrapz(c->insig, n, c->dt, c->insig_skew);
    fft_real_complex(c->insig, c->insig_hat, n);
    for (int i = 0; i < n; i++) {
        c->kom[i] = (c->ww[i] == 0) ? 0 : invers_omega(c->ww[i], c->depthinf);
        c->GVom[i] = group_velocity_i(c->kom[i], c->depthinf);
    }
    if (!strcmp(c->influxing, "Point")) {
        cpx* a = (cpx*)malloc(sizeof(cpx) * (size_t)n);
        double* m = (double*)malloc(sizeof(double) * (size_t)n);
        double* ms = (double*)malloc(sizeof(double) * (size_t)n);
        for (int i = 0; i < n; i++) { a[i].re = c->GVom[i] * c->insig_hat[i].re; a[i].im = c->GVom[i] * c->insig_hat[i].im; }
        ifft_complex_real(a, m, n);
        cpx* sh = (cpx*)malloc(sizeof(cpx) * (size_t)n);
        fft_real_complex(c->insig_skew, sh, n);
        for (int i = 0; i < n; i++) { a[i].re = c->GVom[i] * sh[i].re; a[i].im = c->GVom[i] * sh[i].im; }
        ifft_complex_real(a, ms, n);
        for (int j = 0; j < n; j++) { c->insig[j] = m[j]; c->insig_skew[j] = ms[j]; }
        free(a); free(m); free(ms); free(sh);
    } else if (!strcmp(c->influxing, "AreaShort")) {
        double g0 = c->GVom[0];
        for (int j = 0; j < n; j++) c->GVom[j] = c->GVom[j] * sqrt(G * c->depthinf) / g0;
    }
}

/* scaling_influx (1d/functions.c:1747) */
static void scaling_influx(cpx* gX, int Nx, double fact, double dx, double cp) {
    for (int i = 0; i < Nx; i++) { gX[i].re = gX[i].re * fact; gX[i].im = gX[i].im * fact; }
    double scale = gX[0].re * dx;
    for (int i = 0; i < Nx; i++) { gX[i].re = gX[i].re * cp / scale; gX[i].im = gX[i].im * cp / scale; }
}

/* x_space (1d/x_space.c:18-164) */
static int x_space(or_ctx* c) {
    int Nx = c->Nx;
    dampzone(c, c->Xstart + c->dampL, c->Xend - c->dampR);
    if (c->has_influx) {
        c->Cpeak = omega_i(c->kp, c->depthinf) / c->kp;
        c->CpLeft = omega_i(c->kp, c->depth[0]) / c->kp;
        c->CpRight = omega_i(c->kp, c->depth[Nx - 1]) / c->kp;
    } else {
        c->Cpeak = sqrt(G * c->depthinf);
        c->CpLeft = sqrt(G * c->depth[0]);
        c->CpRight = sqrt(G * c->depth[Nx - 1]);
    }
    for (int j = 0; j < Nx / 2; j++) {
        c->dampcoef[j] = 7 * c->CpLeft / (0.9 * c->dampL);
        c->dampcoef[j + Nx / 2] = 7 * c->CpRight / (0.9 * c->dampR);
    }
    freqspace(c->k, c->length, Nx);
    double fact = 1 / c->dx;
    double cp = sqrt(G * c->depthinf);
    for (int i = 0; i < Nx; i++) c->Ug[i] = group_velocity_i(c->k[i], c->depthinf);
    if (c->has_influx) {
        if (!strcmp(c->influxing, "Point")) {
            for (int i = 0; i < Nx; i++) {
                c->spatgamX[i] = 0;
                c->gamX[i].re = cos(c->k[i] * (c->Xinflux - c->Xstart)) * fact;
                c->gamX[i].im = -sin(c->k[i] * (c->Xinflux - c->Xstart)) * fact;
            }
            c->spatgamX[c->idx_inf] = fact;
        } else {
            double* spgam = (double*)malloc(sizeof(double) * (size_t)Nx);
            ifft_real_real(c->Ug, spgam, Nx);
            circshift(spgam, (int)((c->Xinflux - c->Xstart) / c->dx), Nx);
            const int area_short = !strcmp(c->influxing, "AreaShort");
            if (area_short) {   /* 1d/x_space.c:64-78: the kernel under a Gaussian window */
                double Lb = 2 * pow(0.4 * c->lambda_p, 2);
                double* gaussInf = (double*)calloc((size_t)Nx, sizeof(double));
                int ind1 = closest(c->x, c->Xinflux - 2 * c->lambda_p, Nx);
                int ind2 = closest(c->x, c->Xinflux + 2 * c->lambda_p, Nx);
                for (int i = ind1; i < ind2 + 1; i++) gaussInf[i] = exp(-pow((c->x[i] - c->Xinflux), 2) / Lb);
                for (int i = 0; i < Nx; i++) spgam[i] = spgam[i] * gaussInf[i];
                free(gaussInf);
            }
            fft_real_complex(spgam, c->gamX, Nx);
            scaling_influx(c->gamX, Nx, fact, c->dx, cp);
            ifft_complex_real(c->gamX, c->spatgamX, Nx);
            free(spgam);
            if (area_short) {   /* 1d/x_space.c:86-109: the signal divided by the kernel's spectrum */
                int n = c->n;
                double* abs_gamX = (double*)malloc(sizeof(double) * (size_t)Nx);
                double* ktemp = (double*)malloc(sizeof(double) * (size_t)Nx);
                cpx* temp = (cpx*)malloc(sizeof(cpx) * (size_t)n);
                for (int i = 0; i < Nx / 2; i++) {
                    abs_gamX[i] = sqrt(pow(c->gamX[Nx / 2 + i].re, 2) + pow(c->gamX[Nx / 2 + i].im, 2));
                    abs_gamX[Nx / 2 + i] = sqrt(pow(c->gamX[i].re, 2) + pow(c->gamX[i].im, 2));
                    ktemp[i] = c->k[Nx / 2 + i];
                    ktemp[Nx / 2 + i] = c->k[i];
                }
                cspline sg;
                cspline_init(&sg, ktemp, abs_gamX, Nx);
                for (int i = 0; i < n; i++) {
                    double gamXom = fabs(c->kom[i]) > fabs(ktemp[Nx - 1]) ? abs_gamX[Nx - 1] : cspline_eval(&sg, c->kom[i]);
                    temp[i].re = c->insig_hat[i].re * c->GVom[i] / gamXom / c->dx;
                    temp[i].im = c->insig_hat[i].im * c->GVom[i] / gamXom / c->dx;
                }
                ifft_complex_real(temp, c->insig, n);
                cumtrapz(c->insig, n, c->dt, c->insig_skew);
                cspline_free(&sg);
                free(abs_gamX); free(ktemp); free(temp);
            }
        }
        for (int i = 0; i < Nx; i++) {
            c->gamX_skew[i].re = -omega_i(c->k[i], c->depthinf) * c->gamX[i].im;
            c->gamX_skew[i].im = omega_i(c->k[i], c->depthinf) * c->gamX[i].re;
        }
        cspline_init(&c->sp_in, c->ttrace, c->insig, c->n);
        cspline_init(&c->sp_skew, c->ttrace, c->insig_skew, c->n);
    }
    if (!strcmp(c->dynmodel, "HS1") || !c->has_influx) {
        for (int j = 0; j < Nx; j++) c->ChiAdj[j] = 1;
    } else if (!strcmp(c->propagation, "Uni+")) {
        double* t = cf(c->x, c->Xinflux, c->adjcoef * c->lambda_p, Nx);
        memcpy(c->ChiAdj, t, sizeof(double) * (size_t)Nx); free(t);
    } else if (!strcmp(c->propagation, "Uni-")) {
        double* t = cf(c->x, (c->Xinflux - c->adjcoef * c->lambda_p), c->adjcoef * c->lambda_p, Nx);
        for (int j = 0; j < Nx; j++) c->ChiAdj[j] = 1 - t[j];
        free(t);
    } else if (!strcmp(c->propagation, "Bi")) {
        double* L = cf(c->x, c->Xinflux, c->adjcoef * c->lambda_p, Nx);
        double* R = cf(c->x, c->Xinflux - c->adjcoef * c->lambda_p, c->adjcoef * c->lambda_p, Nx);
        for (int j = 0; j < Nx; j++) c->ChiAdj[j] = 1 - R[j] + L[j];
        free(L); free(R);
    } else {
        for (int j = 0; j < Nx; j++) c->ChiAdj[j] = 0;   /* reference leaves ChiAdj unallocated */
    }
    return 0;
}

/* Up2IP (1d/functions.c:2195) and Up3IP (1d/functions.c:2247) */
static void up_ip(or_ctx* c, double nu, int three) {
    int Nx = c->Nx;
    double D_min = search_min_val(c->depth, Nx);
    double D_plus = search_max_val(c->depth, Nx);
    double D_mid = (D_plus + D_min) / 2;
    if (three && strcmp(c->mid_temp, "default") != 0) D_mid = c->mid[1];
    int n = 101;
    double dD = (D_plus - D_min) / (n - 1);
    double* Dd = (double*)malloc(sizeof(double) * (size_t)n);
    double* gm = (double*)malloc(sizeof(double) * (size_t)n);
    double* gc = (double*)malloc(sizeof(double) * (size_t)n);
    double* gp = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) {
        Dd[i] = D_min + i * dD;
        double kap = invers_omega(nu, Dd[i]);
        if (!three) {
            double Cp_min = pow(phase_velocity_i(kap, D_min), 2);
            double Cp_plus = pow(phase_velocity_i(kap, D_plus), 2);
            double Cp_D = pow(phase_velocity_i(kap, Dd[i]), 2);
            double Om_min = omega_i(kap, D_min), Om_plus = omega_i(kap, D_plus), Om_D = omega_i(kap, Dd[i]);
            double det = Cp_min * Om_plus - Cp_plus * Om_min;
            gm[i] = (Om_plus * Cp_D - Cp_plus * Om_D) / det;
            gp[i] = (-Om_min * Cp_D + Cp_min * Om_D) / det;
            gc[i] = 0;
        } else {
            double C0_min = sqrt(G * D_min), C0_mid = sqrt(G * D_mid), C0_plus = sqrt(G * D_plus), C0_D = sqrt(G * Dd[i]);
            double Cp_min = pow(phase_velocity_i(kap, D_min), 2);
            double Cp_mid = pow(phase_velocity_i(kap, D_mid), 2);
            double Cp_plus = pow(phase_velocity_i(kap, D_plus), 2);
            double Cp_D = pow(phase_velocity_i(kap, Dd[i]), 2);
            double Om_min = omega_i(kap, D_min), Om_mid = omega_i(kap, D_mid), Om_plus = omega_i(kap, D_plus), Om_D = omega_i(kap, Dd[i]);
            double A = (Om_mid * Cp_plus) - (Om_plus * Cp_mid);
            double B = -(Om_min * Cp_plus) + (Om_plus * Cp_min);
            double C = (Om_min * Cp_mid) - (Om_mid * Cp_min);
            double D = -(C0_mid * Cp_plus) + (C0_plus * Cp_mid);
            double E = (C0_min * Cp_plus) - (C0_plus * Cp_min);
            double F = -(C0_min * Cp_mid) + (C0_mid * Cp_min);
            double Gg = (C0_mid * Om_plus) - (C0_plus * Om_mid);
            double H = -(C0_min * Om_plus) + (C0_plus * Om_min);
            double J = (C0_min * Om_mid) - (C0_mid * Om_min);
            double det = C0_min * A + C0_mid * B + C0_plus * C;
            gm[i] = (A * C0_D + D * Om_D + Gg * Cp_D) / det;
            gc[i] = (B * C0_D + E * Om_D + H * Cp_D) / det;
            gp[i] = (C * C0_D + F * Om_D + J * Cp_D) / det;
        }
    }
    cspline sm, sc, sp;
    cspline_init(&sm, Dd, gm, n); cspline_init(&sp, Dd, gp, n);
    if (three) cspline_init(&sc, Dd, gc, n);
    for (int i = 0; i < Nx; i++) {
        c->Csq_min[i] = pow(phase_velocity_i(c->k[i], D_min), 2);
        c->Csq_plus[i] = pow(phase_velocity_i(c->k[i], D_plus), 2);
        c->gam_min[i] = cspline_eval(&sm, c->depth[i]);
        c->gam_plus[i] = cspline_eval(&sp, c->depth[i]);
        if (three) {
            c->Csq_mid[i] = pow(phase_velocity_i(c->k[i], D_mid), 2);
            c->gam_mid[i] = cspline_eval(&sc, c->depth[i]);
        } else { c->Csq_mid[i] = 0; c->gam_mid[i] = 0; }
    }
    cspline_free(&sm); cspline_free(&sp);
    if (three) cspline_free(&sc);
    free(Dd); free(gm); free(gc); free(gp);
}

/* K-reference operator (no counterpart in the reference, which stops at 3): K
 * log-spaced reference depths D_0 < ... < D_{K-1} spanning [min h, max h]; each point
 * takes the two-reference system of Up2IP (1d/functions.c:2195-2245) on its
 * bracketing pair, solved at its own depth (no 101-sample spline), so at most two of
 * the K weights are nonzero at any point. */
static void up_k(or_ctx* c, double nu, int K) {
    int Nx = c->Nx;
    double D_min = search_min_val(c->depth, Nx), D_plus = search_max_val(c->depth, Nx);
    double* D = (double*)malloc(sizeof(double) * (size_t)K);
    for (int j = 0; j < K; j++) D[j] = D_min * pow(D_plus / D_min, (double)j / (double)(K - 1));
    D[0] = D_min; D[K - 1] = D_plus;
    c->CsqK = (double*)calloc((size_t)K * Nx, sizeof(double));
    c->gamK = (double*)calloc((size_t)K * Nx, sizeof(double));
    for (int j = 0; j < K; j++)
        for (int i = 0; i < Nx; i++) c->CsqK[(size_t)j * Nx + i] = pow(phase_velocity_i(c->k[i], D[j]), 2);
    for (int i = 0; i < Nx; i++) {
        double h = c->depth[i];
        int j = 0;
        while (j < K - 2 && h > D[j + 1]) j++;
        double kap = invers_omega(nu, h);
        double Cp_a = pow(phase_velocity_i(kap, D[j]), 2), Cp_b = pow(phase_velocity_i(kap, D[j + 1]), 2);
        double Cp_h = pow(phase_velocity_i(kap, h), 2);
        double Om_a = omega_i(kap, D[j]), Om_b = omega_i(kap, D[j + 1]), Om_h = omega_i(kap, h);
        double det = Cp_a * Om_b - Cp_b * Om_a;
        c->gamK[(size_t)j * Nx + i] = (Om_b * Cp_h - Cp_b * Om_h) / det;
        c->gamK[(size_t)(j + 1) * Nx + i] = (-Om_a * Cp_h + Cp_a * Om_h) / det;
    }
    free(D);
}

/* define_operator (1d/functions.c:2828) + alias (1d/functions.c:1774) */
static void define_operator(or_ctx* c, double nu) {
    int Nx = c->Nx;
    for (int i = 0; i < Nx; i++) c->Csqr[i] = pow(phase_velocity_i(c->k[i], c->depthinf), 2);
    if (c->flat) {
        for (int i = 0; i < Nx; i++) {
            c->L[i] = pow(c->k[i], 2) * pow(phase_velocity_i(c->k[i], c->depthinf), 2) / G;
            c->M0im[i] = -c->k[i] * c->Csqr[i] / G;
        }
    } else if (c->nref > 3) {
        up_k(c, nu, c->nref);
    } else {
        up_ip(c, nu, c->nref != 2);
    }
    int idk = (int)(Nx / (double)c->cutfracwn) - 1;
    double k0 = c->k[idk];
    for (int i = 0; i < Nx; i++)
        c->aal[i] = (i != idk) ? ((k0 - fabs(c->k[i])) / fabs(k0 - fabs(c->k[i])) + 1) / 2 : 0.5;
}

#define ALLOC(p, n) ((p) = calloc((size_t)(n), sizeof(*(p))))

static void ctx_free(or_ctx* c) {
    if (!c) return;
    void* ps[] = {c->wave_t, c->wave_eta, c->ttrace, c->ww, c->spinflux, c->insig, c->insig_skew, c->kom, c->GVom, c->insig_hat,
                  c->x, c->k, c->depth, c->dampchar, c->dampcoef, c->spatgamX, c->Ug, c->aal, c->ChiAdj, c->gauge, c->gamX, c->gamX_skew,
                  c->temp_wave, c->temp_u, c->Csqr, c->L, c->M0im, c->Csq_min, c->Csq_mid, c->Csq_plus, c->gam_min, c->gam_mid, c->gam_plus,
                  c->CrestBreak, c->CrestBreakNew, c->CrestBreakPrev, c->ID_Node_end, c->Break_nodes, c->B, c->blog, c->dy, c->Rb_hat,
                  c->y0, c->yerr, c->dydt_in, c->dydt_out, c->k1, c->k2, c->k3, c->k4, c->k5, c->k6, c->ytmp,
                  c->CsqK, c->gamK, c->kin_z};
    for (size_t i = 0; i < sizeof ps / sizeof ps[0]; i++) free(ps[i]);
    cspline_free(&c->sp_in); cspline_free(&c->sp_skew);
    plan_free(&c->plan);
    free(c);
}
void or_destroy(or_ctx* c) { ctx_free(c); }

static void set_init_CB(CB* a, int n) {   /* 1d/functions.c:2057 (BindexNow untouched) */
    for (int j = 0; j < n; j++) { a[j].Bindex = 0; a[j].Ucrest = 0; a[j].DirProp = 0; a[j].Bposition = 0; a[j].Btime = 0; a[j].Bcount = 0; }
}

void or_reset(or_ctx* c) {
    c->rhs_calls = c->accepted = c->rejected = 0;
    c->flag = 0; c->ITERbdt = 0; c->ITERbn = 0;
    c->blog_len = 0; if (c->blog) c->blog[0] = 0;
    if (c->brk) {
        int q = c->Nx / 4;
        memset(c->CrestBreak, 0, sizeof(CB) * (size_t)q);
        memset(c->CrestBreakNew, 0, sizeof(CB) * (size_t)q);
        memset(c->CrestBreakPrev, 0, sizeof(CB) * (size_t)q);
        memset(c->ID_Node_end, 0, sizeof(int) * (size_t)q);
        memset(c->Break_nodes, 0, sizeof(int) * (size_t)c->Nx);
        memset(c->B, 0, sizeof(double) * (size_t)c->Nx);
    }
    memset(c->Rb_hat, 0, sizeof(cpx) * (size_t)c->Nx);
    memset(c->dy, 0, sizeof(double) * 4 * (size_t)c->Nx);
}

or_ctx* or_create(const char* dir, const or_opts* o) {
    or_ctx* c = (or_ctx*)calloc(1, sizeof(or_ctx));
    or_opts d; memset(&d, 0, sizeof d);
    if (!o) o = &d;
    c->eps_abs = o->eps_abs > 0 ? o->eps_abs : 1e-5;
    c->eps_rel = o->eps_rel > 0 ? o->eps_rel : 1e-4;
    c->h0 = o->h0 > 0 ? o->h0 : 1e-4;
    c->t_stop = o->t_stop;
    c->seed = o->seed;
    c->nref = o->nref ? o->nref : 3;
    c->write_fields = o->write_fields;
    if (o->outdir) snprintf(c->outdir, sizeof c->outdir, "%s", o->outdir);
    c->mid[0] = 3; c->mid[1] = 0.5;          /* 1d/main.cc:35-36 */
    if (read_input_file(c, dir)) goto fail;
    if (!strcmp(c->rampbool, "no")) c->nTramp = 0;   /* 1d/main.cc:47-49 */
    if (strcmp(c->dynmodel, "HS1") && strcmp(c->dynmodel, "HS2") && strcmp(c->dynmodel, "HS3")) { set_err("unsupported dynamics '%s'", c->dynmodel); goto fail; }
    c->model = c->dynmodel[2] - '0';
    if (!strcmp(c->friction, "yes") || !strcmp(c->wall, "yes") || !strcmp(c->coupling, "yes")) { set_err("friction/wall/coupling are not supported"); goto fail; }
    if (influxlib(c, dir)) goto fail;
    if (primeFactors_bad(c->Nx)) { set_err("Nx=%d has a largest prime factor > 13", c->Nx); goto fail; }
    int Nx = c->Nx, n = c->n;
    ALLOC(c->ttrace, n);
    for (int j = 0; j < n; j++) c->ttrace[j] = c->wave_t[j];
    c->dt = c->ttrace[1] - c->ttrace[0];
    ALLOC(c->depth, Nx);
    c->flat = !strcmp(c->bath, "flat");
    if (!strcmp(c->bath, "user_defined")) {
        if (read_vector_file(dir, "bath.dat", c->depth, Nx)) goto fail;
        c->depthinf = c->depth[c->idx_inf];
        for (int j = 0; j < Nx; j++) if (c->depth[j] < 0) { set_err("runup (negative depth) is not supported"); goto fail; }
    } else if (c->flat) {
        for (int i = 0; i < Nx; i++) { c->depth[i] = c->depthflat; c->depthinf = c->depthflat; }
    } else { set_err("unsupported bathymetry '%s'", c->bath); goto fail; }
    if (c->ngauge > 0) {
        ALLOC(c->gauge, c->ngauge);
        char p[1024]; snprintf(p, sizeof p, "%s/gauges.dat", dir);
        FILE* fg = fopen(p, "r");
        if (!fg) { set_err("cannot open %s", p); goto fail; }
        for (int j = 0; j < c->ngauge; j++) if (fscanf(fg, "%lf \n", &c->gauge[j]) != 1) c->gauge[j] = 0;
        fclose(fg);
    }
    /* set_memory (1d/functions.c:223) */
    ALLOC(c->k, Nx); ALLOC(c->dampchar, Nx); ALLOC(c->gamX, Nx); ALLOC(c->spatgamX, Nx); ALLOC(c->Ug, Nx); ALLOC(c->aal, Nx);
    ALLOC(c->ww, n); ALLOC(c->spinflux, n); ALLOC(c->insig, n); ALLOC(c->insig_skew, n); ALLOC(c->insig_hat, n);
    ALLOC(c->kom, n); ALLOC(c->GVom, n); ALLOC(c->gamX_skew, Nx); ALLOC(c->dampcoef, Nx); ALLOC(c->ChiAdj, Nx);
    c->has_influx = strcmp(c->wavename, "zero") != 0;
    if (c->has_influx) {   /* 1d/main.cc:78-91 */
        set_influx(c);
        c->kp = invers_omega(c->nu_peak, c->depthinf);
        c->Tp_peak = 2 * PI / c->nu_peak;
        if (!strcmp(c->wavename, "jonswap")) { c->nu_peak = 2 * PI / c->Tp; c->kp = invers_omega(c->nu_peak, c->depthinf); }
        c->lambda_p = 2 * PI / c->kp;
        double avg = 0; for (int i = 0; i < n; i++) avg += c->wave_eta[i]; avg /= n;
        double var = 0; for (int i = 0; i < n; i++) var += pow(c->wave_eta[i] - avg, 2); var /= n;
        c->Hs_in = 4 * sqrt(var);
        c->MaxEtaInit = (c->Hs_in / 2) * 0.8;
        modified_influx(c);
    } else { c->Hs_in = 0; c->MaxEtaInit = 0; }
    if (x_space(c)) goto fail;
    if (!strcmp(c->initial, "user_defined")) {   /* 1d/main.cc:104-136 */
        ALLOC(c->temp_wave, Nx); ALLOC(c->temp_u, Nx);
        char p[1024]; snprintf(p, sizeof p, "%s/initial.dat", dir);
        FILE* fi = fopen(p, "r");
        if (!fi) { set_err("cannot open %s", p); goto fail; }
        for (int j = 0; j < Nx; j++) if (fscanf(fi, "%lf %lf\n", &c->temp_wave[j], &c->temp_u[j]) != 2) { fclose(fi); set_err("initial.dat: short file"); goto fail; }
        fclose(fi);
        cpx* sp = (cpx*)malloc(sizeof(cpx) * (size_t)Nx);
        double* ab = (double*)malloc(sizeof(double) * (size_t)Nx);
        fft_real_complex(c->temp_wave, sp, Nx);
        for (int i = 0; i < Nx; i++) ab[i] = sqrt(pow(sp[i].re, 2) + pow(sp[i].im, 2));
        double mx; int idx = 0;
        search_max_half(ab, Nx, &mx, &idx);
        c->kp = fabs(c->k[idx]);
        if (idx == 0) c->kp = fabs(c->k[1]);
        double avgD = mean_array(c->depth, Nx);
        c->nu_peak = omega_i(c->kp, avgD);
        double Hh = 2 * search_max_val(c->temp_wave, Nx);
        if (Hh > c->Hs_in) c->Hs_in = Hh;
        c->MaxEtaInit = (c->Hs_in / 2) * 0.8;
        free(sp); free(ab);
    } else if (strcmp(c->initial, "zero") != 0) { set_err("unsupported initial '%s'", c->initial); goto fail; }
    ALLOC(c->Rb_hat, Nx);
    c->brk = !strcmp(c->breaking, "yes") && c->model >= 2;
    if (!strcmp(c->breaking, "yes")) {   /* parambreak (1d/breaking.c:1-34) */
        c->KBC = c->parKBC; c->TC = c->parTC;
        c->Tstar = strcmp(c->initial, "zero") != 0 ? 5 * sqrt(c->depthinf * G) : c->parTchar * c->Tp_peak;
        if (!strcmp(c->propagation, "Uni+")) {
            c->xbstart = closest(c->x, c->Xinflux + 0.1 * c->adjcoef * c->lambda_p, Nx);
            c->xbend = Nx - 1; c->lenIF = c->xbend - c->xbstart;
        } else if (!strcmp(c->propagation, "Uni-")) {
            c->xbend = closest(c->x, c->Xinflux - 0.1 * c->adjcoef * c->lambda_p, Nx);
            c->xbstart = 0; c->lenIF = c->xbend - c->xbstart;
        } else if (!strcmp(c->propagation, "Bi")) {
            c->xbstart = 0;
            c->xbendL = closest(c->x, c->Xinflux - 0.1 * c->adjcoef * c->lambda_p, Nx);
            c->xbstartR = closest(c->x, c->Xinflux + 0.1 * c->adjcoef * c->lambda_p, Nx);
            c->xbend = Nx - 1; c->ILL = c->xbendL - c->xbstart; c->IFF = c->xbend - c->xbstartR;
        } else {
            c->xbstart = 0; c->xbend = Nx - 1; c->lenIF = c->xbend - c->xbstart;
        }
        int q = Nx / 4;
        ALLOC(c->B, Nx); ALLOC(c->CrestBreak, q); ALLOC(c->CrestBreakNew, q); ALLOC(c->CrestBreakPrev, q);
        ALLOC(c->Break_nodes, Nx); ALLOC(c->ID_Node_end, q);
        c->blog_cap = 1 << 16; c->blog = (char*)malloc(c->blog_cap); c->blog[0] = 0;
    }
    /* read_kinematics (1d/functions.c:3555-3560): cutfrac and mid-depth overrides */
    if (c->cut_temp[0] && strcmp(c->cut_temp, "default") != 0) c->cutfracwn = atoi(c->cut_temp);
    if (c->mid_temp[0] && strcmp(c->mid_temp, "default") != 0) c->mid[1] = atof(c->mid_temp);
    if (c->npartition <= 0) c->npartition = 1;
    ALLOC(c->Csqr, Nx); ALLOC(c->L, Nx); ALLOC(c->M0im, Nx);
    ALLOC(c->Csq_min, Nx); ALLOC(c->Csq_mid, Nx); ALLOC(c->Csq_plus, Nx);
    ALLOC(c->gam_min, Nx); ALLOC(c->gam_mid, Nx); ALLOC(c->gam_plus, Nx);
    define_operator(c, c->nu_peak);
    ALLOC(c->dy, 4 * Nx);
    plan_make(&c->plan, Nx);
    if (strcmp(c->kinematic, "yes") == 0) {
        c->kin = 1;
        if (kin_setup(c)) goto fail;
    }
    int D = 4 * Nx;
    ALLOC(c->y0, D); ALLOC(c->yerr, D); ALLOC(c->dydt_in, D); ALLOC(c->dydt_out, D);
    ALLOC(c->k1, D); ALLOC(c->k2, D); ALLOC(c->k3, D); ALLOC(c->k4, D); ALLOC(c->k5, D); ALLOC(c->k6, D); ALLOC(c->ytmp, D);
    return c;
fail:
    ctx_free(c);
    return NULL;
}

/* ------------------------------------------------------------------------ */
/* RHS                                                                      */
/* ------------------------------------------------------------------------ */
static cpx* cnew(int n) { return (cpx*)calloc((size_t)n, sizeof(cpx)); }
static double* dnew(int n) { return (double*)calloc((size_t)n, sizeof(double)); }
/* plan_ift_nx / plan_ft_nx executions (unnormalised) */
static void ift_nx(or_ctx* c, const cpx* in, cpx* out) { fft_exec(&c->plan, in, out, +1); }
static void ft_nx(or_ctx* c, const cpx* in, cpx* out) { fft_exec(&c->plan, in, out, -1); }
/* ifft_complex_real_nx (1d/functions.c:1642) */
static void ifft_cr_nx(or_ctx* c, const cpx* in, double* out) {
    cpx* b = cnew(c->Nx); ift_nx(c, in, b);
    for (int i = 0; i < c->Nx; i++) out[i] = b[i].re / c->Nx;
    free(b);
}
/* fft_real_complex_nx (1d/functions.c:1721) */
static void fft_rc_nx(or_ctx* c, const double* in, cpx* out) {
    cpx* a = cnew(c->Nx);
    for (int i = 0; i < c->Nx; i++) { a[i].re = in[i]; a[i].im = 0; }
    ft_nx(c, a, out); free(a);
}
/* prod_1ik (1d/functions.c:297): (i*A_Im) * B */
static double p1ik_re(double a, double br, double bi) { (void)br; return (0.0 * br) - (a * bi); }
static double p1ik_im(double a, double br, double bi) { (void)bi; return (0.0 * bi) + (a * br); }

/* HSS over K > 3 references: 1/2 sum_j [F(gam_j Re F^-1(Csq_j u^)) + Csq_j F(gam_j Re F^-1(u^))] */
static void HSS_K(or_ctx* c, const cpx* uh, cpx* out) {
    int Nx = c->Nx, K = c->nref;
    double *iu = dnew(Nx), *is = dnew(Nx), *a = dnew(Nx), *b = dnew(Nx);
    cpx *Cu = cnew(Nx), *F1 = cnew(Nx), *F2 = cnew(Nx);
    ifft_cr_nx(c, uh, iu);
    for (int i = 0; i < Nx; i++) { out[i].re = 0; out[i].im = 0; }
    for (int j = 0; j < K; j++) {
        const double* Cs = c->CsqK + (size_t)j * Nx;
        const double* gm = c->gamK + (size_t)j * Nx;
        for (int i = 0; i < Nx; i++) { Cu[i].re = Cs[i] * uh[i].re; Cu[i].im = Cs[i] * uh[i].im; }
        ifft_cr_nx(c, Cu, is);
        for (int i = 0; i < Nx; i++) { a[i] = gm[i] * is[i]; b[i] = gm[i] * iu[i]; }
        fft_rc_nx(c, a, F1); fft_rc_nx(c, b, F2);
        for (int i = 0; i < Nx; i++) {
            out[i].re += (F1[i].re + Cs[i] * F2[i].re) / 2;
            out[i].im += (F1[i].im + Cs[i] * F2[i].im) / 2;
        }
    }
    free(iu); free(is); free(a); free(b); free(Cu); free(F1); free(F2);
}

/* HSS (1d/functions.c:2861-2977): varying-depth operator with 2 or 3 refs */
static void HSS(or_ctx* c, const cpx* uh, cpx* out) {
    int Nx = c->Nx;
    if (c->nref > 3) { HSS_K(c, uh, out); return; }
    cpx *Cm = cnew(Nx), *Cp = cnew(Nx);
    for (int i = 0; i < Nx; i++) {
        Cm[i].re = c->Csq_min[i] * uh[i].re; Cm[i].im = c->Csq_min[i] * uh[i].im;
        Cp[i].re = c->Csq_plus[i] * uh[i].re; Cp[i].im = c->Csq_plus[i] * uh[i].im;
    }
    double *iu = dnew(Nx), *iCm = dnew(Nx), *iCp = dnew(Nx), *a = dnew(Nx), *b = dnew(Nx), *cc = dnew(Nx), *d = dnew(Nx);
    ifft_cr_nx(c, uh, iu); ifft_cr_nx(c, Cm, iCm); ifft_cr_nx(c, Cp, iCp);
    for (int i = 0; i < Nx; i++) {
        cc[i] = c->gam_min[i] * iu[i];   /* gammin_ift_uh */
        d[i] = c->gam_plus[i] * iu[i];   /* gamplus_ift_uh */
        a[i] = c->gam_min[i] * iCm[i];   /* gam_ift_Cminuh */
        b[i] = c->gam_plus[i] * iCp[i];  /* gam_ift_Cplusuh */
    }
    cpx *H1m = cnew(Nx), *H1p = cnew(Nx), *fm = cnew(Nx), *fp = cnew(Nx);
    fft_rc_nx(c, a, H1m); fft_rc_nx(c, b, H1p); fft_rc_nx(c, cc, fm); fft_rc_nx(c, d, fp);
    for (int i = 0; i < Nx; i++) {
        double H2m_re = c->Csq_min[i] * fm[i].re, H2m_im = c->Csq_min[i] * fm[i].im;
        double H2p_re = c->Csq_plus[i] * fp[i].re, H2p_im = c->Csq_plus[i] * fp[i].im;
        out[i].re = (H1m[i].re + H1p[i].re + H2m_re + H2p_re) / 2;
        out[i].im = (H1m[i].im + H1p[i].im + H2m_im + H2p_im) / 2;
    }
    if (c->nref != 2) {
        cpx* Cc = cnew(Nx);
        for (int i = 0; i < Nx; i++) { Cc[i].re = c->Csq_mid[i] * uh[i].re; Cc[i].im = c->Csq_mid[i] * uh[i].im; }
        double* iCc = dnew(Nx);
        ifft_cr_nx(c, Cc, iCc);
        for (int i = 0; i < Nx; i++) { cc[i] = c->gam_mid[i] * iu[i]; a[i] = c->gam_mid[i] * iCc[i]; }
        cpx *H1c = cnew(Nx), *fc = cnew(Nx);
        fft_rc_nx(c, a, H1c); fft_rc_nx(c, cc, fc);
        for (int i = 0; i < Nx; i++) {
            double H2c_re = c->Csq_mid[i] * fc[i].re, H2c_im = c->Csq_mid[i] * fc[i].im;
            out[i].re = out[i].re + (H1c[i].re + H2c_re) / 2;
            out[i].im = out[i].im + (H1c[i].im + H2c_im) / 2;
        }
        free(Cc); free(iCc); free(H1c); free(fc);
    }
    free(Cm); free(Cp); free(iu); free(iCm); free(iCp); free(a); free(b); free(cc); free(d);
    free(H1m); free(H1p); free(fm); free(fp);
}

/* Op_M0 / Op_M1 (1d/functions.c:2979-3015): -(1/g) ik HSS(A) */
static void Op_M0(or_ctx* c, const cpx* A, cpx* out) {
    int Nx = c->Nx;
    cpx* h = cnew(Nx);
    HSS(c, A, h);
    for (int j = 0; j < Nx; j++) {
        out[j].re = -1 / G * p1ik_re(c->k[j], h[j].re, h[j].im);
        out[j].im = -1 / G * p1ik_im(c->k[j], h[j].re, h[j].im);
    }
    free(h);
}

/* define_delH1 (1d/functions.c:3414) */
static void define_delH1(or_ctx* c, const double* z, cpx* duH1, cpx* deH1) {
    int Nx = c->Nx;
    if (c->flat) {
        for (int i = 0; i < Nx; i++) {
            duH1[i].re = (c->Csqr[i] / G) * c->k[i] * z[i + 3 * Nx];
            duH1[i].im = -(c->Csqr[i] / G) * c->k[i] * z[i + 2 * Nx];
            deH1[i].re = G * c->k[i] * z[i + Nx];
            deH1[i].im = -G * c->k[i] * z[i];
        }
    } else {
        cpx *uh = cnew(Nx), *Cv = cnew(Nx);
        for (int i = 0; i < Nx; i++) { uh[i].re = z[i + 2 * Nx]; uh[i].im = z[i + 3 * Nx]; }
        HSS(c, uh, Cv);
        for (int i = 0; i < Nx; i++) {
            duH1[i].re = (Cv[i].im / G) * c->k[i];
            duH1[i].im = -(Cv[i].re / G) * c->k[i];
            deH1[i].re = G * c->k[i] * z[i + Nx];
            deH1[i].im = -G * c->k[i] * z[i];
        }
        free(uh); free(Cv);
    }
}

/* ifft_fft_Hsf1 (1d/functions.c:1528): damping only */
static void hsf1(or_ctx* c, const double* z, cpx* de, cpx* du) {
    int N = c->Nx;
    cpx *eh = cnew(N), *e = cnew(N), *uh = cnew(N), *u = cnew(N), *a = cnew(N), *b = cnew(N);
    for (int i = 0; i < N; i++) { eh[i].re = z[i]; eh[i].im = z[i + N]; uh[i].re = z[i + 2 * N]; uh[i].im = z[i + 3 * N]; }
    ift_nx(c, eh, e); ift_nx(c, uh, u);
    for (int i = 0; i < N; i++) {
        a[i].re = c->dampcoef[i] * (e[i].re / N) * c->dampchar[i]; a[i].im = 0;
        b[i].re = c->dampcoef[i] * (u[i].re / N) * c->dampchar[i]; b[i].im = 0;
    }
    ft_nx(c, a, de); ft_nx(c, b, du);
    free(eh); free(e); free(uh); free(u); free(a); free(b);
}

/* ifft_fft_Hsf2 (1d/functions.c:1458) and ifft_fft_Hsf2_v (1d/functions.c:3334) */
static void hsf2(or_ctx* c, const double* z, cpx* eu_hat, cpx* LeM_hat, cpx* u2_hat, cpx* de, cpx* du) {
    int N = c->Nx;
    cpx *eh = cnew(N), *e = cnew(N), *uh = cnew(N), *u = cnew(N), *Mh = cnew(N), *M = cnew(N);
    for (int i = 0; i < N; i++) {
        eh[i].re = z[i]; eh[i].im = z[i + N]; uh[i].re = z[i + 2 * N]; uh[i].im = z[i + 3 * N];
        if (c->flat) { Mh[i].re = p1ik_re(c->M0im[i], z[i + 2 * N], z[i + 3 * N]); Mh[i].im = p1ik_im(c->M0im[i], z[i + 2 * N], z[i + 3 * N]); }
    }
    if (!c->flat) Op_M0(c, uh, Mh);
    ift_nx(c, eh, e); ift_nx(c, uh, u); ift_nx(c, Mh, M);
    cpx *eu = cnew(N), *eM = cnew(N), *eMh = cnew(N), *u2 = cnew(N), *dpe = cnew(N), *dpu = cnew(N);
    for (int i = 0; i < N; i++) {
        eu[i].re = (e[i].re / N) * (u[i].re / N);
        eM[i].re = (e[i].re / N) * (M[i].re / N);
        u2[i].re = (pow(u[i].re / N, 2) - pow(M[i].re / N, 2));
        dpe[i].re = c->dampcoef[i] * (e[i].re / N) * c->dampchar[i];
        dpu[i].re = c->dampcoef[i] * (u[i].re / N) * c->dampchar[i];
    }
    ft_nx(c, eu, eu_hat); ft_nx(c, eM, eMh); ft_nx(c, u2, u2_hat); ft_nx(c, dpe, de); ft_nx(c, dpu, du);
    if (c->flat) {
        for (int i = 0; i < N; i++) { LeM_hat[i].re = c->L[i] * eMh[i].re; LeM_hat[i].im = c->L[i] * eMh[i].im; }
    } else {
        cpx* M1 = cnew(N);
        Op_M0(c, eMh, M1);   /* Op_M1 is the same operator */
        for (int i = 0; i < N; i++) { LeM_hat[i].re = p1ik_re(c->k[i], M1[i].re, M1[i].im); LeM_hat[i].im = p1ik_im(c->k[i], M1[i].re, M1[i].im); }
        free(M1);
    }
    free(eh); free(e); free(uh); free(u); free(Mh); free(M); free(eu); free(eM); free(eMh); free(u2); free(dpe); free(dpu);
}

/* ifft_fft_Hsf3 (1d/functions.c:1568) and ifft_fft_Hsf3_v (1d/functions.c:3440) */
static void hsf3(or_ctx* c, const double* z, const cpx* LeM_hat, cpx* deH3_hat, cpx* duH3_hat) {
    int N = c->Nx;
    cpx *eh = cnew(N), *e = cnew(N), *dxh = cnew(N), *dx = cnew(N), *Mh = cnew(N), *M = cnew(N), *LM = cnew(N), *uh = cnew(N);
    for (int i = 0; i < N; i++) {
        eh[i].re = z[i]; eh[i].im = z[i + N]; uh[i].re = z[i + 2 * N]; uh[i].im = z[i + 3 * N];
        dxh[i].re = p1ik_re(c->k[i], z[i + 2 * N], z[i + 3 * N]); dxh[i].im = p1ik_im(c->k[i], z[i + 2 * N], z[i + 3 * N]);
        if (c->flat) { Mh[i].re = p1ik_re(c->M0im[i], z[i + 2 * N], z[i + 3 * N]); Mh[i].im = p1ik_im(c->M0im[i], z[i + 2 * N], z[i + 3 * N]); }
    }
    if (!c->flat) Op_M0(c, uh, Mh);
    ift_nx(c, eh, e); ift_nx(c, dxh, dx); ift_nx(c, Mh, M); ift_nx(c, LeM_hat, LM);
    cpx *a = cnew(N), *ah = cnew(N), *b = cnew(N), *bh = cnew(N), *d = cnew(N), *dh = cnew(N), *f = cnew(N);
    for (int i = 0; i < N; i++) {
        a[i].re = (e[i].re / N) * (LM[i].re / N);
        b[i].re = pow(e[i].re / N, 2) * (dx[i].re / N);
        d[i].re = pow(e[i].re / N, 2) * (M[i].re / N);
        f[i].re = (M[i].re / N) * ((e[i].re / N) * (dx[i].re / N) + (LM[i].re / N));
    }
    ft_nx(c, a, ah); ft_nx(c, b, bh); ft_nx(c, d, dh); ft_nx(c, f, deH3_hat);
    if (c->flat) {
        for (int i = 0; i < N; i++) {
            duH3_hat[i].re = c->L[i] * ah[i].re + (1 / 2.) * c->L[i] * bh[i].re - (1 / 2.) * pow(c->k[i], 2) * dh[i].re;
            duH3_hat[i].im = c->L[i] * ah[i].im + (1 / 2.) * c->L[i] * bh[i].im - (1 / 2.) * pow(c->k[i], 2) * dh[i].im;
        }
    } else {
        cpx *Ma = cnew(N), *Mb = cnew(N);
        Op_M0(c, ah, Ma); Op_M0(c, bh, Mb);
        for (int i = 0; i < N; i++) {
            double tr = Ma[i].re + (1 / 2.) * Mb[i].re, ti = Ma[i].im + (1 / 2.) * Mb[i].im;
            duH3_hat[i].re = p1ik_re(c->k[i], tr, ti) - (1 / 2.) * pow(c->k[i], 2) * dh[i].re;
            duH3_hat[i].im = p1ik_im(c->k[i], tr, ti) - (1 / 2.) * pow(c->k[i], 2) * dh[i].im;
        }
        free(Ma); free(Mb);
    }
    free(eh); free(e); free(dxh); free(dx); free(Mh); free(M); free(LM); free(uh); free(a); free(ah); free(b); free(bh); free(d); free(dh); free(f);
}

/* adjust_delH (1d/rhs.c:695) */
static void adjust_delH(or_ctx* c, cpx* du_adj, cpx* de_adj, const cpx* du, const cpx* de) {
    int N = c->Nx;
    double *a = dnew(N), *b = dnew(N);
    ifft_cr_nx(c, du, a); ifft_cr_nx(c, de, b);
    for (int i = 0; i < N; i++) { a[i] = a[i] * c->ChiAdj[i]; b[i] = b[i] * c->ChiAdj[i]; }
    fft_rc_nx(c, a, du_adj); fft_rc_nx(c, b, de_adj);
    free(a); free(b);
}

/* ---------------- breaking (1d/breaking.c) ---------------- */
static void gradient(const double* a, double d, int n, double* g) {   /* 1d/functions.c:1850 */
    g[0] = (a[1] - a[0]) / d;
    g[n - 1] = (a[n - 1] - a[n - 2]) / d;
    for (int i = 1; i < n - 1; i++) g[i] = (a[i + 1] - a[i - 1]) / (2 * d);
}
/* findpeaks (1d/breaking.c:36): local maxima above MaxEtaInit; locs[0] = count */
static int findpeaks(or_ctx* c, const double* a, int len, int* locs) {
    int j = 1, Nh = 0;
    while (j < len - 1) {
        if (a[j] < c->MaxEtaInit) { j++; continue; }
        if ((a[j] > a[j + 1]) && (a[j] > a[j - 1])) { locs[Nh] = j; Nh++; }
        j++;
    }
    return Nh;
}
/* breaking_criterion (1d/breaking.c:63) */
static void breaking_criterion(or_ctx* c, double time, const double* eta, const cpx* etahat, const double* u) {
    int Nx = c->Nx, Npks = 0, flaghere = 0;
    int* indj = (int*)calloc((size_t)Nx, sizeof(int));
    int any = 0;
    for (int i = 0; i < c->lenIF; i++) if (eta[c->xbstart + i] > c->MaxEtaInit) { any = 1; break; }
    if (any) {
        int* locs = (int*)calloc((size_t)Nx, sizeof(int));
        if (c->xbendL == 0 && c->xbstartR == 0) {
            Npks = findpeaks(c, eta + c->xbstart, c->lenIF, locs);
            for (int i = 0; i < Npks; i++) indj[i] = locs[i] + c->xbstart;
        } else {
            int* l2 = (int*)calloc((size_t)Nx, sizeof(int));
            int n1 = findpeaks(c, eta + c->xbstart, c->ILL, locs);
            int n2 = findpeaks(c, eta + c->xbstartR, c->IFF, l2);
            Npks = n1 + n2;
            for (int i = 0; i < n1; i++) indj[i] = locs[i] + c->xbstart;
            for (int i = n1; i < Npks; i++) indj[i] = l2[i - n1] + c->xbstartR;
            free(l2);
        }
        free(locs);
        flaghere = Npks > 0;
    }
    if (flaghere) {
        double* Hx = dnew(Nx);
        cpx* Hh = cnew(Nx);
        for (int i = 0; i < Nx; i++) {
            if (c->k[i] == 0) { Hh[i].re = 0; Hh[i].im = 0; }
            else { Hh[i].re = (c->k[i] / fabs(c->k[i])) * etahat[i].im; Hh[i].im = -(c->k[i] / fabs(c->k[i])) * etahat[i].re; }
        }
        ifft_cr_nx(c, Hh, Hx);
        double *gH = dnew(Nx), *ge = dnew(Nx);
        gradient(Hx, c->dx, Nx, gH); gradient(eta, c->dx, Nx, ge);
        int itCB = 0;
        CB* tmp = (CB*)calloc((size_t)(Npks > 0 ? Npks : 1), sizeof(CB));
        for (int i = 0; i < Npks; i++) {
            int J = indj[i];
            double KxJ = (eta[J] * gH[J] - Hx[J] * ge[J]) / (pow(eta[J], 2) + pow(Hx[J], 2));
            double Cc = phase_velocity_i(KxJ, c->depth[J] + eta[J]);
            double Up = u[J];
            if (fabs(Up) > (c->KBC * fabs(Cc))) {
                tmp[itCB].Bindex = J; tmp[itCB].BindexNow = J; tmp[itCB].Ucrest = fabs(Up);
                tmp[itCB].DirProp = (int)(Up / fabs(Up)); tmp[itCB].Bposition = c->x[J]; tmp[itCB].Btime = time;
                itCB++;
            }
        }
        for (int j = 0; j < itCB; j++) { c->CrestBreak[j] = tmp[j]; c->CrestBreak[j].Bcount = itCB; }
        free(tmp); free(Hx); free(Hh); free(gH); free(ge);
    } else {
        set_init_CB(c->CrestBreak, Nx / 4);
    }
    free(indj);
}

/* breaking_process (1d/breaking.c:200-449) */
static void breaking_process(or_ctx* c, const double* eta, const cpx* etahat, const double* u, double t) {
    int Nx = c->Nx;
    double* au = dnew(Nx);
    for (int j = 0; j < Nx; j++) au[j] = fabs(u[j]);
    memset(c->B, 0, sizeof(double) * (size_t)Nx);
    breaking_criterion(c, t, eta, etahat, u);
    CB *CBk = c->CrestBreak, *New = c->CrestBreakNew, *Prev = c->CrestBreakPrev;
    int NCB = CBk[0].Bcount;
    if (NCB > 0 && c->flag == 0) {
        c->flag = 1;
        for (int j = 0; j < NCB; j++) New[j] = CBk[j];
    } else if (NCB == 0 && c->flag == 2) {
        int NCBprev = Prev[0].Bcount;
        for (int j = 0; j < NCBprev; j++) New[j] = Prev[j];
    } else if (NCB > 0 && c->flag == 2) {
        int NCBprev = Prev[0].Bcount;
        for (int j = 0; j < NCBprev; j++) New[j] = Prev[j];
        int add = 0;
        for (int kk = 0; kk < NCB; kk++) {
            int isnew = 1;
            for (int l = 0; l < NCBprev; l++) {
                int dleft = abs(c->ID_Node_end[l] - Prev[l].BindexNow);
                if (Prev[l].DirProp == 1) {
                    if (CBk[kk].Bindex >= (Prev[l].BindexNow - 3 * dleft) && CBk[kk].Bindex <= c->ID_Node_end[l]) { isnew = 0; break; }
                } else {
                    if (CBk[kk].Bindex >= Prev[l].BindexNow && CBk[kk].Bindex <= (c->ID_Node_end[l] + 3 * dleft)) { isnew = 0; break; }
                }
            }
            if (isnew) {
                CB* d = &New[NCBprev + add];
                d->Bindex = CBk[kk].Bindex; d->BindexNow = CBk[kk].Bindex;
                c->ID_Node_end[NCBprev + add] = CBk[kk].Bindex;
                d->Ucrest = CBk[kk].Ucrest; d->Bposition = CBk[kk].Bposition; d->Btime = CBk[kk].Btime;
                d->DirProp = CBk[kk].DirProp; d->Bcount = CBk[kk].Bcount;
                add++;
            }
        }
        int j = 0;
        while (j < Nx / 4 && New[j].Bindex > 0) j++;
        for (int i = 0; i < j; i++) New[i].Bcount = j;
    }
    if (c->flag == 1 || c->flag == 2) {
        int NCBnow = New[0].Bcount;
        int it_indexb = 0, iterNprev = 0;
        int* IDT = (int*)calloc((size_t)(NCBnow > 0 ? NCBnow : 1), sizeof(int));
        set_init_CB(Prev, Nx / 4);
        for (int lx = 0; lx < NCBnow; lx++) {
            int indxMaxNow;
            if (c->flag == 1) {
                indxMaxNow = New[lx].Bindex;
            } else {
                int st = New[lx].BindexNow;
                int lenloc = abs(c->ID_Node_end[lx] - st);
                /* idx_max over etaloc[j] = eta[st + j*DirProp] (1d/functions.c:1282) */
                int best = 0;
                if (lenloc > 0) {
                    double tmpv = eta[st];
                    for (int j = 0; j < lenloc; j++) { double v = eta[st + j * New[lx].DirProp]; if (v > tmpv) { tmpv = v; best = j; } }
                }
                indxMaxNow = st + best * New[lx].DirProp;
            }
            New[lx].BindexNow = indxMaxNow;
            if (lx != 0 && indxMaxNow == New[lx - 1].BindexNow) { IDT[lx] = 0; continue; }
            double tbreak = New[lx].Btime, U_I = New[lx].Ucrest, U_F = c->TC * U_I, U_star;
            if ((t - tbreak) >= c->Tstar) U_star = U_F;
            else if ((t - tbreak) >= 0 && (t - tbreak) < c->Tstar) U_star = U_I + ((t - tbreak) / c->Tstar) * (U_F - U_I);
            else U_star = U_I;
            int indEND = (New[lx].DirProp == 1) ? c->xbend : c->xbstart;
            int Node_end = indxMaxNow, fh = 0;
            for (int ly = indxMaxNow; ly < indEND; ly += New[lx].DirProp) {
                if (au[ly] < U_F) { Node_end = ly; break; }
                if (au[ly] > (2 * U_star)) c->B[ly] = 1;
                else if (au[ly] <= U_star) c->B[ly] = 0;
                else c->B[ly] = (au[ly] / U_star) - 1;
                if (au[ly] >= U_star) fh = 1;
                c->Break_nodes[it_indexb] = ly;
                it_indexb++;
                if (New[lx].DirProp == 0) break;   /* guard: the reference loops forever here */
            }
            if (fh == 0) IDT[lx] = 0;
            else {
                IDT[lx] = 1;
                c->ID_Node_end[iterNprev] = Node_end;
                Prev[iterNprev] = New[lx];
                iterNprev++;
            }
        }
        int j = 0;
        while (j < Nx / 4 && Prev[j].Bindex > 0) j++;
        for (int i = 0; i < j; i++) Prev[i].Bcount = j;
        for (int i = 0; i < NCBnow; i++) { if (IDT[i] == 1) { c->flag = 2; break; } else c->flag = 0; }
        if (t > (c->ITERbdt * c->dt) && it_indexb > 0) {
            blog_append(c, "%lf %d ", t, it_indexb);
            for (int q = 0; q < it_indexb; q++) blog_append(c, "%d ", c->Break_nodes[q]);
            blog_append(c, "\n");
            c->ITERbn++;
        }
        free(IDT);
    }
    if (t > (c->ITERbdt * c->dt)) c->ITERbdt++;
    set_init_CB(New, Nx / 4);
    set_init_CB(CBk, Nx / 4);
    free(au);
}

/* rhs_breaking (1d/rhs.c:617) */
static void rhs_breaking(or_ctx* c, const double* eta, const cpx* etahat, const double* u, double t, const cpx* dteta_hat) {
    int Nx = c->Nx;
    double *dte = dnew(Nx), *Fl = dnew(Nx), *dF = dnew(Nx), *Rb = dnew(Nx);
    breaking_process(c, eta, etahat, u, t);
    ifft_cr_nx(c, dteta_hat, dte);
    for (int j = 0; j < Nx; j++) Fl[j] = -c->B[j] * pow(DELB, 2) * (c->depth[j] + eta[j]) * dte[j] * dte[j];
    gradient(Fl, c->dx, Nx, dF);
    for (int j = 0; j < Nx; j++) Rb[j] = 1 / (c->depth[j] + eta[j]) * dF[j];
    fft_rc_nx(c, Rb, c->Rb_hat);
    free(dte); free(Fl); free(dF); free(Rb);
}

/* rhs_HsF1/2/3 (1d/rhs.c:1-398) with define_forcing (1d/rhs.c:659) */
int or_rhs(or_ctx* c, double t, const double* z, double* dz) {
    int Nx = c->Nx;
    c->rhs_calls++;
    cpx *duH1 = cnew(Nx), *deH1 = cnew(Nx), *dpe = cnew(Nx), *dpu = cnew(Nx);
    cpx *duT = cnew(Nx), *deT = cnew(Nx);   /* joined H1 + adjusted nonlinear */
    define_delH1(c, z, duH1, deH1);
    if (c->model == 1) {
        hsf1(c, z, dpe, dpu);
        for (int i = 0; i < Nx; i++) { duT[i] = duH1[i]; deT[i] = deH1[i]; }
    } else {
        cpx *eu = cnew(Nx), *LeM = cnew(Nx), *u2 = cnew(Nx), *de3 = cnew(Nx), *du3 = cnew(Nx);
        hsf2(c, z, eu, LeM, u2, dpe, dpu);
        if (c->model == 3) hsf3(c, z, LeM, de3, du3);
        cpx *duN = cnew(Nx), *deN = cnew(Nx), *duA = cnew(Nx), *deA = cnew(Nx);
        for (int i = 0; i < Nx; i++) {
            double k = c->k[i];
            double du2r = -LeM[i].re - p1ik_re(k, eu[i].re, eu[i].im);
            double du2i = -LeM[i].im - p1ik_im(k, eu[i].re, eu[i].im);
            double de2r = -p1ik_re(k, u2[i].re, u2[i].im) / 2;
            double de2i = -p1ik_im(k, u2[i].re, u2[i].im) / 2;
            if (c->model == 3) {
                double du3r = du3[i].re, du3i = du3[i].im;
                double de3r = -p1ik_re(k, de3[i].re, de3[i].im), de3i = -p1ik_im(k, de3[i].re, de3[i].im);
                duN[i].re = du2r + du3r; duN[i].im = du2i + du3i;
                deN[i].re = de2r + de3r; deN[i].im = de2i + de3i;
            } else {
                duN[i].re = du2r; duN[i].im = du2i; deN[i].re = de2r; deN[i].im = de2i;
            }
        }
        adjust_delH(c, duA, deA, duN, deN);
        for (int i = 0; i < Nx; i++) {
            duT[i].re = duH1[i].re + duA[i].re; duT[i].im = duH1[i].im + duA[i].im;
            deT[i].re = deH1[i].re + deA[i].re; deT[i].im = deH1[i].im + deA[i].im;
        }
        free(eu); free(LeM); free(u2); free(de3); free(du3); free(duN); free(deN); free(duA); free(deA);
        if (c->brk) {
            double *eta = dnew(Nx), *u = dnew(Nx);
            cpx *eh = cnew(Nx), *uh = cnew(Nx);
            for (int j = 0; j < Nx; j++) { eh[j].re = z[j]; eh[j].im = z[Nx + j]; uh[j].re = z[2 * Nx + j]; uh[j].im = z[3 * Nx + j]; }
            ifft_cr_nx(c, eh, eta); ifft_cr_nx(c, uh, u);
            rhs_breaking(c, eta, eh, u, t, duT);
            free(eta); free(u); free(eh); free(uh);
        }
    }
    double pp = 0, ps = 0;
    if (c->has_influx) { pp = cspline_eval(&c->sp_in, t); ps = cspline_eval(&c->sp_skew, t); }
    int mode = !strcmp(c->propagation, "Uni+") ? 0 : !strcmp(c->propagation, "Uni-") ? 1 : !strcmp(c->propagation, "Bi") ? 2 : 3;
    for (int i = 0; i < Nx; i++) {
        double fr = 0, fi = 0;
        if (c->has_influx) {
            if (mode == 0) { fr = 0.5 * (pp * (c->gamX[i].re) - ps * (c->gamX_skew[i].re)); fi = 0.5 * (pp * (c->gamX[i].im) - ps * (c->gamX_skew[i].im)); }
            else if (mode == 1) { fr = 0.5 * (pp * (c->gamX[i].re) + ps * (c->gamX_skew[i].re)); fi = 0.5 * (pp * (c->gamX[i].im) + ps * (c->gamX_skew[i].im)); }
            else if (mode == 2) { fr = pp * (c->gamX[i].re); fi = pp * (c->gamX[i].im); }
        }
        double Sw = 0.0;   /* Swall_hat is zero without a wall (1d/functions.c:44-46) */
        double Rbr = c->Rb_hat[i].re, Rbi = c->Rb_hat[i].im;
        if (c->model == 3) {
            dz[i] = (duT[i].re + 2 * fr - dpe[i].re) * c->aal[i];
            dz[i + Nx] = (duT[i].im + 2 * fi - dpe[i].im) * c->aal[i];
        } else {
            dz[i] = (duT[i].re + Sw + 2 * fr - dpe[i].re) * c->aal[i];
            dz[i + Nx] = (duT[i].im + Sw + 2 * fi - dpe[i].im) * c->aal[i];
        }
        if (c->model == 1) { Rbr = 0; Rbi = 0; }
        dz[i + 2 * Nx] = (deT[i].re + Rbr - dpu[i].re) * c->aal[i];
        dz[i + 3 * Nx] = (deT[i].im + Rbi - dpu[i].im) * c->aal[i];
    }
    memcpy(c->dy, dz, sizeof(double) * 4 * (size_t)Nx);
    free(duH1); free(deH1); free(dpe); free(dpu); free(duT); free(deT);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* GSL rkf45 stepper, standard control (control_y_new) and legacy evolve.   */
/* ------------------------------------------------------------------------ */
static const double ah[] = {1.0 / 4.0, 3.0 / 8.0, 12.0 / 13.0, 1.0, 1.0 / 2.0};
static const double b3[] = {3.0 / 32.0, 9.0 / 32.0};
static const double b4[] = {1932.0 / 2197.0, -7200.0 / 2197.0, 7296.0 / 2197.0};
static const double b5[] = {8341.0 / 4104.0, -32832.0 / 4104.0, 29440.0 / 4104.0, -845.0 / 4104.0};
static const double b6[] = {-6080.0 / 20520.0, 41040.0 / 20520.0, -28352.0 / 20520.0, 9295.0 / 20520.0, -5643.0 / 20520.0};
static const double c1 = 902880.0 / 7618050.0;
static const double c3 = 3953664.0 / 7618050.0;
static const double c4 = 3855735.0 / 7618050.0;
static const double c5 = -1371249.0 / 7618050.0;
static const double c6 = 277020.0 / 7618050.0;
static const double ec[] = {0.0, 1.0 / 360.0, 0.0, -128.0 / 4275.0, -2197.0 / 75240.0, 1.0 / 50.0, 2.0 / 55.0};

/* rkf45_apply: propagates the 5th-order solution, yerr = 5th - 4th */
static int rkf45_apply(or_ctx* c, double t, double h, double* y, double* yerr, const double* dydt_in, double* dydt_out) {
    int D = 4 * c->Nx;
    double *k1 = c->k1, *k2 = c->k2, *k3 = c->k3, *k4 = c->k4, *k5 = c->k5, *k6 = c->k6, *yt = c->ytmp;
    memcpy(k1, dydt_in, sizeof(double) * (size_t)D);
    for (int i = 0; i < D; i++) yt[i] = y[i] + ah[0] * h * k1[i];
    or_rhs(c, t + ah[0] * h, yt, k2);
    for (int i = 0; i < D; i++) yt[i] = y[i] + h * (b3[0] * k1[i] + b3[1] * k2[i]);
    or_rhs(c, t + ah[1] * h, yt, k3);
    for (int i = 0; i < D; i++) yt[i] = y[i] + h * (b4[0] * k1[i] + b4[1] * k2[i] + b4[2] * k3[i]);
    or_rhs(c, t + ah[2] * h, yt, k4);
    for (int i = 0; i < D; i++) yt[i] = y[i] + h * (b5[0] * k1[i] + b5[1] * k2[i] + b5[2] * k3[i] + b5[3] * k4[i]);
    or_rhs(c, t + ah[3] * h, yt, k5);
    for (int i = 0; i < D; i++) yt[i] = y[i] + h * (b6[0] * k1[i] + b6[1] * k2[i] + b6[2] * k3[i] + b6[3] * k4[i] + b6[4] * k5[i]);
    or_rhs(c, t + ah[4] * h, yt, k6);
    for (int i = 0; i < D; i++) {
        const double di = c1 * k1[i] + c3 * k3[i] + c4 * k4[i] + c5 * k5[i] + c6 * k6[i];
        y[i] += h * di;
    }
    or_rhs(c, t + h, y, dydt_out);
    for (int i = 0; i < D; i++)
        yerr[i] = h * (ec[1] * k1[i] + ec[3] * k3[i] + ec[4] * k4[i] + ec[5] * k5[i] + ec[6] * k6[i]);
    return 0;
}

/* std_control_hadjust with a_y = 1, a_dydt = 0, order 5: -1 dec, 0 nil, 1 inc */
static int hadjust(or_ctx* c, const double* y, const double* yerr, const double* yp, double* h) {
    int D = 4 * c->Nx;
    const double S = 0.9, h_old = *h;
    double rmax = 2.2250738585072014e-308;   /* DBL_MIN */
    for (int i = 0; i < D; i++) {
        const double D0 = c->eps_rel * (1.0 * fabs(y[i]) + 0.0 * fabs(h_old * yp[i])) + c->eps_abs;
        const double r = fabs(yerr[i]) / fabs(D0);
        rmax = r > rmax ? r : rmax;
    }
    const unsigned ord = 5;
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

/* gsl_odeiv_evolve_apply (legacy), rkf45 uses dydt_in */
int or_evolve_apply(or_ctx* c, double* t, double t1, double* h, double* y) {
    int D = 4 * c->Nx;
    const double t0 = *t;
    double h0 = *h;
    double dt = t1 - t0;
    if ((dt < 0.0 && h0 > 0.0) || (dt > 0.0 && h0 < 0.0)) { set_err("step direction must match interval direction"); return 4; }
    memcpy(c->y0, y, sizeof(double) * (size_t)D);
    or_rhs(c, t0, y, c->dydt_in);
    for (;;) {
        int final_step;
        if ((dt >= 0.0 && h0 > dt) || (dt < 0.0 && h0 < dt)) { h0 = dt; final_step = 1; }
        else final_step = 0;
        rkf45_apply(c, t0, h0, y, c->yerr, c->dydt_in, c->dydt_out);
        if (final_step) *t = t1; else *t = t0 + h0;
        double h_old = h0;
        int st = hadjust(c, y, c->yerr, c->dydt_out, &h0);
        if (st == -1) {
            double t_curr = *t, t_next = (*t) + h0;
            if (fabs(h0) < fabs(h_old) && t_next != t_curr) {
                memcpy(y, c->y0, sizeof(double) * (size_t)D);
                c->rejected++;
                continue;
            }
            h0 = h_old;
        }
        break;
    }
    c->accepted++;
    *h = h0;
    return 0;
}

/* set_initial_ode (1d/functions.c:314), runup == 1 path */
int or_initial_state(or_ctx* c, double* y) {
    int nx = c->Nx;
    memset(y, 0, sizeof(double) * 4 * (size_t)nx);
    if (strcmp(c->initial, "zero") != 0) {
        double* w = dnew(nx);
        cpx* h = cnew(nx);
        for (int j = 0; j < nx; j++) w[j] = c->temp_u[j] * (1 - c->dampchar[j]);
        fft_rc_nx(c, w, h);
        for (int j = 0; j < nx; j++) { y[j + 2 * nx] = h[j].re; y[j + 3 * nx] = h[j].im; }
        for (int j = 0; j < nx; j++) w[j] = c->temp_wave[j] * (1 - c->dampchar[j]);
        fft_rc_nx(c, w, h);
        for (int j = 0; j < nx; j++) { y[j] = h[j].re; y[j + nx] = h[j].im; }
        free(w); free(h);
    }
    return 0;
}

/* ode_solver_Ham output loop (1d/functions.c:528-782): gauges (natural cspline
 * of eta and d_t eta over x, 1d/functions.c:500) and optional binary fields. */
int or_run(or_ctx* c, double* gauge_eta, double* gauge_dteta, double* tim_out, int cap) {
    int Nx = c->Nx, n = c->n, rows = 0;
    double* y = dnew(4 * Nx);
    or_initial_state(c, y);
    double t = c->ttrace[0], h = c->h0;
    double *etaf = dnew(Nx), *dtetaf = dnew(Nx), *uf = dnew(Nx), *phif = dnew(Nx);
    cpx *eh = cnew(Nx), *uh = cnew(Nx), *dh = cnew(Nx), *ph = cnew(Nx);
    FILE *fe = NULL, *fu = NULL, *fp = NULL;
    int NtoutIP = n / c->npartition, ip = 0;
    for (int i = 0; i < n; i++) {
        double ti = c->wave_t[i];
        while (t < ti) {
            if (or_evolve_apply(c, &t, ti, &h, y) != 0) { fprintf(stderr, "Time integration is failed\n"); break; }
        }
        for (int j = 0; j < Nx; j++) {
            eh[j].re = y[j]; eh[j].im = y[Nx + j]; uh[j].re = y[2 * Nx + j]; uh[j].im = y[3 * Nx + j];
            dh[j].re = c->dy[j]; dh[j].im = c->dy[j + Nx];
            if (c->k[j] == 0) { ph[j].re = 0; ph[j].im = 0; }
            else { ph[j].re = p1ik_re(-1 / c->k[j], uh[j].re, uh[j].im); ph[j].im = p1ik_im(-1 / c->k[j], uh[j].re, uh[j].im); }
        }
        ifft_cr_nx(c, eh, etaf); ifft_cr_nx(c, dh, dtetaf);
        if (c->write_fields && c->outdir[0]) {
            ifft_cr_nx(c, uh, uf); ifft_cr_nx(c, ph, phif);
            if (i % NtoutIP == 0) {
                ip++;
                char p[1024];
                if (fe) fclose(fe); if (fu) fclose(fu); if (fp) fclose(fp);
                /* print_xt (1d/functions.c:784-801): the rest partition is recognised by
                 * its length, N1 == Ntrest */
                int Ntrest = n - c->npartition * NtoutIP;
                int N1 = ip <= c->npartition ? NtoutIP : Ntrest;
                snprintf(p, sizeof p, "%s/Constants_%02d.dat", c->outdir, ip);
                FILE* fc = fopen(p, "wb");
                if (fc) {
                    double NX = (double)Nx, NT = (double)N1;
                    fwrite(&NX, sizeof(double), 1, fc);
                    fwrite(c->x, sizeof(double), (size_t)Nx, fc);
                    fwrite(&NT, sizeof(double), 1, fc);
                    if (N1 == Ntrest) fwrite(c->ttrace + (size_t)c->npartition * NtoutIP, sizeof(double), (size_t)N1, fc);
                    else fwrite(c->ttrace + (size_t)(ip - 1) * NtoutIP, sizeof(double), (size_t)N1, fc);
                    fwrite(c->depth, sizeof(double), (size_t)Nx, fc);
                    fwrite(c->k, sizeof(double), (size_t)Nx, fc);
                    fwrite(&c->nu_peak, sizeof(double), 1, fc);
                    fclose(fc);
                }
                snprintf(p, sizeof p, "%s/Hawassi_eta_%02d.dat", c->outdir, ip); fe = fopen(p, "wb");
                snprintf(p, sizeof p, "%s/Hawassi_u_%02d.dat", c->outdir, ip); fu = fopen(p, "wb");
                snprintf(p, sizeof p, "%s/Hawassi_phi_%02d.dat", c->outdir, ip); fp = fopen(p, "wb");
            }
            if (fe) fwrite(etaf, sizeof(double), (size_t)Nx, fe);
            if (fu) fwrite(uf, sizeof(double), (size_t)Nx, fu);
            if (fp) fwrite(phif, sizeof(double), (size_t)Nx, fp);
        }
        if (rows < cap) {
            if (tim_out) tim_out[rows] = t;
            if (c->ngauge > 0 && (gauge_eta || gauge_dteta)) {
                cspline s1, s2;
                cspline_init(&s1, c->x, etaf, Nx); cspline_init(&s2, c->x, dtetaf, Nx);
                for (int g = 0; g < c->ngauge; g++) {
                    if (gauge_eta) gauge_eta[(size_t)rows * c->ngauge + g] = cspline_eval(&s1, c->gauge[g]);
                    if (gauge_dteta) gauge_dteta[(size_t)rows * c->ngauge + g] = cspline_eval(&s2, c->gauge[g]);
                }
                cspline_free(&s1); cspline_free(&s2);
            }
            rows++;
        }
        if (c->t_stop > 0 && t >= c->t_stop) break;
    }
    if (fe) fclose(fe); if (fu) fclose(fu); if (fp) fclose(fp);
    if (c->brk && c->outdir[0]) {
        char p[1024]; snprintf(p, sizeof p, "%s/breaking.dat", c->outdir);
        FILE* fb = fopen(p, "w");
        if (fb) { fputs(c->blog ? c->blog : "", fb); fclose(fb); }
    }
    free(y); free(etaf); free(dtetaf); free(uf); free(phif); free(eh); free(uh); free(dh); free(ph);
    return rows;
}

void or_stats(const or_ctx* c, long long* r, long long* a, long long* j) {
    if (r) *r = c->rhs_calls; if (a) *a = c->accepted; if (j) *j = c->rejected;
}
const char* or_breaking_log(const or_ctx* c) { return c->blog ? c->blog : ""; }
int or_nx(const or_ctx* c) { return c->Nx; }
int or_nt(const or_ctx* c) { return c->n; }

double or_scalar(const or_ctx* c, const char* nm) {
#define S(name, expr) if (!strcmp(nm, name)) return (double)(expr);
    S("Nx", c->Nx) S("n", c->n) S("dx", c->dx) S("dt", c->dt) S("nu_peak", c->nu_peak) S("kp", c->kp)
    S("Tp_peak", c->Tp_peak) S("lambda_p", c->lambda_p) S("Hs_in", c->Hs_in) S("MaxEtaInit", c->MaxEtaInit)
    S("depthinf", c->depthinf) S("Cpeak", c->Cpeak) S("CpLeft", c->CpLeft) S("CpRight", c->CpRight)
    S("cutfracwn", c->cutfracwn) S("model", c->model) S("flat", c->flat) S("breaking", c->brk)
    S("Tstar", c->Tstar) S("KBC", c->KBC) S("TC", c->TC) S("xbstart", c->xbstart) S("xbend", c->xbend)
    S("idx_inf", c->idx_inf) S("Xinflux", c->Xinflux) S("ngauge", c->ngauge) S("has_influx", c->has_influx)
    S("eps_abs", c->eps_abs) S("eps_rel", c->eps_rel) S("h0", c->h0) S("flag", c->flag) S("ITERbdt", c->ITERbdt)
    S("nref", c->nref) S("Xstart", c->Xstart) S("Xend", c->Xend) S("length", c->length)
    S("propagation", !strcmp(c->propagation, "Uni+") ? 0 : !strcmp(c->propagation, "Uni-") ? 1 : !strcmp(c->propagation, "Bi") ? 2 : 3)
#undef S
    return NAN;
}

int or_table(const or_ctx* c, const char* nm, double* out, int cap) {
    int Nx = c->Nx;
#define R(name, ptr, len) if (!strcmp(nm, name)) { if (!(ptr)) return 0; int L_ = (len) < cap ? (len) : cap; memcpy(out, ptr, sizeof(double) * (size_t)L_); return L_; }
#define C(name, ptr) if (!strcmp(nm, name)) { if (!(ptr)) return 0; if (cap < 2 * Nx) return 0; for (int i = 0; i < Nx; i++) { out[i] = (ptr)[i].re; out[i + Nx] = (ptr)[i].im; } return 2 * Nx; }
    R("x", c->x, Nx) R("k", c->k, Nx) R("depth", c->depth, Nx) R("dampchar", c->dampchar, Nx) R("dampcoef", c->dampcoef, Nx)
    R("aal", c->aal, Nx) R("ChiAdj", c->ChiAdj, Nx) R("Csqr", c->Csqr, Nx) R("L", c->L, Nx) R("M0im", c->M0im, Nx)
    R("gam_min", c->gam_min, Nx) R("gam_mid", c->gam_mid, Nx) R("gam_plus", c->gam_plus, Nx)
    R("Csq_min", c->Csq_min, Nx) R("Csq_mid", c->Csq_mid, Nx) R("Csq_plus", c->Csq_plus, Nx)
    R("insig", c->insig, c->n) R("insig_skew", c->insig_skew, c->n) R("ttrace", c->ttrace, c->n) R("dy", c->dy, 4 * Nx)
    R("spatgamX", c->spatgamX, Nx) R("B", c->B, Nx) R("gauge", c->gauge, c->ngauge)
    C("gamX", c->gamX) C("gamX_skew", c->gamX_skew) C("Rb_hat", c->Rb_hat)
    R("CsqK", c->CsqK, (c->CsqK ? c->nref * Nx : 0)) R("gamK", c->gamK, (c->gamK ? c->nref * Nx : 0))
#undef R
#undef C
    return -1;
}

/* ------------------------------------------------------------------------ */
/* Kinematics: read_kinematics (1d/functions.c:3555-3669) and kinematic_modul */
/* (1d/kinematic_modul.c:1-247): velocity potential derivatives and pressure */
/* under the surface on the overlay window [xinterv1, xinterv2] x zoutIP.    */
/* ------------------------------------------------------------------------ */
/* sinhcosh2IP (1d/functions.c:1889-1928): two-depth interpolation weights of
 * cosh/sinh(kappa D) between Dmin and Dplus, kappa the linear wavenumber of nupeak */
static void sinhcosh2ip(int sizD, const double* D, double Dmin, double Dplus, const double* k, double nupeak,
                        double* gmin, double* gplus) {
    for (int j = 0; j < sizD; j++) {
        const double kap = (D[j] == 0) ? k[2] : invers_omega(nupeak, D[j]);
        const double cmin = cosh(kap * Dmin), cplus = cosh(kap * Dplus), cD = cosh(kap * D[j]);
        const double smin = sinh(kap * Dmin), splus = sinh(kap * Dplus), sD = sinh(kap * D[j]);
        const double det = cmin * splus - cplus * smin;
        gmin[j] = (splus * cD - cplus * sD) / det;
        gplus[j] = (-(smin * cD) + cmin * sD) / det;
    }
}

static int kin_setup(or_ctx* c) {
    const int Nx = c->Nx;
    if (c->nsurf < 2 || c->ndeep < 1) { set_err("kinematics: nsurf must be >= 2 and ndeep >= 1"); return -1; }
    for (int i = 0; i < Nx; i++)
        if (c->depth[i] == 0) { set_err("kinematics: runup (zero depth) is not supported"); return -1; }
    double zs1, zs2;
    if (strcmp(c->min_z, "default") == 0) {
        zs1 = -2.5 * c->Hs_in;
        if (strcmp(c->initial, "user_defined") == 0) zs1 = -0.6 * c->Hs_in;
    } else zs1 = atof(c->min_z);
    if (strcmp(c->max_z, "default") == 0) {
        zs2 = 2.5 * c->Hs_in;
        if (strcmp(c->initial, "user_defined") == 0) zs2 = 0.6 * c->Hs_in;
    } else zs2 = atof(c->max_z);
    c->kin_maxD = search_max_val(c->depth, Nx);
    c->kin_minD = search_min_val(c->depth, Nx);
    c->kin_i1 = closest(c->x, c->xinterv1, Nx);
    c->kin_i2 = closest(c->x, c->xinterv2, Nx);
    c->kin_nx = c->kin_i2 - c->kin_i1 + 1;
    if (c->kin_nx < 1) { set_err("kinematics: empty overlay window"); return -1; }
    c->kin_maxEta = zs2;
    c->kin_minEta = zs1;
    const int ns = c->nsurf, nd = c->ndeep, nz = ns + nd;
    double* zs = malloc(sizeof(double) * ns);
    double* zd = malloc(sizeof(double) * nd);
    const double dzs = (zs2 - zs1) / (ns - 1);
    const double kpk = invers_omega(c->nu_peak, c->kin_maxD);
    for (int j = 0; j < ns; j++) zs[j] = zs1 + j * dzs;
    /* deeper levels: Riemann upper sum of the cosh profile (1d/functions.c:3627-3637) */
    const double Flux = 1 / (kpk * sinh(kpk * c->kin_maxD)) * (cosh(kpk * (c->kin_maxD + zs1)) - 1);
    const double tol = Flux / nd;
    zd[0] = -1 * (zs1 - dzs);
    for (int i = 1; i < nd; i++)
        zd[i] = zd[i - 1] + (tol / (sinh(kpk * (c->kin_maxD - zd[i - 1])) / sinh(kpk * c->kin_maxD)));
    c->kin_nz = nz;
    c->kin_z = malloc(sizeof(double) * nz);
    for (int i = 0; i < ns; i++) c->kin_z[i] = zs[i];
    for (int i = ns; i < nz; i++) c->kin_z[i] = -1 * zd[i - ns];
    for (int i = 0; i < nz; i++)            /* sorting (1d/functions1.c) */
        for (int j = i + 1; j < nz; j++)
            if (c->kin_z[j] < c->kin_z[i]) { double tt = c->kin_z[i]; c->kin_z[i] = c->kin_z[j]; c->kin_z[j] = tt; }
    free(zs); free(zd);
    return 0;
}

int or_kin_dims(const or_ctx* c, int* nxout, int* nzout) {
    if (!c || !c->kin) return -1;
    if (nxout) *nxout = c->kin_nx;
    if (nzout) *nzout = c->kin_nz;
    return 0;
}

int or_kin_grid(const or_ctx* c, double* xout, double* zout) {
    if (!c || !c->kin) return -1;
    if (xout) for (int i = 0; i < c->kin_nx; i++) xout[i] = c->x[c->kin_i1 + i];
    if (zout) memcpy(zout, c->kin_z, sizeof(double) * c->kin_nz);
    return 0;
}

/* gradient (1d/functions1.c): one-sided at the ends */
static void gradient1(const double* a, double d, int n, double* g) {
    g[0] = (a[1] - a[0]) / d;
    g[n - 1] = (a[n - 1] - a[n - 2]) / d;
    for (int i = 1; i < n - 1; i++) g[i] = (a[i + 1] - a[i - 1]) / (2 * d);
}

int or_kinematics(or_ctx* c, double t, double tprev, const double* y, const double* dy, double* eta_cut, double* P,
                  double* dxphi, double* dzphi, double* ax, double* az) {
    if (!c || !c->kin) { set_err("kinematics: the deck has kinematic no"); return -1; }
    const int Nx = c->Nx, nxo = c->kin_nx, nz = c->kin_nz, NH = 100;
    const double* k = c->k;
    /* the output stage's fields (1d/functions.c:570-596) */
    cpx *eh = cnew(Nx), *uh = cnew(Nx), *dh = cnew(Nx), *dph = cnew(Nx);
    double *eta = dnew(Nx), *dteta = dnew(Nx);
    for (int j = 0; j < Nx; j++) {
        eh[j].re = y[j]; eh[j].im = y[Nx + j];
        uh[j].re = y[2 * Nx + j]; uh[j].im = y[3 * Nx + j];
        dh[j].re = dy[j]; dh[j].im = dy[Nx + j];
        if (k[j] == 0) { dph[j].re = 0; dph[j].im = 0; }
        else {   /* prod_1ik(-1/k, du^): (0 - (-1/k) Im) + i (0 + (-1/k) Re) */
            const double a = -1 / k[j];
            dph[j].re = (0 * dy[2 * Nx + j]) - (a * dy[3 * Nx + j]);
            dph[j].im = (0 * dy[3 * Nx + j]) + (a * dy[2 * Nx + j]);
        }
    }
    ifft_cr_nx(c, eh, eta);
    ifft_cr_nx(c, dh, dteta);
    /* kinematic_modul */
    const double nupeak = c->nu_peak;
    const double Hplus = c->kin_maxEta + c->kin_maxD, Hmin = c->kin_minEta + c->kin_minD;
    const double dhtot = (Hplus - Hmin) / NH;
    double Htot[101], gHm0[101], gHp0[101], DZtot[101], gDm0[101], gDp0[101];
    for (int i = 0; i < NH + 1; i++) Htot[i] = Hmin + i * dhtot;
    sinhcosh2ip(NH + 1, Htot, Hmin, Hplus, k, nupeak, gHm0, gHp0);
    double cHm[101], cHp[101], cDm[101], cDp[101];
    or_cspline_coeffs(NH + 1, Htot, gHm0, cHm);
    or_cspline_coeffs(NH + 1, Htot, gHp0, cHp);
    const double DZmin0 = 0, DZplus0 = Hplus;
    for (int i = 0; i < NH + 1; i++) DZtot[i] = DZmin0 + i * (DZplus0 - DZmin0) / NH;
    sinhcosh2ip(NH + 1, DZtot, DZmin0, DZplus0, k, nupeak, gDm0, gDp0);
    or_cspline_coeffs(NH + 1, DZtot, gDm0, cDm);
    or_cspline_coeffs(NH + 1, DZtot, gDp0, cDp);
    cpx* phi = cnew(Nx);
    double *H = dnew(Nx), *gH = dnew(Nx), *gD = dnew(Nx), *coshH = dnew(Nx), *tanhH = dnew(Nx);
    for (int j = 0; j < Nx; j++) {
        H[j] = (eta[j] + c->depth[j]);
        const double gm = or_cspline_eval(NH + 1, Htot, gHm0, cHm, H[j]);
        const double gp = or_cspline_eval(NH + 1, Htot, gHp0, cHp, H[j]);
        coshH[j] = gm * cosh(k[j] * Hmin) + gp * cosh(k[j] * Hplus);
        tanhH[j] = gm * tanh(k[j] * Hmin) + gp * tanh(k[j] * Hplus);
        if (k[j] == 0) { phi[j].re = 0; phi[j].im = 0; }
        else { phi[j].re = (uh[j].im) / k[j]; phi[j].im = -(uh[j].re) / k[j]; }
    }
    gradient1(H, c->dx, Nx, gH);
    gradient1(c->depth, c->dx, Nx, gD);
    const int flatb = (c->kin_minD == c->kin_maxD);
    double *DZ = dnew(Nx), *coshZ = dnew(Nx), *sinhZ = dnew(Nx);
    cpx *fa = cnew(Nx), *ft = cnew(Nx), *fx = cnew(Nx), *fz = cnew(Nx);
    double *fac = dnew(Nx), *tdt = dnew(Nx), *tdx = dnew(Nx), *tdz = dnew(Nx);
    for (int zz = 0; zz < nz; zz++) {
        const double zo = c->kin_z[zz];
        if (flatb) {
            for (int j = 0; j < Nx; j++) {
                coshZ[j] = cosh(k[j] * (zo + c->depth[0]));
                sinhZ[j] = sinh(k[j] * (zo + c->depth[0]));
            }
        } else {
            for (int j = 0; j < Nx; j++) {
                DZ[j] = c->depth[j] + zo;
                if (DZ[j] < 0) DZ[j] = 0;
            }
            const double DZplus = search_max_val(DZ, Nx);
            double DZmin = search_min_val(DZ, Nx);
            if (DZmin < 0) DZmin = 0;
            if (DZmin == DZplus) {
                for (int j = 0; j < Nx; j++) {
                    coshZ[j] = cosh(k[j] * (zo + c->depth[0]));
                    sinhZ[j] = sinh(k[j] * (zo + c->depth[0]));
                }
            } else {
                for (int j = 0; j < Nx; j++) {
                    double gm = or_cspline_eval(NH + 1, DZtot, gDm0, cDm, DZ[j]);
                    double gp = or_cspline_eval(NH + 1, DZtot, gDp0, cDp, DZ[j]);
                    if (DZ[j] == DZmin) { gm = 1; gp = 0; }
                    if (DZ[j] == DZplus) { gm = 0; gp = 1; }
                    coshZ[j] = gm * cosh(k[j] * DZmin) + gp * cosh(k[j] * DZplus);
                    sinhZ[j] = gm * sinh(k[j] * DZmin) + gp * sinh(k[j] * DZplus);
                }
            }
        }
        for (int j = 0; j < Nx; j++) {
            const double ratio = coshZ[j] / coshH[j];
            fa[j].re = phi[j].re * ratio * (-k[j] * tanhH[j]);
            fa[j].im = phi[j].im * ratio * (-k[j] * tanhH[j]);
            ft[j].re = dph[j].re * ratio;
            ft[j].im = dph[j].im * ratio;
            fz[j].re = phi[j].re * k[j] * sinhZ[j] / coshH[j];
            fz[j].im = phi[j].im * k[j] * sinhZ[j] / coshH[j];
            fx[j].re = -k[j] * phi[j].im * ratio;
            fx[j].im = k[j] * phi[j].re * ratio;
        }
        ifft_cr_nx(c, fa, fac);
        ifft_cr_nx(c, ft, tdt);
        ifft_cr_nx(c, fz, tdz);
        ifft_cr_nx(c, fx, tdx);
        for (int xo = 0; xo < nxo; xo++) {
            const int j = c->kin_i1 + xo;
            double vt, vx, vz;
            if ((zo > eta[j]) || (zo < -c->depth[j])) { vt = NAN; vz = NAN; vx = NAN; }
            else {
                vt = tdt[j] + dteta[j] * fac[j];
                vx = tdx[j] + gH[j] * fac[j] + gD[j] * tdz[j];
                vz = tdz[j];
            }
            const size_t o = (size_t)xo * nz + zz;
            dxphi[o] = vx;
            dzphi[o] = vz;
            P[o] = -vt - G * zo - 0.5 * (pow(vx, 2) + 2 * vz);
            ax[o] = (vx - 0) / (t - tprev);
            az[o] = (vz - 0) / (t - tprev);
        }
    }
    for (int xo = 0; xo < nxo; xo++) eta_cut[xo] = eta[c->kin_i1 + xo];
    void* ps[] = {eh, uh, dh, dph, eta, dteta, phi, H, gH, gD, coshH, tanhH, DZ, coshZ, sinhZ, fa, ft, fx, fz, fac, tdt,
                  tdx, tdz};
    for (size_t i = 0; i < sizeof ps / sizeof ps[0]; i++) free(ps[i]);
    return 0;
}
