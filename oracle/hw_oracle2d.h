/*
 * hw_oracle2d.h -- CPU oracle for the HAWASSI 2D pseudo-spectral RHS (flat
 * bottom: rhs_AB1_2DF_uv / rhs_AB2_2DF_uv; varying bottom with two reference
 * depths: rhs_AB2_2DB_uv) and its gsl_odeiv2 rkf45 time stepping.
 *
 * TEST INFRASTRUCTURE ONLY: linked by the test-suite, __graft_entry__.smoke() and
 * bench.py's CPU legs, never by the product library.  It restates
 * 2d/fun_odesolver.c (RHS, term functions, symmetrisation, fun_adjust,
 * fun_source, ode_solver_uv) on the operator tables the reference's set-up
 * builds (kx, ky, C2d, L2d, aal, fbdy.charac, ChiAdj, newGam, SkewGam, the
 * influx-line signals): the tables are inputs here, exactly as they are globals
 * there.
 *
 * Parity unpinned: the reference ships no outputs for its 2D decks, so this
 * restatement is checked only by its own consistency tests (linear dispersion of
 * a free wave, Hermitian symmetry, the adjust identity at ChiAdj = 1).
 */
#ifndef HW_ORACLE2D_H
#define HW_ORACLE2D_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or2d_ctx or2d_ctx;

typedef struct or2d_tables {
    int nx, ny;                 /* grid, x fastest: index i*nx + j, i = y row  */
    int model;                  /* 1 = HS1, 2 = HS2                            */
    int propagation;            /* 0 = Uni+, 1 = Uni-, 2 = Bi (vertical line)  */
    double cpeak;               /* Oprt.Cpeak                                  */
    const double* kx;           /* [nx]  dominfo.kx (freqspace)                */
    const double* ky;           /* [ny]  dominfo.ky                            */
    const double* c2d;          /* [ny*nx] Oprt.C2d                            */
    const double* l2d;          /* [ny*nx] Oprt.L2d                            */
    const double* aal;          /* [ny*nx] dominfo.aal                         */
    const double* charac;       /* [ny*nx] dominfo.fbdy.charac                 */
    const double* chiadj;       /* [ny*nx] ChiAdj                              */
    const double* newgam;       /* [ny*nx] newGam[j][i] stored at i*nx + j     */
    const double* skewgam;      /* [ny*nx] SkewGam, same layout; NULL: none    */
    int nt;                     /* samples of each line signal (0: no source)  */
    const double* tsig;         /* [nt]                                        */
    const double* sig;          /* [ny*nt] INsig of row i at sig[i*nt + n]     */
    const double* sigskew;      /* [ny*nt] skew signal, same layout            */
    /* varying bottom, two reference depths (ninterp = 2): NULL for a flat bottom */
    const double* gam_min;      /* [ny*nx] Oprt.InterpD.Gam_min                */
    const double* gam_plus;     /* [ny*nx] Oprt.InterpD.Gam_plus               */
    const double* csq_min;      /* [ny*nx] Oprt.InterpD.Csqr2d_min             */
    const double* csq_plus;     /* [ny*nx] Oprt.InterpD.Csqr2d_plus            */
    const double* om2_min;      /* [ny*nx] Oprt.InterpD.Om2dSq_min             */
    const double* om2_plus;     /* [ny*nx] Oprt.InterpD.Om2dSq_plus            */
    const double* wallchar;     /* [ny*nx] dominfo.wallchar, NULL: no wall                  */
    /* kinematic breaking (2d/breaking.c; fun_sbreaking 2d/fun_odesolver.c:985-1019), HS2
     * (flat or two-depth bottom); breaking = 0 leaves every field below unread */
    int breaking;
    const double* bathy;        /* [ny*nx] dominfo.bathy.data (= -depth)        */
    const double* brchar;       /* [ny*nx] pb.Char: cfSA, 0 where cfSA < 1 or ChiAdj < 1 */
    const double* x;            /* [nx] dominfo.x                               */
    const double* y;            /* [ny] dominfo.y                               */
    double dx, dy;              /* dominfo.dx, dominfo.dy                       */
    double max_eta_init;        /* pb.MaxEtaInit = 0.9 Hs / 2                   */
    double tstar;               /* pb.Tstar = Tchar Tp                          */
    double rsearch;             /* pb.Rsearch = 2 pi / kp / 4                   */
    double kbc, tc, delb;       /* pb.KBC, pb.TC, pb.delb (1.5)                 */
    double cur_u;               /* dominfo.U (ambient current)                  */
    double t0, dt_out;          /* dominfo.t[0], dominfo.dt (breaking.dat cadence) */
    double refl_coef;           /* walls: the reflection coefficient (the flat RHS branches on 1) */
    /* three reference depths (ninterp = 3, HSSgen_3depth): the middle depth's tables;
     * NULL for two reference depths */
    const double* gam_mid;      /* [ny*nx] Oprt.InterpD.Gam_mid                */
    const double* csq_mid;      /* [ny*nx] Oprt.InterpD.Csqr2d_mid             */
    const double* om2_mid;      /* [ny*nx] Oprt.InterpD.Om2dSq_mid             */
    /* K reference depths (no counterpart in the reference: the generalisation of
     * HSSgen_2depth / _3depth to K depths that the plain 16-reference and the learned
     * 4-reference operators use); nrefk = 0 leaves these unread, nrefk >= 2 replaces
     * the min/plus/mid tables above */
    int nrefk;
    const double* gam_k;        /* [K][ny*nx] per-point weights                */
    const double* csq_k;        /* [K][ny*nx] C^2 of each reference depth      */
    const double* om2_k;        /* [K][ny*nx] Omega^2 of each reference depth  */
} or2d_tables;

/* Copies every table.  eps <= 0 selects the reference's 2D values (abs 1e-3,
 * rel 1e-2, 2d/main.c:196-197).  Returns NULL on error (or2d_last_error). */
/* The directional JONSWAP influx of jonswap_influx (2d/functions.c:2226-2446): the
 * components of the Nt-sample time grid t (uniform) -- w = freqspace(t[Nt-1] - t[0], Nt)
 * (2d/functions.c:1810) restricted to its first Nt/2 entries, k(w) at depth (exact
 * dispersion by Newton), a = sqrt(2 S(w) dw) from fun_jonswap (Hs, Tp, gamma; JS[0] = 0,
 * trapezoid m0), one direction each from the cos^2s distribution by inverse-CDF
 * interpolation (GSL natural cspline) of the given uniforms rn (s <= 0: long-crested,
 * every direction 0), phase 2 pi ru -- and the line signal they add up to along a
 * vertical influx line,
 *   eta[j][i] = ramp_t[i] ramp_y[j] sum_c a_c cos(-w_c t_i + phi_c + k_c sin(theta_c + mdir) (y_j - y0)),
 * with skew[j][i] the same sum of sin (the quadrature the 2D source takes beside it).
 * rn and ru hold nt / 2 uniforms each; the outputs a, w, k, theta, phi nt / 2 entries. */
void or2d_jonswap_components(int nt, const double* t, double Hs, double Tp, double gamma, double s, double depth,
                             const double* rn, const double* ru, double* a, double* w, double* k, double* theta,
                             double* phi);
void or2d_directional_signal(int nt, const double* t, int nlines, const double* y, double y0, int nc,
                             const double* a, const double* w, const double* k, const double* theta,
                             const double* phi, double mdir, const double* ramp_t, const double* ramp_y,
                             double* eta, double* skew);

or2d_ctx* or2d_create(const or2d_tables* tb, double eps_abs, double eps_rel);
void or2d_destroy(or2d_ctx* c);
const char* or2d_last_error(void);

/* One RHS evaluation; y, dydt in the reference layout 6*nx*ny
 * [Re eta^ | Im eta^ | Re u^ | Im u^ | Re v^ | Im v^]. */
int or2d_rhs(or2d_ctx* c, double t, const double* y, double* dydt);
/* gsl_odeiv2_evolve_apply restated (rkf45 + control_y).  Returns 0 on success. */
int or2d_evolve_apply(or2d_ctx* c, double* t, double t1, double* h, double* y);
/* evolve_apply until t == t1 (the inner loop of ode_solver_uv) */
int or2d_run_to(or2d_ctx* c, double* t, double t1, double* h, double* y);
void or2d_stats(const or2d_ctx* c, long long* rhs_calls, long long* accepted, long long* rejected);
/* Breaking state (2d/breaking.c globals).  tprev is the reference's global of that
 * name: or2d_evolve_apply sets it to t on entry (ode_solver_uv sets it after every
 * evolve_apply, 2d/fun_odesolver.c:2646); the breaking update of an RHS runs only
 * when its t exceeds tprev. */
void or2d_set_tprev(or2d_ctx* c, double tprev);
/* B (the last RHS's breaking coefficient), Sb_xhat/Sb_yhat as [ny*nx] complex
 * pairs (re, im interleaved), flagbr and the number of tracked crests. */
int or2d_brk_fields(const or2d_ctx* c, double* B, double* sbx, double* sby, int* flagbr, int* ncrest);
/* breaking.dat records: times[r], node counts cnt[r], nodes as (x, y) pairs in
 * order.  Returns the number of records (copies at most cap_rec records and
 * cap_nodes node pairs). */
int or2d_brk_log(const or2d_ctx* c, double* times, int* cnt, int* nodes, int cap_rec, int cap_nodes);
long long or2d_brk_log_nodes(const or2d_ctx* c);
/* 2D complex DFT (FFTW sign convention, unnormalised), for tests. */
void or2d_fft(int nx, int ny, const double* re_in, const double* im_in, double* re_out, double* im_out, int sign);
/* the reference's fftwcomplex_2d_sym applied in place to a complex [ny*nx] array */
void or2d_sym(int nx, int ny, double* re, double* im);

/* eta, u, v in physical space of a state y (6*nx*ny, reference layout):
 * ifftw_2d_c2r of a copy of each spectrum (2d/functions1.c:523-557, called by
 * ode_solver_uv at 2d/fun_odesolver.c:2648-2666).  Any output may be NULL. */
void or2d_fields(int nx, int ny, const double* y, double* eta, double* u, double* v);

/* the output files of ode_solver_uv's time loop (fields named as in the engine's
 * hw2d_outputs) */
typedef struct or2d_outputs {
    const char* outdir;
    int nt;
    const double* tout;
    double dt;
    int npartition;
    int uv_every_sample;
    double hs, kp, wp;
    const double *x, *y;
    double dx, dy;
    const double *kx, *ky, *bathy, *cfsa, *chiadjphi;
    int ngauge;
    const double *xgauge, *ygauge;
} or2d_outputs;

/* ode_solver_uv (2d/fun_odesolver.c:2565-2843) without kinematics, runup,
 * coupling and plots, from (t, h, y): evolve to every output time, write
 * Constant_01.dat, Hawassi_{eta,u,v}_NN.dat, the gauge files and breaking.dat.
 * Returns the samples written or -1 (or2d_last_error). */
int or2d_run_outputs(or2d_ctx* c, double* t, double* h, double* y, const or2d_outputs* o);

#ifdef __cplusplus
}
#endif
#endif
