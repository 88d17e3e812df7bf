/*
 * hw_oracle.h -- CPU oracle for the HAWASSI 1D pseudo-spectral RHS and its
 * RKF45 time stepping.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: it is linked by the
 * test-suite, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg,
 * and never by the product library (hawassi_c_b200/).  It restates, in plain
 * C, the reference's algorithm for this path (file:line citations on every
 * function in hw_oracle.c), plus the published algorithms of the third-party
 * pieces the reference links but does not ship (FFTW3 c2c DFT, GSL rkf45 +
 * standard step control + legacy evolve, GSL natural cubic spline, GSL Newton
 * root finder).
 *
 * Parity pin: the restatement is checked against the golden outputs shipped
 * with the reference deck 1d/Testcases/1dFBr005Bor (breaking.dat onset line,
 * gauge series, Constants_01.dat grids) by tests/test_oracle_golden.py.
 */
#ifndef HW_ORACLE_H
#define HW_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_ctx or_ctx;

typedef struct or_opts {
    double eps_abs;        /* <= 0: reference value 1e-5 (1d/functions.c:529) */
    double eps_rel;        /* <= 0: reference value 1e-4 (1d/functions.c:530) */
    double h0;             /* <= 0: reference value 1e-4 (1d/functions.c:541) */
    double t_stop;         /* > 0: stop the output loop once tim[i] >= t_stop */
    unsigned long long seed; /* phase seed for wavename = jonswap (reference: time(0)) */
    int    nref;           /* 0 or 3: Up3IP (reference default, main.cc:35); 2: Up2IP */
    int    write_fields;   /* 1: write Hawassi_{eta,u,phi}_NN.dat like the reference */
    const char* outdir;    /* output directory for breaking.dat and gauge files, or NULL */
} or_opts;

/* Parse <workdir>/input.txt (+ influx.dat, bath.dat, initial.dat, gauges.dat)
 * and build every table.  Returns NULL on error (message in or_last_error()). */
or_ctx* or_create(const char* workdir, const or_opts* opts);
void    or_destroy(or_ctx* c);
const char* or_last_error(void);

int    or_nx(const or_ctx* c);
int    or_nt(const or_ctx* c);          /* number of influx/output samples n */
double or_scalar(const or_ctx* c, const char* name);
/* Copy a named table (k, x, depth, dampchar, dampcoef, aal, ChiAdj, gamX, gamX_skew,
 * Csqr, L, M0im, gam_min, gam_mid, gam_plus, Csq_min, Csq_mid, Csq_plus, insig,
 * insig_skew, ttrace, dy) into out (complex tables are [Re|Im], 2*Nx).  Returns count. */
int    or_table(const or_ctx* c, const char* name, double* out, int cap);

/* The state y is the reference's 4*Nx layout [Re eta^ | Im eta^ | Re u^ | Im u^]. */
int    or_initial_state(or_ctx* c, double* y);
/* One RHS evaluation, with the reference's side effects (breaking state, dy). */
int    or_rhs(or_ctx* c, double t, const double* y, double* dydt);
/* gsl_odeiv_evolve_apply restated (rkf45 + control_y). Returns 0 on success. */
int    or_evolve_apply(or_ctx* c, double* t, double t1, double* h, double* y);
/* Full output loop of ode_solver_Ham; gauge values land in gauge_eta/gauge_dteta
 * (n_out x ngauge, row-major) when non-NULL.  Returns number of output rows. */
int    or_run(or_ctx* c, double* gauge_eta, double* gauge_dteta, double* tim_out, int cap_rows);
void   or_stats(const or_ctx* c, long long* rhs_calls, long long* accepted, long long* rejected);
/* Breaking log (the breaking.dat lines) as one text buffer. */
const char* or_breaking_log(const or_ctx* c);
/* Reset breaking state and counters (new run on the same tables). */
void   or_reset(or_ctx* c);

/* Kinematics (kinematic_modul, 1d/kinematic_modul.c) on the overlay window
 * [xinterv1, xinterv2] x zoutIP of a deck with "kinematic yes": sizes, grid,
 * and the fields at time t for the state y and its RHS dy (reference layout),
 * with the reference's tprev.  Outputs are [nx_out][nz_out] (x-major) except
 * eta_cut [nx_out].  Returns 0, or -1 when the deck has no kinematics. */
int    or_kin_dims(const or_ctx* c, int* nx_out, int* nz_out);
int    or_kin_grid(const or_ctx* c, double* xout, double* zout);
int    or_kinematics(or_ctx* c, double t, double tprev, const double* y, const double* dy, double* eta_cut,
                     double* P, double* dxphi, double* dzphi, double* dtdxphi, double* dtdzphi);

/* jonswap_influx (1d/influx_lib.c:289) with the seeded splitmix64 phases: the influx
 * signal at T0 + j dt, j < Nt = int((Tend - T0)/dt + 1).  Returns Nt (writes eta
 * when cap >= Nt), -1 on a too short signal. */
int    or_jonswap_signal(double T0, double Tend, double dt, double Tp, double Hs, double gamma, double nTramp,
                         unsigned long long seed, double* eta_out, int cap);

/* Plain FFT utilities (FFTW sign convention, unnormalised), exposed for tests. */
void   or_fft(int n, const double* re_in, const double* im_in, double* re_out, double* im_out, int sign);

#ifdef __cplusplus
}
#endif
#endif
