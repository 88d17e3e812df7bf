/*
 * hawassi_b200.h -- C ABI of the B200 engine for HAWASSI's 1D pseudo-spectral
 * Hamiltonian RHS and its RKF45 time stepping.
 *
 * Plain C linkage, plain pointers and sizes.  State vectors use the
 * reference's layout: 4*Nx doubles [Re eta^ | Im eta^ | Re u^ | Im u^] in FFTW
 * order (1d/rhs.c:33-38).  All pointers passed in are HOST pointers; device
 * memory is owned by the context.  Every call returns 0 on success (GSL_SUCCESS)
 * and a nonzero code otherwise, with a message in hw_last_error().  A context
 * is used by one host thread at a time (the reference's RHS is not re-entrant
 * either).
 */
#ifndef HAWASSI_B200_H
#define HAWASSI_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hw_ctx hw_ctx;

typedef struct hw_opts {
    double eps_abs;          /* <= 0: the reference's 1e-5 (1d/functions.c:529) */
    double eps_rel;          /* <= 0: the reference's 1e-4 (1d/functions.c:530) */
    double h0;               /* <= 0: the reference's first step 1e-4 (1d/functions.c:541) */
    unsigned long long seed; /* phase seed for wavename = jonswap (reference: srand(time(0)));
                                member m of an ensemble uses seed + m, its signal synthesised
                                on the device with every other jonswap member's */
    int nref;                /* varying depth: 0 or 3 = three reference depths (Up3IP), 2 = Up2IP,
                                4..16 = that many log-spaced reference depths, each point on its
                                bracketing pair (no counterpart in the reference) */
    int exact_sequence;      /* 1: evaluate the RHS exactly where GSL does even when it is stateless */
    int cluster;             /* CTAs per member, power of two (0 = automatic) */
    int device;              /* CUDA device ordinal */
    int slice;               /* grid points per CTA when cluster == 0 (0 = 2048) */
    int resident;            /* evolve launches of an ensemble: 0 = one cluster per member
                                (members started longest first); -1 = a persistent grid per
                                grid-size class, its clusters pulling members (longest first)
                                from a device queue, sized to the class's share of the
                                resident clusters; n > 0 = a persistent grid of at most n
                                clusters per class */
} hw_opts;

/* Replaces the reference's set-up (1d/main.cc:42-226): parse <workdir>/input.txt and
 * the files it names, build the tables on the host, upload them. NULL on error. */
hw_ctx* hw_create(const char* workdir, const hw_opts* opts);

/* Batched ragged ensemble: one member per deck directory, uneven grid sizes allowed;
 * all members advance together in one launch per grid-size class. */
hw_ctx* hw_ensemble_create(const char* const* workdirs, int n_members, const hw_opts* opts);
/* The same with the grid points per CTA chosen per member (0: opts->slice); the
 * autotuner (hawassi_c_b200/autotune.py) picks them per grid size by timing. */
hw_ctx* hw_ensemble_create_sliced(const char* const* workdirs, int n_members, const hw_opts* opts,
                                  const int* member_slice);

void        hw_destroy(hw_ctx* ctx);
const char* hw_last_error(const hw_ctx* ctx);   /* ctx may be NULL (last create error) */
int         hw_members(const hw_ctx* ctx);
int         hw_nx(const hw_ctx* ctx, int member);
int         hw_nt(const hw_ctx* ctx, int member); /* output/influx samples of the member */

/* Initial spectral state of set_initial_ode (1d/functions.c:314). */
int hw_initial_state(hw_ctx* ctx, int member, double* y);

/* One RHS evaluation; replaces rhs_HsF1/2/3 (1d/rhs.c:1,96,243) including their side
 * effects (breaking state machine, breaking log, the global dy copy). */
int hw_rhs(hw_ctx* ctx, int member, double t, const double* y, double* dydt);

/* gsl_odeiv_system.function-compatible entry point (member 0, params = hw_ctx*):
 *   gsl_odeiv_system sys = {hw_gsl_rhs, NULL, 4 * Nx, ctx};   (1d/functions.c:71-89) */
int hw_gsl_rhs(double t, const double* y, double* dydt, void* params);

/* No counterpart in the reference.  One RHS evaluation like hw_rhs, for callers
 * that cannot allocate device memory at call time (for instance code that runs
 * under a device-memory budget managed by another framework's pool, or that must
 * not trigger allocations between set-up and tear-down).  y_dev and dydt_dev are
 * DEVICE pointers (4*Nx doubles, reference layout) owned by the caller; the call
 * allocates nothing: its scratch is a 1 MiB static device array held by every GPU
 * that loads the library, so Nx is limited to 4096 (larger grids are rejected with
 * an error).  The first call on a device looks up the array's device address and
 * sets the kernels' attributes (once per device, under a lock); make that call
 * before any stream capture.  All calls share the one array: calls that overlap on
 * the GPU (different streams, contexts or threads) race.  No scratch field needs
 * to start at zero.  cuda_stream NULL: the default stream.  The call makes the
 * context's device current for the launch and restores the caller's device.
 * Side effects are hw_rhs's: the member's RHS counter grows by one and, on a
 * breaking deck, the member's breaking state (crest records, B, the breaking
 * log) advances, as the reference's RHS does on every call.  That state belongs
 * to the context, so order the call against the context's own work: it runs on
 * cuda_stream, not on the context's stream, so a call made while hw_run or
 * hw_evolve_apply work of the same member is in flight races with it. */
int hw_rhs_noalloc(hw_ctx* ctx, int member, double t, const double* y_dev, double* dydt_dev, void* cuda_stream);

/* Replaces gsl_odeiv_evolve_apply(e, c, s, &sys, &t, t1, &h, y) with rkf45 and
 * control_y (1d/functions.c:550): one accepted step, whole step on the device. */
int hw_evolve_apply(hw_ctx* ctx, int member, double* t, double t1, double* h, double* y);

/* The time loop of ode_solver_Ham (1d/functions.c:546-553) for every member at once:
 * integrate through the member's output samples [i_out, i_stop), clipping steps at
 * each sample time like the reference. i_stop < 0 means all samples. Asynchronous on
 * the context's stream. */
int hw_run(hw_ctx* ctx, int i_stop);
/* A launch stops a member after 400000 RHS evaluations (status 3, resumed by the next
 * hw_run), so no launch runs unbounded. */
/* Same with a stop index per member (i_stop[m] <= current index: the member holds). */
int hw_run_members(hw_ctx* ctx, const int* i_stop);
/* Same, stopping at the last output sample whose time is <= t_end. */
int hw_run_to_time(hw_ctx* ctx, double t_end);

/* Current state of a member (synchronises the context's stream). */
int hw_get_state(hw_ctx* ctx, int member, double* t, double* h, double* y);
/* Overwrite the state of a member (t, h, y in the reference layout, output index i_out). */
int hw_set_state(hw_ctx* ctx, int member, double t, double h, const double* y, int i_out);
/* Back to t0, h0 and the initial state, breaking state and counters cleared. */
int hw_reset(hw_ctx* ctx);

/* Counters of a member: RHS evaluations, accepted / rejected steps, status (0 ok). */
int hw_member_stats(hw_ctx* ctx, int member, long long* rhs_calls, long long* accepted,
                    long long* rejected, int* status);
/* The last RHS output (the reference's global dy, 1d/rhs.c:224-227), reference layout. */
int hw_last_dydt(hw_ctx* ctx, int member, double* dydt);
/* Breaking log records (t, node count, nodes...) as doubles; returns the record count
 * written, *len receives the number of doubles. */
int hw_breaking_log(hw_ctx* ctx, int member, double* out, long long cap, long long* len);

/* Seeded JONSWAP influx signals of many members in one device launch
 * (jonswap_influx, 1d/influx_lib.c:137-255; srand(time(0)) replaced by a seeded
 * splitmix64 stream, the spectrum's integer exponent 5/4 and the phase
 * off-by-one kept).  Member m's signal has Nt_m = int((Tend - T0)/dt + 1) samples
 * at T0 + j dt; the signals are concatenated in member order into eta_out.
 * Returns the total sample count (writes only when cap covers it), -1 on error. */
typedef struct hw_jonswap {
    double T0, Tend, dt;        /* the deck's time block                        */
    double Tp, Hs, gamma;       /* spectrum                                     */
    double nTramp;              /* ramp length in peak periods (0: ramp "no")   */
    unsigned long long seed;
} hw_jonswap;
int hw_jonswap_influx(const hw_jonswap* specs, int n, double* eta_out, long long cap, int device);

/* Kinematics of a member whose deck has "kinematic yes" (kinematic_modul,
 * 1d/kinematic_modul.c:1-247; grid of read_kinematics, 1d/functions.c:3555-3669):
 * at the member's current time, from its state and the last RHS (the reference's
 * etaf, u_hatf, dtetaf, dtphi_hatf), on the overlay window [xinterv1, xinterv2]
 * (nx_out points) and the nz_out levels zoutIP (surface layer plus the deeper
 * Riemann-sum levels, ascending).  Outputs are [nx_out][nz_out], x-major, as the
 * reference's fwrite of Ptot, dxPhi, dzPhi, dt_dxPHI, dt_dzPHI: NaN above the
 * surface or below the bed; the accelerations are (velocity - 0) / (t - tprev)
 * with the caller's tprev, as the reference computes them.  eta_cut [nx_out].
 * Any output pointer may be NULL.  Returns 0, nonzero with hw_last_error set
 * (e.g. kinematic no, runup). */
int hw_kinematics_dims(hw_ctx* ctx, int member, int* nx_out, int* nz_out);
int hw_kinematics_grid(hw_ctx* ctx, int member, double* x_out, double* z_out);
int hw_kinematics(hw_ctx* ctx, int member, double tprev, double* eta_cut, double* P, double* dxphi,
                  double* dzphi, double* dtdxphi, double* dtdzphi);

/* All members' states, concatenated in member order (4*Nx doubles each), host buffers. */
int hw_get_states(hw_ctx* ctx, double* y_all);
int hw_set_states(hw_ctx* ctx, const double* y_all);

/* Device time (ms) of the last hw_run launch of each grid-size class, with the
 * class's member count and grid size; returns the number of classes. */
int hw_class_timing(hw_ctx* ctx, double* ms, int* members, int* grid_n, int cap);

/* Replace the K reference depths and the per-point weights gam[K][Nx] of a
 * varying-depth member created with nref = K (no counterpart in the reference: used to
 * install the learned operator's weights). */
int hw_set_operator_weights(hw_ctx* ctx, int member, int K, const double* depths, const double* gam);

/* The learned operator's per-point network (no counterpart in the reference):
 * 5 features -> 32 -> 32 (tanh) -> 4 softmax weights, FP32, trained on the GPU.
 * A training record is 45 floats: 5 features, the 8x4 band matrix
 * G[m][j] = C^2(kappa_m, D_j) and 8 targets T[m]; loss = mean_m ((G w - T)_m / T_m)^2. */
typedef struct hw_mlp hw_mlp;
int         hw_mlp_sizes(int* n_in, int* n_hidden, int* n_out, int* n_band, int* n_params);
hw_mlp*     hw_mlp_create(unsigned long long seed, int device);
void        hw_mlp_destroy(hw_mlp* mlp);
const char* hw_mlp_last_error(const hw_mlp* mlp);
int         hw_mlp_get_params(hw_mlp* mlp, float* params);
int         hw_mlp_set_params(hw_mlp* mlp, const float* params);
/* summed loss and parameter gradients over n host records */
int         hw_mlp_grad(hw_mlp* mlp, const float* records, int n, float* grad, float* loss);
int         hw_mlp_grad_device(hw_mlp* mlp, const float* records_dev, int n, float* grad, float* loss);
/* Adam over minibatches of `batch` records for `epochs` passes; losses[e] = mean loss */
int         hw_mlp_train(hw_mlp* mlp, const float* records, int n, int epochs, int batch, float lr, float* losses);
/* per-point weights w[4][n] (double) from n feature rows of 5 floats */
int         hw_mlp_infer(hw_mlp* mlp, const float* features, int n, double* w);

/* Energy diagnostic (no counterpart in the reference): the quadratic Hamiltonian
 * 1/2 int (g eta^2 + u (C^2/g) u) dx of a state in spectral form (Parseval), with C^2
 * at the influx depth.  y: a host state in the reference layout, or NULL for the
 * member's current state. */
int hw_energy(hw_ctx* ctx, int member, const double* y, double* energy);

/* Host-only (no GPU needed): build the set-up of <workdir> and copy the named table
 * (x, k, depth, dampchar, dampcoef, aal, ChiAdj, Csqr, L, M0im, gamX, gamX_skew, insig,
 * insig_skew, ttrace, y0, gam_min/plus/mid, Csq_min/plus/mid) or scalar (Nx, n, dx, dt,
 * nu_peak, kp, lambda_p, Hs_in, MaxEtaInit, depthinf, Tstar, xbstart, xbend, cutfracwn,
 * Tp_peak) into out.  Returns the full length, -1 on error. */
int hw_deck_table(const char* workdir, const hw_opts* opts, const char* name, double* out, int cap);

/* Run on a caller-provided cudaStream_t (NULL: the context's own stream; pass
 * cudaStreamLegacy explicitly for the legacy default stream). */
/* Output stage (1d/functions.c:700-760) computed on the device at every output
 * sample of hw_run: elevation and d eta / dt at the gauges of gauges.dat (GSL
 * natural cubic spline of the physical fields, print_data_gauge), rows of ngauge
 * values per sample, and the sample times.  Returns the rows copied (samples
 * reached so far, at most cap) or -1. */
int hw_gauges(hw_ctx* ctx, int member, double* eta, double* dteta, double* tim, int cap);
int hw_ngauge(const hw_ctx* ctx, int member);

/* Keep eta, u and phi of every output sample on the device (enable = 1, before
 * hw_run; 3 * Nx doubles per sample of the member's deck). */
int hw_enable_fields(hw_ctx* ctx, int member, int enable);
/* Write the reference's output files of a member into outdir (1d/functions.c:557-801):
 * Constants_NN.dat and Hawassi_{eta,u,phi}_NN.dat per partition (when fields are
 * kept), Hawassi_eta_gauge.txt / Hawassi_dteta_gauge.txt (when the deck has gauges)
 * and breaking.dat (breaking decks).  Returns the samples written or -1. */
int hw_write_outputs(hw_ctx* ctx, int member, const char* outdir);

int hw_set_stream(hw_ctx* ctx, void* cuda_stream);
int hw_synchronize(hw_ctx* ctx);

/* FP64 FMA throughput of the device in TFLOP/s (a DFMA microbenchmark: eight
 * independent FMA chains per thread on every SM, best of five launches): the
 * denominator of the FP64 roofline.  Returns a negative value on error. */
double hw_fp64_peak_tflops(int device);

/* ------------------------------------------------------------------------ */
/* 2D twin (HS1-HS3): rhs_AB2_2DF_uv / rhs_AB2_2DB_uv (walls, kinematic breaking, */
/* both bottoms), rhs_AB3_2DF_uv, rhs_AB1_2D*_uv and the                      */
/* gsl_odeiv2 rkf45 loop of ode_solver_uv (2d/fun_odesolver.c:2565-2647,     */
/* 4458-4540).  State: 6*nx*ny doubles [Re eta^|Im eta^|Re u^|Im u^|Re v^|    */
/* Im v^], row-major i*nx + j (2d/main.c:198-201).  The operator tables are   */
/* the ones the reference's 2D set-up leaves in its globals (dominfo, Oprt,   */
/* ChiAdj, newGam, SkewGam, Spline_Signal); the caller passes them here.      */
/* ------------------------------------------------------------------------ */
typedef struct hw2d_ctx hw2d_ctx;

typedef struct hw2d_tables {
    int nx, ny;                 /* powers of two, 64..1024                      */
    int model;                  /* evolinfo.model: 2 = HS2; 1 = HS1 (no breaking process);
                                   3 = HS3 (flat bottom: rhs_AB3_2DF_uv) */
    int propagation;            /* 0 = Uni+, 1 = Uni-, 2 = Bi (vertical line)   */
    double cpeak;               /* Oprt.Cpeak                                   */
    const double* kx;           /* [nx] dominfo.kx                              */
    const double* ky;           /* [ny] dominfo.ky                              */
    const double* c2d;          /* [ny*nx] Oprt.C2d                             */
    const double* l2d;          /* [ny*nx] Oprt.L2d                             */
    const double* aal;          /* [ny*nx] dominfo.aal                          */
    const double* charac;       /* [ny*nx] dominfo.fbdy.charac                  */
    const double* chiadj;       /* [ny*nx] ChiAdj                               */
    const double* newgam;       /* [ny*nx] newGam[j][i] at i*nx + j             */
    const double* skewgam;      /* [ny*nx] SkewGam[j][i] at i*nx + j (or NULL)  */
    int nt;                     /* samples per line signal (0: wavename zero)   */
    const double* tsig;         /* [nt] dominfo.t                               */
    const double* sig;          /* [ny*nt] Signal[i] (row i of the line)        */
    const double* sigskew;      /* [ny*nt] SkewSignal[i] (or NULL)              */
    /* varying bottom, two reference depths (rhs_AB2_2DB_uv, ninterp = 2); all NULL
     * for a flat bottom (rhs_AB2_2DF_uv, which reads c2d and l2d instead) */
    const double* gam_min;      /* [ny*nx] Oprt.InterpD.Gam_min                 */
    const double* gam_plus;     /* [ny*nx] Oprt.InterpD.Gam_plus                */
    const double* csq_min;      /* [ny*nx] Oprt.InterpD.Csqr2d_min              */
    const double* csq_plus;     /* [ny*nx] Oprt.InterpD.Csqr2d_plus             */
    const double* om2_min;      /* [ny*nx] Oprt.InterpD.Om2dSq_min              */
    const double* om2_plus;     /* [ny*nx] Oprt.InterpD.Om2dSq_plus             */
    /* harbour walls: dominfo.wallchar (1 - cutoff(refl_coef) inside the walls,
     * 2d/functions.c:260-390); NULL for no wall.  On the flat bottom walls also
     * enter fun_delphiH1hat (2d/fun_odesolver.c:2100-2219, both branches). */
    const double* wallchar;     /* [ny*nx]                                      */
    /* kinematic breaking (2d/breaking.c: parambreak, breaking_process; fun_sbreaking
     * 2d/fun_odesolver.c:985-1019), two-depth tables only; breaking = 0 leaves the
     * fields below unread.  The scalars are parambreak's pb.* values. */
    int breaking;
    const double* bathy;        /* [ny*nx] dominfo.bathy.data (= -depth)        */
    const double* brchar;       /* [ny*nx] pb.Char (cfSA, 0 where cfSA or ChiAdj < 1) */
    const double* x;            /* [nx] dominfo.x                               */
    const double* y;            /* [ny] dominfo.y                               */
    double dx, dy;              /* dominfo.dx, dominfo.dy (also read by walls with
                                   refl_coef == 1 on the flat bottom)            */
    double max_eta_init;        /* pb.MaxEtaInit = 0.9 Hs / 2                   */
    double tstar;               /* pb.Tstar = Tchar Tp                          */
    double rsearch;             /* pb.Rsearch = 2 pi / kp / 4                   */
    double kbc, tc, delb;       /* pb.KBC, pb.TC, pb.delb (1.5)                 */
    double cur_u;               /* dominfo.U                                    */
    double t0, dt_out;          /* dominfo.t[0], dominfo.dt (breaking.dat cadence) */
    double refl_coef;           /* walls: refl_coef (the flat RHS's fun_delphiH1hat takes its
                                   flux branch when it is 1)                     */
    /* three reference depths (ninterp = 3, HSSgen_3depth): the middle depth's tables
     * (served by the general path); NULL for two reference depths */
    const double* gam_mid;      /* [ny*nx] Oprt.InterpD.Gam_mid                 */
    const double* csq_mid;      /* [ny*nx] Oprt.InterpD.Csqr2d_mid              */
    const double* om2_mid;      /* [ny*nx] Oprt.InterpD.Om2dSq_mid              */
    /* K reference depths, 2 <= nrefk <= 16 (no counterpart in the reference: HSSgen's
     * sum over K depths, used by the plain 16-reference operator and the learned
     * 4-reference blend); nrefk = 0 leaves the three fields below unread, nrefk > 0
     * replaces the min/plus/mid tables above (which must then be NULL) */
    int nrefk;
    const double* gam_k;        /* [K][ny*nx] per-point weight of each depth    */
    const double* csq_k;        /* [K][ny*nx] C^2 of each reference depth       */
    const double* om2_k;        /* [K][ny*nx] Omega^2 of each reference depth   */
} hw2d_tables;

/* The directional JONSWAP line signal of the 2D set-up's jonswap_influx
 * (2d/functions.c:2310-2446, vertical influx line) on the device: for the nt samples
 * t0 + i dt and the nlines line points y[j],
 *   eta[j*nt + i]  = ramp_t[i] ramp_y[j] sum_c a[c] cos(-w[c] t_i + phi[c] + k[c] sin(theta[c] + mdir) (y[j] - y0)),
 *   skew[j*nt + i] = the same sum of sin (the quadrature the 2D source takes beside it),
 * in the [line][sample] layout of hw2d_tables.sig / .sigskew.  The nc components (the
 * reference draws nt/2 of them, one direction each, from srand(time(0)); the Python
 * set-up draws them from a seeded stream, decks2d.reference_directional_components)
 * are host arrays, as are the outputs; the call allocates and frees its device
 * buffers and restores the caller's current device.  Returns 0, or 1 with the reason
 * in hw2d_influx_last_error(). */
int hw2d_directional_influx(int nt, double t0, double dt, int nlines, const double* y, double y0, int nc,
                            const double* a, const double* w, const double* k, const double* theta,
                            const double* phi, double mdir, const double* ramp_t, const double* ramp_y,
                            double* eta, double* skew, int device);
const char* hw2d_influx_last_error(void);

/* opts: eps_abs/eps_rel (<= 0: the 2D reference's 1e-3 / 1e-2, 2d/main.c:196-197),
 * h0 (<= 0: dt/5 of the signal grid, 2d/fun_odesolver.c:2580), device. */
hw2d_ctx*   hw2d_create(const hw2d_tables* tables, const hw_opts* opts);
void        hw2d_destroy(hw2d_ctx* ctx);
const char* hw2d_last_error(const hw2d_ctx* ctx);   /* ctx may be NULL */
int         hw2d_nx(const hw2d_ctx* ctx);
int         hw2d_ny(const hw2d_ctx* ctx);

/* One RHS evaluation (replaces rhs_AB2_2DF_uv). */
int hw2d_rhs(hw2d_ctx* ctx, double t, const double* y, double* dydt);
/* gsl_odeiv2_system.function-compatible (params = hw2d_ctx*):
 *   gsl_odeiv2_system sys = {hw2d_gsl_rhs, NULL, 6 * nx * ny, ctx};  (2d/main.c:205) */
int hw2d_gsl_rhs(double t, const double* y, double* dydt, void* params);
/* gsl_odeiv2_evolve_apply(e, c, s, &sys, &t, t1, &h, y) with rkf45 + control_y. */
int hw2d_evolve_apply(hw2d_ctx* ctx, double* t, double t1, double* h, double* y);

/* Device-resident state: set it, run the evolve loop to t1 (the inner loop of
 * ode_solver_uv) without returning to the host, read it back. */
int hw2d_set_state(hw2d_ctx* ctx, double t, double h, const double* y);
int hw2d_get_state(hw2d_ctx* ctx, double* t, double* h, double* y);   /* y may be NULL */
int hw2d_run_to_time(hw2d_ctx* ctx, double t1);
int hw2d_stats(const hw2d_ctx* ctx, long long* rhs_calls, long long* accepted, long long* rejected);
/* kernels this context has launched so far (each node of a replayed graph counted) */
long long hw2d_launches(const hw2d_ctx* ctx);
/* Breaking state after the last RHS (the globals B, Sb_xhat, Sb_yhat, flagbr and
 * CBPrev[0].NB of 2d/breaking.c): B [ny*nx], Sb as interleaved complex [2*ny*nx];
 * any pointer may be NULL.  Returns -1 when the context has no breaking. */
int hw2d_breaking_fields(hw2d_ctx* ctx, double* B, double* sbx, double* sby, int* flagbr, int* ncrest);
/* breaking.dat (2d/breaking.c:707-718): record r is times[r] and counts[r] node
 * pairs (x index, y index), all records' pairs concatenated in nodes.  Copies at
 * most cap_rec records and cap_nodes pairs; returns the number of records (-1:
 * no breaking, -2: the device log overflowed and stopped). */
int hw2d_breaking_log(hw2d_ctx* ctx, double* times, int* counts, int* nodes, int cap_rec, long long cap_nodes);
long long hw2d_breaking_log_nodes(hw2d_ctx* ctx);

/* Output stage of ode_solver_uv (2d/fun_odesolver.c:2565-2843).
 * eta, u, v in physical space of the current device state: ifftw_2d_c2r of a copy
 * of each spectrum (2d/functions1.c:523-557; the loop's :2648-2666), [ny*nx] each,
 * row-major; any pointer may be NULL. */
int hw2d_fields(hw2d_ctx* ctx, double* eta, double* u, double* v);

typedef struct hw2d_outputs {
    const char* outdir;         /* prefix of every file name (arg2, with its '/')      */
    int nt;                     /* dominfo.Nt output samples                           */
    const double* tout;         /* [nt] dominfo.t, the output times (tinterv)          */
    double dt;                  /* dominfo.dt (time axis of Constant_01.dat)           */
    int npartition;             /* "No of Partition": files hold Nt / npartition samples */
    int uv_every_sample;        /* 0: u, v of each partition's first sample only (kinematic
                                   "no", :2736-2748); 1: every sample (what kinematic "yes"
                                   writes ahead of the kinematics module, :2756-2767) */
    double hs, kp, wp;          /* seainfo.Hs, kp, wp                                  */
    const double* x;            /* [nx] dominfo.x                                      */
    const double* y;            /* [ny] dominfo.y                                      */
    double dx, dy;              /* dominfo.dx, dominfo.dy (gauge indices)              */
    const double* kx;           /* [nx] dominfo.kx                                     */
    const double* ky;           /* [ny] dominfo.ky                                     */
    const double* bathy;        /* [ny*nx] dominfo.bathy.data                          */
    const double* cfsa;         /* [ny*nx] cfSA                                        */
    const double* chiadjphi;    /* [ny*nx] ChiAdjPhi; NULL when wavename is zero       */
    int ngauge;                 /* gauges.dat lines (0: no gauge files)                */
    const double* xgauge;       /* [ngauge]                                            */
    const double* ygauge;       /* [ngauge]                                            */
} hw2d_outputs;

/* The time loop of ode_solver_uv from the current device state (the reference
 * starts it at t = tout[0] with h = (tout[1] - tout[0]) / 5: hw2d_set_state).  For
 * every sample i it evolves to tout[i] on the device, transforms eta, u, v there
 * and writes, with the reference's names under outdir:
 *   Constant_01.dat        print_xt (:2532-2563) at i = 0 (:2687-2718)
 *   Hawassi_eta_NN.dat     float32 eta [ny][nx] of every sample of partition NN (:2727-2734)
 *   Hawassi_u_NN.dat, Hawassi_v_NN.dat   float32 u, v (uv_every_sample)
 *   Hawassi_{eta,u,v}_gauge.dat          print_data_gauges_uv text (:427-476)
 *   breaking.dat           the breaking records (2d/breaking.c:707-718), at the end
 * Kinematics, runup, coupling and the gnuplot frames are not part of it.  Like the
 * reference (:2819-2823; fun_max2darray's running comparison ends NaN exactly when
 * the last grid point is NaN), it stops when the last grid point of eta is NaN.  Returns the samples written, or -1 (hw2d_last_error). */
int hw2d_run_outputs(hw2d_ctx* ctx, const hw2d_outputs* spec);

int hw2d_set_stream(hw2d_ctx* ctx, void* cuda_stream);
int hw2d_synchronize(hw2d_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
