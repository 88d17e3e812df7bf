// hw_device.cuh -- device-side data of one member (tank realisation) and the
// shared helpers of the RHS / stepper kernels.
#pragma once

#include <cuda_runtime.h>

#include "hw_fft.cuh"

namespace hwdev {

constexpr double kG = 9.80665;       // gravity (1d/header.h:27)
constexpr double kDelb = 1.2;        // breaking coefficient delta_b (1d/header.h:29)
constexpr int kScratch = 12;         // N-point double2 scratch arrays per member
constexpr int kMaxRef = 16;          // reference depths of the varying-depth operator

// status codes stored per member (mirrors GSL: 0 success)
enum : int { kOk = 0, kStepFailed = 1, kNonFinite = 2, kBudget = 3 };

// crest record of the breaking state machine (1d/header.h:48-56)
struct Crest {
  int Bindex, BindexNow, DirProp, Bcount;
  double Ucrest, Bposition, Btime;
};

// breaking state of one member, in global memory
struct BrkDev {
  int flag, ITERbdt, ITERbn, n_touched;
  int npk;            // candidate crests found by the parallel criterion
  int any_above;      // eta above MaxEtaInit somewhere in the breaking window
  int cap;            // Nx / 4
  int dirty_cb, dirty_cbn, dirty_cbp;   // records [0, dirty) may be nonzero
  Crest* cb;          // CrestBreak (from the criterion)
  Crest* cbn;         // CrestBreakNew
  Crest* cbp;         // CrestBreakPrev
  int* id_node_end;
  int* nodes;         // Break_nodes of the current call
  int* touched;       // nodes where B was set by the previous call (reset lazily)
  int* pk;            // peak indices (unsorted) found by the criterion
  double* B;          // breaking indicator per grid point
  double* log;        // breaking.dat records: t, count, nodes...
  long long log_len, log_cap;
};

struct DevMember {
  // geometry / model
  int N, C, M, logC;
  int model, flat, nref, brk, has_influx, prop_mode, n_in, exact;
  double invN, dx, eps_abs, eps_rel;
  // spectral tables, permuted "cyclic" order (position c*M + i holds wavenumber c + C*i)
  const double* k;
  const double* aal;
  const double* c1;     // (Csqr/g) k
  const double* gk;     // g k
  const double* M0im;   // -k Csqr/g
  const double* L;      // k^2 Csqr / g
  const double2* gamX;
  const double2* gamXs;
  const double* Csq;    // [nref][N]
  // physical tables, natural order
  const double* dcoef;
  const double* dchar;
  const double* chi;
  const double* depth;
  const double* gam;    // [nref][N]
  // influx splines over ttrace
  const double* tt;
  const double* ins;
  const double* insc;
  const double* skw;
  const double* skwc;
  const double2* tw;    // exp(-2 pi i q / N)
  // breaking parameters
  double KBC, TC, Tstar, MaxEtaInit, dt_in;
  int xbstart, xbend, xbendL, xbstartR, lenIF, ILL, IFF;
  // RK buffers (2N double2, [eta^ | u^], permuted)
  double2* y;
  double2* ynew;
  double2* kb[7];       // k1..k6, kout
  double2* zs;          // stage input
  double2* sc[kScratch];
  BrkDev* bk;
  // output stage: gauge series on the device (1d/functions.c:700-760)
  int ngauge;
  const double* xg;     // grid x (natural order)
  const double* gpos;   // gauge positions
  const int* gidx;      // spline interval of each gauge (-1: outside the grid)
  double* gout;         // [n][2 ngauge]: eta, d eta / dt at the gauges per output sample
  double* gtim;         // [n]: time of each output sample
  double* fields;       // [n][3][N]: eta, u, phi per output sample (nullptr: not kept)
  // control state
  double t, h, t1;      // current time, step, target of a single evolve_apply
  int i_out, i_stop;    // next output index, stop index (exclusive)
  int status, k1_valid;
  long long rhs_calls, accepted, rejected, rhs_budget;
  double last_rmax;
};

}  // namespace hwdev
