// hw_stepper.cuh -- the RKF45 stage / error-norm / step-control loop of one
// member, entirely on the device.  It restates GSL's rkf45 stepper (Fehlberg
// tableau, 5th-order solution propagated), the standard control built by
// gsl_odeiv_control_y_new (a_y = 1, a_dydt = 0, safety 0.9, order 5, decrease
// above 1.1, increase below 0.5, factors clamped to [0.2, 5]) and the legacy
// gsl_odeiv_evolve_apply (dydt_in at every call, final-step clipping, retry on
// decrease).  The reference calls these at 1d/functions.c:532-553.
#pragma once

#include "hw_rhs.cuh"

namespace hwdev {

struct Bufs {
  double2* y;
  double2* yn;
  double2* k[7];   // k1..k6, kout
};

// stage input zs = y + h sum_j b_sj k_j for stage s = 2..6 (GSL's expression forms)
template <int M>
__device__ __forceinline__ void stage_input(Ctx<M>& X, const Bufs& B, int s, double h) {
  const DevMember& d = X.d;
  const StageSrc st{B.y, {B.k[0], B.k[1], B.k[2], B.k[3], B.k[4]}, s, h};
  for (int part = 0; part < 2; ++part) {
    const int off = part * d.N;
    HW_FOREACH(X) {
      (void)idx;
      d.zs[p + off] = stage_val(st, p + off);
    }
  }
}

// max over the member (all CTAs of the cluster); identical result in every thread
template <int M>
__device__ __forceinline__ double member_max(Ctx<M>& X, double v) {
  const DevMember& d = X.d;
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = X.tid >> 5;
  constexpr int NW = Ctx<M>::T / 32;
  __syncthreads();
  if ((X.tid & 31) == 0) X.red[w] = v;
  __syncthreads();
  double m = X.red[0];
  for (int i = 1; i < NW; ++i) m = fmax(m, X.red[i]);
  if (d.C > 1) {
    cg::cluster_group cl = cg::this_cluster();
    if (X.tid == 0) X.red[NW] = m;
    cl.sync();
    m = *cl.map_shared_rank(X.red + NW, 0);
    for (int r = 1; r < d.C; ++r) m = fmax(m, *cl.map_shared_rank(X.red + NW, r));
    cl.sync();
  }
  return m;
}

// ynew = y + h sum c_i k_i ; yerr = h sum ec_i k_i ; returns max |yerr| / D0
template <int M>
__device__ __forceinline__ double final_combine(Ctx<M>& X, const Bufs& B, double h) {
  const DevMember& d = X.d;
  double rm = 2.2250738585072014e-308;   // DBL_MIN
  bool bad = false;
  for (int part = 0; part < 2; ++part) {
    const int off = part * d.N;
    HW_FOREACH(X) {
      (void)idx;
      const int q = p + off;
      const double2 y = B.y[q], a = B.k[0][q], c = B.k[2][q], e = B.k[3][q], f = B.k[4][q], g = B.k[5][q];
      const double dix = radd(radd(radd(radd(rmul(RK_c1, a.x), rmul(RK_c3, c.x)), rmul(RK_c4, e.x)), rmul(RK_c5, f.x)),
                              rmul(RK_c6, g.x));
      const double diy = radd(radd(radd(radd(rmul(RK_c1, a.y), rmul(RK_c3, c.y)), rmul(RK_c4, e.y)), rmul(RK_c5, f.y)),
                              rmul(RK_c6, g.y));
      const double2 yn = make_double2(radd(y.x, rmul(h, dix)), radd(y.y, rmul(h, diy)));
      B.yn[q] = yn;
      const double ex = rmul(h, radd(radd(radd(radd(rmul(RK_ec1, a.x), rmul(RK_ec3, c.x)), rmul(RK_ec4, e.x)),
                                           rmul(RK_ec5, f.x)), rmul(RK_ec6, g.x)));
      const double ey = rmul(h, radd(radd(radd(radd(rmul(RK_ec1, a.y), rmul(RK_ec3, c.y)), rmul(RK_ec4, e.y)),
                                           rmul(RK_ec5, f.y)), rmul(RK_ec6, g.y)));
      const double rx = fabs(ex) / fabs(radd(rmul(d.eps_rel, fabs(yn.x)), d.eps_abs));
      const double ry = fabs(ey) / fabs(radd(rmul(d.eps_rel, fabs(yn.y)), d.eps_abs));
      bad = bad || !(rx == rx) || !(ry == ry) || isinf(yn.x) || isinf(yn.y);
      rm = fmax(rm, fmax(rx, ry));
    }
  }
  if (bad) rm = __longlong_as_double(0x7ff0000000000000ULL);   // +inf: forces a failure path
  return member_max(X, rm);
}

struct StepState {
  double t, h;
  int status, k1_valid;
  long long rhs, acc, rej;
};

template <int M>
__device__ __forceinline__ void rhs_into(Ctx<M>& X, StepState& S, double t, double2* out) {
  // the flat HS2 RHS directly (one call level less on the ensemble's hot path)
  if (X.d.model == 2 && X.d.flat) rhs_hs2_flat<M>(X, t, out);
  else rhs_eval<M>(X, t, out);
  ++S.rhs;
}

// one RHS evaluation at the state src itself (the RHS copies it into zs)
template <int M>
__device__ __forceinline__ void rhs_at(Ctx<M>& X, StepState& S, double t, const double2* src, double2* out) {
  const StageSrc st{src, {nullptr, nullptr, nullptr, nullptr, nullptr}, 1, 0.0};
  X.stg = &st;
  rhs_into(X, S, t, out);
  X.stg = nullptr;
}

// copy a state buffer into the stage-input buffer
template <int M>
__device__ __forceinline__ void load_stage(Ctx<M>& X, const double2* src) {
  const DevMember& d = X.d;
  for (int part = 0; part < 2; ++part) {
    const int off = part * d.N;
    HW_FOREACH(X) {
      (void)idx;
      d.zs[p + off] = src[p + off];
    }
  }
}

// gsl_odeiv_evolve_apply with rkf45 and control_y, one member
template <int M>
__device__ __noinline__ void evolve_apply(Ctx<M>& X, Bufs& B, StepState& S, double t1) {
  const DevMember& d = X.d;
  const double t0 = S.t;
  double h0 = S.h;
  const double dt = t1 - t0;
  if ((dt < 0.0 && h0 > 0.0) || (dt > 0.0 && h0 < 0.0)) { S.status = kStepFailed; return; }
  if (d.exact || !S.k1_valid) rhs_at(X, S, t0, B.y, B.k[0]);
  int attempts = 0;
  for (;;) {
    bool final_step = false;
    if ((dt >= 0.0 && h0 > dt) || (dt < 0.0 && h0 < dt)) { h0 = dt; final_step = true; }
    for (int s = 2; s <= 6; ++s) {
      // the RHS forms its own stage input from y and the k's (into zs as well)
      const StageSrc st{B.y, {B.k[0], B.k[1], B.k[2], B.k[3], B.k[4]}, s, h0};
      X.stg = &st;
      rhs_into(X, S, t0 + RK_ah[s - 2] * h0, B.k[s - 1]);
      X.stg = nullptr;
    }
    member_sync(d.C);
    const double rmax = final_combine(X, B, h0);
    if (d.exact) rhs_at(X, S, t0 + h0, B.yn, B.k[6]);
    const double tn = final_step ? t1 : t0 + h0;
    // std_control_hadjust (order 5)
    const double h_old = h0;
    int adj = 0;
    double hn = h0;
    if (rmax > 1.1) {
      double r = 0.9 / pow(rmax, 1.0 / 5.0);
      if (r < 0.2) r = 0.2;
      hn = r * h_old;
      adj = -1;
    } else if (rmax < 0.5) {
      double r = 0.9 / pow(rmax, 1.0 / 6.0);
      if (r > 5.0) r = 5.0;
      if (r < 1.0) r = 1.0;
      hn = r * h_old;
      adj = 1;
    }
    if (!(rmax <= 1.7976931348623157e308)) { S.status = kNonFinite; return; }   // NaN/inf state: freeze
    if (adj == -1) {
      const double t_next = tn + hn;
      if (fabs(hn) < fabs(h_old) && t_next != tn) {
        ++S.rej;
        h0 = hn;
        if (++attempts > 200) { S.status = kStepFailed; return; }
        continue;
      }
      hn = h_old;
    }
    // accepted
    if (!d.exact) {
      // pure RHS: derivative at the new point serves as the next dydt_in when the
      // next call starts exactly at t0 + h0
      const double tk = t0 + h0;
      if (tk == tn) {
        rhs_at(X, S, tk, B.yn, B.k[6]);
        double2* tmp = B.k[0]; B.k[0] = B.k[6]; B.k[6] = tmp;
        S.k1_valid = 1;
      } else {
        S.k1_valid = 0;
      }
    } else {
      S.k1_valid = 0;
    }
    double2* ty = B.y; B.y = B.yn; B.yn = ty;
    S.t = tn;
    S.h = hn;
    ++S.acc;
    return;
  }
}

}  // namespace hwdev
