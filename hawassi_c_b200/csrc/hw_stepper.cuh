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

// Fehlberg coefficients (GSL rkf45)
__device__ constexpr double RK_ah[5] = {1.0 / 4.0, 3.0 / 8.0, 12.0 / 13.0, 1.0, 1.0 / 2.0};
__device__ constexpr double RK_b3[2] = {3.0 / 32.0, 9.0 / 32.0};
__device__ constexpr double RK_b4[3] = {1932.0 / 2197.0, -7200.0 / 2197.0, 7296.0 / 2197.0};
__device__ constexpr double RK_b5[4] = {8341.0 / 4104.0, -32832.0 / 4104.0, 29440.0 / 4104.0, -845.0 / 4104.0};
__device__ constexpr double RK_b6[5] = {-6080.0 / 20520.0, 41040.0 / 20520.0, -28352.0 / 20520.0, 9295.0 / 20520.0,
                                        -5643.0 / 20520.0};
__device__ constexpr double RK_c1 = 902880.0 / 7618050.0;
__device__ constexpr double RK_c3 = 3953664.0 / 7618050.0;
__device__ constexpr double RK_c4 = 3855735.0 / 7618050.0;
__device__ constexpr double RK_c5 = -1371249.0 / 7618050.0;
__device__ constexpr double RK_c6 = 277020.0 / 7618050.0;
__device__ constexpr double RK_ec1 = 1.0 / 360.0;
__device__ constexpr double RK_ec3 = -128.0 / 4275.0;
__device__ constexpr double RK_ec4 = -2197.0 / 75240.0;
__device__ constexpr double RK_ec5 = 1.0 / 50.0;
__device__ constexpr double RK_ec6 = 2.0 / 55.0;

// stage input zs = y + h sum_j b_sj k_j for stage s = 2..6 (GSL's expression forms)
template <int M>
__device__ __forceinline__ void stage_input(Ctx<M>& X, const Bufs& B, int s, double h) {
  const DevMember& d = X.d;
  double2* zs = d.zs;
  for (int part = 0; part < 2; ++part) {
    const int off = part * d.N;
    HW_FOREACH(X) {
      (void)idx;
      const int q = p + off;
      const double2 y = B.y[q], a = B.k[0][q];
      double2 r;
      if (s == 2) {
        r = make_double2(y.x + RK_ah[0] * h * a.x, y.y + RK_ah[0] * h * a.y);
      } else {
        const double2 b = B.k[1][q];
        if (s == 3) {
          r = make_double2(y.x + h * (RK_b3[0] * a.x + RK_b3[1] * b.x), y.y + h * (RK_b3[0] * a.y + RK_b3[1] * b.y));
        } else {
          const double2 c3 = B.k[2][q];
          if (s == 4) {
            r = make_double2(y.x + h * (RK_b4[0] * a.x + RK_b4[1] * b.x + RK_b4[2] * c3.x),
                             y.y + h * (RK_b4[0] * a.y + RK_b4[1] * b.y + RK_b4[2] * c3.y));
          } else {
            const double2 c4 = B.k[3][q];
            if (s == 5) {
              r = make_double2(y.x + h * (RK_b5[0] * a.x + RK_b5[1] * b.x + RK_b5[2] * c3.x + RK_b5[3] * c4.x),
                               y.y + h * (RK_b5[0] * a.y + RK_b5[1] * b.y + RK_b5[2] * c3.y + RK_b5[3] * c4.y));
            } else {
              const double2 c5 = B.k[4][q];
              r = make_double2(
                  y.x + h * (RK_b6[0] * a.x + RK_b6[1] * b.x + RK_b6[2] * c3.x + RK_b6[3] * c4.x + RK_b6[4] * c5.x),
                  y.y + h * (RK_b6[0] * a.y + RK_b6[1] * b.y + RK_b6[2] * c3.y + RK_b6[3] * c4.y + RK_b6[4] * c5.y));
            }
          }
        }
      }
      zs[q] = r;
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
      const double dix = RK_c1 * a.x + RK_c3 * c.x + RK_c4 * e.x + RK_c5 * f.x + RK_c6 * g.x;
      const double diy = RK_c1 * a.y + RK_c3 * c.y + RK_c4 * e.y + RK_c5 * f.y + RK_c6 * g.y;
      const double2 yn = make_double2(y.x + h * dix, y.y + h * diy);
      B.yn[q] = yn;
      const double ex = h * (RK_ec1 * a.x + RK_ec3 * c.x + RK_ec4 * e.x + RK_ec5 * f.x + RK_ec6 * g.x);
      const double ey = h * (RK_ec1 * a.y + RK_ec3 * c.y + RK_ec4 * e.y + RK_ec5 * f.y + RK_ec6 * g.y);
      const double rx = fabs(ex) / fabs(d.eps_rel * fabs(yn.x) + d.eps_abs);
      const double ry = fabs(ey) / fabs(d.eps_rel * fabs(yn.y) + d.eps_abs);
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
  rhs_eval<M>(X, t, out);
  ++S.rhs;
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
  if (d.exact || !S.k1_valid) {
    load_stage(X, B.y);
    rhs_into(X, S, t0, B.k[0]);
  }
  int attempts = 0;
  for (;;) {
    bool final_step = false;
    if ((dt >= 0.0 && h0 > dt) || (dt < 0.0 && h0 < dt)) { h0 = dt; final_step = true; }
    for (int s = 2; s <= 6; ++s) {
      stage_input(X, B, s, h0);
      rhs_into(X, S, t0 + RK_ah[s - 2] * h0, B.k[s - 1]);
    }
    member_sync(d.C);
    const double rmax = final_combine(X, B, h0);
    if (d.exact) {
      load_stage(X, B.yn);
      rhs_into(X, S, t0 + h0, B.k[6]);
    }
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
        load_stage(X, B.yn);
        rhs_into(X, S, tk, B.k[6]);
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
