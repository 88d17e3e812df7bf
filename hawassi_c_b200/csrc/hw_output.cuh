// hw_output.cuh -- the output stage of ode_solver_Ham (1d/functions.c:557-760) on
// the device: at every output sample the physical elevation and its time derivative
// (real parts of the inverse transforms of eta^ and of the last RHS's d eta^/dt,
// the reference's global dy), their GSL natural cubic splines evaluated at the gauge
// positions (print_data_gauge), and, when the member keeps fields, eta, u and
// phi = Re F^-1(-i u^ / k) for the Hawassi_{eta,u,phi}_NN.dat files.
//
// The spline's second-derivative coefficients solve a tridiagonal system over the
// whole grid; on a grid of near-uniform spacing the inverse of that matrix decays
// like (2 - sqrt 3)^|i - j| = 0.268^|i - j|, so the coefficients around a gauge
// follow from the data within kWin points of it to below double rounding
// (0.268^48 < 1e-27).  Each gauge thread eliminates that window from both sides
// (natural end conditions wherever it reaches the true ends of the grid) down to
// the two coefficients of the gauge's interval.
#pragma once

#include "hw_stepper.cuh"

namespace hwdev {

constexpr int kWin = 48;

// value m of the physical field held in the cluster's slices (block layout)
template <int M>
__device__ __forceinline__ double2 phys_at(double2* buf, int C, int m) {
  if (C == 1) return buf[pidx(m)];
  cg::cluster_group cl = cg::this_cluster();
  return cl.map_shared_rank(buf, m / M)[pidx(m % M)];
}

template <int M>
__device__ __noinline__ void output_stage(Ctx<M>& X, Bufs& B, StepState& S, int row) {
  const DevMember& d = X.d;
  const int N = d.N, C = d.C;
  // the derivative the reference's dy holds at this sample: the RHS it evaluated
  // last (the accepted step's dydt_out), zero before any RHS call
  const bool none = (d.rhs_calls + S.rhs) == 0;
  const double2* dy = B.k[6];
  if (!d.exact && !none) {
    if (!S.k1_valid) {
      rhs_at(X, S, S.t, B.y, B.k[0]);
      S.k1_valid = 1;
    }
    dy = B.k[0];
  }
  double2* A = X.buf;
  double2* Bf = X.buf2;
  HW_FOREACH(X) {
    A[pidx(idx)] = B.y[p];
    Bf[pidx(idx)] = none ? make_double2(0.0, 0.0) : dy[p];
  }
  member_sync(C);
  const double2* Ap = A;
  const double2* Bp = Bf;
  if (C > 1) {
    cg::cluster_group cl = cg::this_cluster();
    const int cp = (C - X.c) & (C - 1);
    Ap = cl.map_shared_rank(A, cp);
    Bp = cl.map_shared_rank(Bf, cp);
  }
  double2 va[kPts];
  HW_FOREACH(X) {
    (void)p;
    const int jp = X.c == 0 ? ((M - idx) & (M - 1)) : (M - 1 - idx);
    va[u] = pack(herm(A[pidx(idx)], Ap[pidx(jp)]), herm(Bf[pidx(idx)], Bp[pidx(jp)]), d.invN);
  }
  member_sync(C);
  HW_FOREACH(X) {
    (void)p;
    A[pidx(idx)] = va[u];
  }
  fft_inverse<M>(A, d.tw, N, C, X.c);
  member_sync(C);
  // A: (eta, d eta / dt) at grid points c*M + i
  double* fr = d.fields ? d.fields + (size_t)row * 3 * N : nullptr;
  if (fr) {
    HW_FOREACH(X) {
      (void)idx;
      fr[X.c * M + idx] = A[pidx(idx)].x;
    }
  }
  if (X.c == 0 && d.ngauge > 0) {
    for (int g = X.tid; g < d.ngauge; g += Ctx<M>::T) {
      const int i = d.gidx[g];
      double ve = __longlong_as_double(0x7ff8000000000000ULL), vd = ve;
      if (i >= 0) {
        // rows m = a+1 .. b-1 of h0 c_{m-1} + 2 (h0 + h1) c_m + h1 c_{m+1} = R_m with
        // c_a = c_b = 0; a forward sweep up to row i and a backward sweep down to row
        // i+1 leave the 2 x 2 system for c_i, c_{i+1} (both right-hand sides share it)
        const int a = i - kWin < 0 ? 0 : i - kWin;
        const int b = i + 1 + kWin > N - 1 ? N - 1 : i + 1 + kWin;
        auto row_terms = [&](int m, double& h0, double& h1, double& re, double& rd) {
          h0 = d.xg[m] - d.xg[m - 1];
          h1 = d.xg[m + 1] - d.xg[m];
          const double2 y0 = phys_at<M>(A, C, m - 1), y1 = phys_at<M>(A, C, m), y2 = phys_at<M>(A, C, m + 1);
          const double g0 = h0 != 0.0 ? 1.0 / h0 : 0.0, g1 = h1 != 0.0 ? 1.0 / h1 : 0.0;
          re = 3.0 * ((y2.x - y1.x) * g1 - (y1.x - y0.x) * g0);
          rd = 3.0 * ((y2.y - y1.y) * g1 - (y1.y - y0.y) * g0);
        };
        double al = 0.0, ze = 0.0, zd = 0.0, h1i = 0.0;   // forward: al c_i + h1i c_{i+1} = z
        for (int m = a + 1; m <= i; ++m) {
          double h0, h1, re, rd;
          row_terms(m, h0, h1, re, rd);
          if (m == a + 1) { al = 2.0 * (h0 + h1); ze = re; zd = rd; }
          else {
            const double f = h0 / al;
            al = 2.0 * (h0 + h1) - f * h1i;
            ze = re - f * ze;
            zd = rd - f * zd;
          }
          h1i = h1;
        }
        double be = 0.0, we = 0.0, wd = 0.0, h0n = 0.0;   // backward: be c_{i+1} + h0n c_i = w
        for (int m = b - 1; m >= i + 1; --m) {
          double h0, h1, re, rd;
          row_terms(m, h0, h1, re, rd);
          if (m == b - 1) { be = 2.0 * (h0 + h1); we = re; wd = rd; }
          else {
            const double f = h1 / be;
            be = 2.0 * (h0 + h1) - f * h0n;
            we = re - f * we;
            wd = rd - f * wd;
          }
          h0n = h0;
        }
        double ce_i, ce_i1, cd_i, cd_i1;
        if (i == a) {            // c_i = 0 (left end of the grid)
          ce_i = cd_i = 0.0;
          ce_i1 = we / be;
          cd_i1 = wd / be;
        } else if (i + 1 == b) { // c_{i+1} = 0 (right end of the grid)
          ce_i1 = cd_i1 = 0.0;
          ce_i = ze / al;
          cd_i = zd / al;
        } else {
          const double det = al * be - h1i * h0n;
          ce_i = (ze * be - h1i * we) / det;
          ce_i1 = (al * we - h0n * ze) / det;
          cd_i = (zd * be - h1i * wd) / det;
          cd_i1 = (al * wd - h0n * zd) / det;
        }
        const double xl = d.xg[i], h = d.xg[i + 1] - xl, dx = d.gpos[g] - xl;
        const double2 yl = phys_at<M>(A, C, i), yh = phys_at<M>(A, C, i + 1);
        {
          const double dyv = yh.x - yl.x;
          const double bi = dyv / h - h * (ce_i1 + 2.0 * ce_i) / 3.0, di = (ce_i1 - ce_i) / (3.0 * h);
          ve = yl.x + dx * (bi + dx * (ce_i + dx * di));
        }
        {
          const double dyv = yh.y - yl.y;
          const double bi = dyv / h - h * (cd_i1 + 2.0 * cd_i) / 3.0, di = (cd_i1 - cd_i) / (3.0 * h);
          vd = yl.y + dx * (bi + dx * (cd_i + dx * di));
        }
      }
      d.gout[(size_t)row * 2 * d.ngauge + g] = ve;
      d.gout[(size_t)row * 2 * d.ngauge + d.ngauge + g] = vd;
    }
    if (X.tid == 0) d.gtim[row] = S.t;
  }
  if (X.c == 0 && X.tid == 0 && d.ngauge == 0) d.gtim[row] = S.t;
  member_sync(C);
  if (!fr) return;
  // u and phi = Re F^-1(-i u^ / k) (1d/functions.c:571-590: the k == 0 mode is zero)
  HW_FOREACH(X) {
    A[pidx(idx)] = B.y[N + p];
  }
  member_sync(C);
  HW_FOREACH(X) {
    const int jp = X.c == 0 ? ((M - idx) & (M - 1)) : (M - 1 - idx);
    const int pp = partner_pos(X, idx);
    const double2 uh = A[pidx(idx)], up = Ap[pidx(jp)];
    const double kq = d.k[p], kpp = d.k[pp];
    const double2 ph = kq == 0 ? make_double2(0.0, 0.0) : mul_ik(-1 / kq, uh);
    const double2 php = kpp == 0 ? make_double2(0.0, 0.0) : mul_ik(-1 / kpp, up);
    va[u] = pack(herm(uh, up), herm(ph, php), d.invN);
  }
  member_sync(C);
  HW_FOREACH(X) {
    (void)p;
    A[pidx(idx)] = va[u];
  }
  fft_inverse<M>(A, d.tw, N, C, X.c);
  member_sync(C);
  HW_FOREACH(X) {
    (void)p;
    const double2 v = A[pidx(idx)];
    fr[N + X.c * M + idx] = v.x;
    fr[2 * N + X.c * M + idx] = v.y;
  }
  member_sync(C);
}

}  // namespace hwdev
