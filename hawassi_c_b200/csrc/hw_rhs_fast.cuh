// hw_rhs_fast.cuh -- HS2 on a flat bottom (rhs_HsF2 with ifft_fft_Hsf2,
// 1d/rhs.c:96-241, 1d/functions.c:1458-1526), the hot path of the plain and the
// batched runs, with the fields kept in two shared-memory slices:
//   * stage input -> Hermitian packing through shared memory / DSMEM partners;
//   * eta, u and M0 u, Hilbert(eta) from one dual inverse transform;
//   * the five real products from one dual forward transform;
//   * the nonlinear adjustment: one inverse transform, ChiAdj, and a dual forward
//     transform that also carries the damping of u.
// Global memory sees the stage input, the per-point tables and five spectral
// results per point (d^ eta, d^ u, adjusted nonlinear terms, damping), instead
// of a round trip per transform.
#pragma once

#include "hw_rhs.cuh"

namespace hwdev {

// Hilbert-transform multiplier of the breaking criterion (1d/breaking.c:133-143)
__device__ __forceinline__ double2 hilbert_hat(double k, double2 e) {
  if (k == 0) return make_double2(0.0, 0.0);
  const double s = k / fabs(k);
  return make_double2(s * e.y, -s * e.x);
}

template <int M>
__device__ __noinline__ void rhs_hs2_flat(Ctx<M>& X, double t, double2* __restrict__ dz) {
  const DevMember& d = X.d;
  const int N = d.N, C = d.C;
  double2* A = X.buf;
  double2* Bf = X.buf2;
  const double2* ZE = d.zs;
  const double2* ZU = d.zs + N;
  double2* PE = d.sc[0];   // physical (eta, u)          [breaking only]
  double2* PM = d.sc[1];   // physical (., Hilbert eta)  [breaking only]
  double2* AE = d.sc[2];   // adjusted nonlinear eta term
  double2* AU = d.sc[3];   // adjusted nonlinear u term
  double2* DE = d.sc[4];   // FFT(damping eta)
  double2* DU = d.sc[5];   // FFT(damping u)
  double2* RB = d.sc[11];  // FFT(breaking force)
  const bool brk = d.brk != 0;
  const double2* Ap = A;
  const double2* Bp = Bf;
  if (C > 1) {
    cg::cluster_group cl = cg::this_cluster();
    const int cp = (C - X.c) & (C - 1);
    Ap = cl.map_shared_rank(A, cp);
    Bp = cl.map_shared_rank(Bf, cp);
  }
  auto jpart = [&](int idx) { return X.c == 0 ? ((M - idx) & (M - 1)) : (M - 1 - idx); };
  double2 va[kPts], vb[kPts];

  // (0) stage input into the two slices (spectral, cyclic), formed here from y and
  // the k's during an RK step (and kept in zs for the assembly)
  if (X.stg) {
    double2* zw = d.zs;
    HW_FOREACH(X) {
      (void)idx;
      const double2 ze = stage_val(*X.stg, p), zu = stage_val(*X.stg, N + p);
      zw[p] = ze;
      zw[N + p] = zu;
      A[pidx(idx)] = ze;
      Bf[pidx(idx)] = zu;
    }
  } else {
    HW_FOREACH(X) {
      A[pidx(idx)] = ZE[p];
      Bf[pidx(idx)] = ZU[p];
    }
  }
  member_sync(C);
  // (1) Hermitian packing: A <- eta^ + i u^, B <- M0 u^ + i H(eta)^ (real parts only, as the reference)
  HW_FOREACH(X) {
    const int jp = jpart(idx), pp = partner_pos(X, idx);
    const double2 e = A[pidx(idx)], ep = Ap[pidx(jp)], w = Bf[pidx(idx)], wp = Bp[pidx(jp)];
    va[u] = pack(herm(e, ep), herm(w, wp), d.invN);
    const double2 m0 = mul_ik(d.M0im[p], w), m0p = mul_ik(d.M0im[pp], wp);
    const double2 s2 = brk ? herm(hilbert_hat(d.k[p], e), hilbert_hat(d.k[pp], ep)) : make_double2(0.0, 0.0);
    vb[u] = pack(herm(m0, m0p), s2, d.invN);
  }
  member_sync(C);
  HW_FOREACH(X) {
    (void)p;
    A[pidx(idx)] = va[u];
    Bf[pidx(idx)] = vb[u];
  }
  fft_inverse2<M>(A, Bf, d.tw, N, C, X.c);
  // (2) products in physical space (1d/functions.c:1486-1498)
  double du[kPts];
  HW_FOREACH(X) {
    const double2 e = A[pidx(idx)], m = Bf[pidx(idx)];
    if (brk) {
      PE[p] = e;
      PM[p].y = m.y;
    }
    du[u] = (d.dcoef[p] * e.y) * d.dchar[p];
    A[pidx(idx)] = make_double2(e.x * e.y, e.x * m.x);
    Bf[pidx(idx)] = make_double2(e.y * e.y - m.x * m.x, (d.dcoef[p] * e.x) * d.dchar[p]);
  }
  fft_forward2<M>(A, Bf, d.tw, N, C, X.c);
  // (3) spectra of the products; H2 terms (1d/rhs.c:141-147)
  member_sync(C);
  HW_FOREACH(X) {
    const int jp = jpart(idx);
    const double2 z1 = A[pidx(idx)], z1p = Ap[pidx(jp)], z2 = Bf[pidx(idx)], z2p = Bp[pidx(jp)];
    const double2 ah = split_re(z1, z1p), bh = split_im(z1, z1p), ch = split_re(z2, z2p);
    DE[p] = split_im(z2, z2p);
    const double kp = d.k[p];
    const double2 lem = cscale(bh, d.L[p]), ik = mul_ik(kp, ah), ikc = mul_ik(kp, ch);
    va[u] = make_double2(-lem.x - ik.x, -lem.y - ik.y);
    vb[u] = make_double2(-ikc.x / 2, -ikc.y / 2);
  }
  member_sync(C);
  HW_FOREACH(X) {
    (void)p;
    A[pidx(idx)] = va[u];
    Bf[pidx(idx)] = vb[u];
  }
  member_sync(C);
  // (4) nonlinear adjustment (1d/rhs.c:695-715): ChiAdj applied in physical space
  HW_FOREACH(X) {
    (void)p;
    const int jp = jpart(idx);
    va[u] = pack(herm(A[pidx(idx)], Ap[pidx(jp)]), herm(Bf[pidx(idx)], Bp[pidx(jp)]), d.invN);
  }
  member_sync(C);
  HW_FOREACH(X) {
    (void)p;
    A[pidx(idx)] = va[u];
  }
  fft_inverse<M>(A, d.tw, N, C, X.c);
  HW_FOREACH(X) {
    const double2 v = A[pidx(idx)];
    const double ch = d.chi[p];
    A[pidx(idx)] = make_double2(v.x * ch, v.y * ch);
    Bf[pidx(idx)] = make_double2(du[u], 0.0);
  }
  fft_forward2<M>(A, Bf, d.tw, N, C, X.c);
  member_sync(C);
  HW_FOREACH(X) {
    const int jp = jpart(idx);
    const double2 z = A[pidx(idx)], zp = Ap[pidx(jp)], zb = Bf[pidx(idx)], zbp = Bp[pidx(jp)];
    AE[p] = split_re(z, zp);
    AU[p] = split_im(z, zp);
    DU[p] = split_re(zb, zbp);
  }
  member_sync(C);
  // (5) kinematic breaking: eddy-viscosity force on the u-equation
  const bool rb_live = brk && breaking_rhs<M>(X, t, PE, &PM[0].y, 2, AE, RB);
  // (6) assembly (1d/rhs.c:217-228) with the source term (1d/rhs.c:659)
  double pv = 0.0, ps = 0.0;
  if (d.has_influx) {
    pv = spline_eval(d.tt, d.ins, d.insc, d.n_in, t);
    ps = spline_eval(d.tt, d.skw, d.skwc, d.n_in, t);
  }
  HW_FOREACH(X) {
    (void)idx;
    const double2 ze = ZE[p], zu = ZU[p];
    const double c1 = d.c1[p], gk = d.gk[p];
    double2 te = make_double2(c1 * zu.y, -c1 * zu.x);
    double2 tu = make_double2(gk * ze.y, -gk * ze.x);
    double fr = 0.0, fi = 0.0;
    if (d.has_influx) {
      const double2 gx = d.gamX[p], gs = d.gamXs[p];
      if (d.prop_mode == 0) { fr = 0.5 * (pv * gx.x - ps * gs.x); fi = 0.5 * (pv * gx.y - ps * gs.y); }
      else if (d.prop_mode == 1) { fr = 0.5 * (pv * gx.x + ps * gs.x); fi = 0.5 * (pv * gx.y + ps * gs.y); }
      else if (d.prop_mode == 2) { fr = pv * gx.x; fi = pv * gx.y; }
    }
    const double al = d.aal[p];
    const double2 de = DE[p], dd = DU[p];
    te = cadd(te, AE[p]);
    tu = cadd(tu, AU[p]);
    if (rb_live) tu = cadd(tu, RB[p]);
    dz[p] = make_double2((te.x + 2 * fr - de.x) * al, (te.y + 2 * fi - de.y) * al);
    dz[N + p] = make_double2((tu.x - dd.x) * al, (tu.y - dd.y) * al);
  }
}

}  // namespace hwdev
