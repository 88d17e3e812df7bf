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

// the influx source term of the assembly (1d/rhs.c:659-693): force = (fr, fi)
__device__ __forceinline__ void source_term(const DevMember& d, int p, double pv, double ps, double& fr, double& fi) {
  fr = 0.0;
  fi = 0.0;
  if (d.has_influx) {
    const double2 gx = d.gamX[p], gs = d.gamXs[p];
    if (d.prop_mode == 0) { fr = 0.5 * (pv * gx.x - ps * gs.x); fi = 0.5 * (pv * gx.y - ps * gs.y); }
    else if (d.prop_mode == 1) { fr = 0.5 * (pv * gx.x + ps * gs.x); fi = 0.5 * (pv * gx.y + ps * gs.y); }
    else if (d.prop_mode == 2) { fr = pv * gx.x; fi = pv * gx.y; }
  }
}

// assembly of dz at spectral position p (1d/rhs.c:217-228): delta H1 + adjusted
// nonlinear terms (ae, au) + breaking force (rb) + 2 force - damping (de, du), times aal
__device__ __forceinline__ void assemble_flat(const DevMember& d, int p, double2 ae, double2 au, double2 rb, double2 de,
                                              double2 du, double pv, double ps, double2* __restrict__ dz) {
  const int N = d.N;
  const double2 ze = d.zs[p], zu = d.zs[N + p];
  const double c1 = d.c1[p], gk = d.gk[p];
  double2 te = make_double2(c1 * zu.y, -c1 * zu.x);
  double2 tu = make_double2(gk * ze.y, -gk * ze.x);
  double fr, fi;
  source_term(d, p, pv, ps, fr, fi);
  const double al = d.aal[p];
  te = cadd(te, ae);
  tu = cadd(cadd(tu, au), rb);
  dz[p] = make_double2((te.x + 2 * fr - de.x) * al, (te.y + 2 * fi - de.y) * al);
  dz[N + p] = make_double2((tu.x - du.x) * al, (tu.y - du.y) * al);
}

// Cluster members: the inverse transform's cross-CTA step, the pointwise work in
// physical space and the next forward transform's cross-CTA step meet at the same
// index set -- position i of every CTA's slice, i.e. the physical points r M + i
// (r = 0..C-1) -- so the thread owning position i (the ownership of cross_gs) does
// all three in registers: gather, twiddle, inverse C-point DFT, pointwise step,
// forward C-point DFT, twiddle, scatter.  Two cluster barriers replace four and the
// physical fields never pass through shared memory.
//
// First meeting (1d/functions.c:1486-1498): A = eta + i u, B = M0 u + i H(eta) in;
// out A = (eta u) + i (eta M0 u), B = (u^2 - (M0 u)^2) + i (damping of eta); the
// damping of u waits in the member's scratch (damp_u_field) for the second meeting;
// eta, u and H(eta) go to global memory for the breaking criterion.
// the physical damping of u between the products and the adjustment, one double per
// grid point in the member's scratch field 5 (used for the spectral damping of u only
// after that); kept out of shared memory, which leaves the SM more L1 cache
__device__ __forceinline__ double* damp_u_field(const DevMember& d) { return reinterpret_cast<double*>(d.sc[5]); }

template <int M, int C>
__device__ __forceinline__ void cross_products(Ctx<M>& X, double2* A, double2* B, bool brk, double2* PE, double2* PM) {
  constexpr int T = M / kPts;
  constexpr int PER = kPts / C;
  const DevMember& d = X.d;
  double* du = damp_u_field(d);
  cg::cluster_group cl = cg::this_cluster();
  cl.sync();
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int i = X.c * T + X.tid + q * (C * T);
    double2 va[C], vb[C], w[C > 1 ? C : 2];
#pragma unroll
    for (int r = 0; r < C; ++r) {
      va[r] = cl.map_shared_rank(A, r)[pidx(i)];
      vb[r] = cl.map_shared_rank(B, r)[pidx(i)];
    }
    twiddle_powers<C>(twd(d.tw, i, +1), w);
#pragma unroll
    for (int r = 1; r < C; ++r) {
      va[r] = cmul(va[r], w[r]);
      vb[r] = cmul(vb[r], w[r]);
    }
    dft_small<C>(va, +1);
    dft_small<C>(vb, +1);
#pragma unroll
    for (int r = 0; r < C; ++r) {
      const int n = r * M + i;
      const double2 e = va[r], m = vb[r];
      if (brk) {
        PE[n] = e;
        PM[n].y = m.y;
      }
      const double dc = d.dcoef[n], ch = d.dchar[n];
      du[n] = (dc * e.y) * ch;
      va[r] = make_double2(e.x * e.y, e.x * m.x);
      vb[r] = make_double2(e.y * e.y - m.x * m.x, (dc * e.x) * ch);
    }
    dft_small<C>(va, -1);
    dft_small<C>(vb, -1);
    twiddle_powers<C>(twd(d.tw, i, -1), w);
#pragma unroll
    for (int r = 1; r < C; ++r) {
      va[r] = cmul(va[r], w[r]);
      vb[r] = cmul(vb[r], w[r]);
    }
#pragma unroll
    for (int r = 0; r < C; ++r) {
      cl.map_shared_rank(A, r)[pidx(i)] = va[r];
      cl.map_shared_rank(B, r)[pidx(i)] = vb[r];
    }
  }
  cl.sync();
}

// Second meeting (1d/rhs.c:695-715): the nonlinear terms' inverse transform times
// ChiAdj, paired with the damping of u kept by the first meeting, into the forward
// dual transform: A in (one transform), out A = ChiAdj-adjusted terms, B = damping of u.
template <int M, int C>
__device__ __forceinline__ void cross_adjust(Ctx<M>& X, double2* A, double2* B) {
  constexpr int T = M / kPts;
  constexpr int PER = kPts / C;
  const DevMember& d = X.d;
  const double* du = damp_u_field(d);
  cg::cluster_group cl = cg::this_cluster();
  cl.sync();
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int i = X.c * T + X.tid + q * (C * T);
    double2 va[C], vb[C], w[C > 1 ? C : 2];
#pragma unroll
    for (int r = 0; r < C; ++r) va[r] = cl.map_shared_rank(A, r)[pidx(i)];
    twiddle_powers<C>(twd(d.tw, i, +1), w);
#pragma unroll
    for (int r = 1; r < C; ++r) va[r] = cmul(va[r], w[r]);
    dft_small<C>(va, +1);
#pragma unroll
    for (int r = 0; r < C; ++r) {
      const double ch = d.chi[r * M + i];
      va[r] = make_double2(va[r].x * ch, va[r].y * ch);
      vb[r] = make_double2(du[r * M + i], 0.0);
    }
    dft_small<C>(va, -1);
    dft_small<C>(vb, -1);
    twiddle_powers<C>(twd(d.tw, i, -1), w);
#pragma unroll
    for (int r = 1; r < C; ++r) {
      va[r] = cmul(va[r], w[r]);
      vb[r] = cmul(vb[r], w[r]);
    }
#pragma unroll
    for (int r = 0; r < C; ++r) {
      cl.map_shared_rank(A, r)[pidx(i)] = va[r];
      cl.map_shared_rank(B, r)[pidx(i)] = vb[r];
    }
  }
  cl.sync();
}

template <int M>
__device__ __forceinline__ void cross_products_any(Ctx<M>& X, double2* A, double2* B, bool brk, double2* PE, double2* PM) {
  if (X.d.C == 2) cross_products<M, 2>(X, A, B, brk, PE, PM);
  else if (X.d.C == 4) cross_products<M, 4>(X, A, B, brk, PE, PM);
  else cross_products<M, 8>(X, A, B, brk, PE, PM);
}
template <int M>
__device__ __forceinline__ void cross_adjust_any(Ctx<M>& X, double2* A, double2* B) {
  if (X.d.C == 2) cross_adjust<M, 2>(X, A, B);
  else if (X.d.C == 4) cross_adjust<M, 4>(X, A, B);
  else cross_adjust<M, 8>(X, A, B);
}

template <int M>
__device__ __noinline__ void rhs_hs2_flat(Ctx<M>& X, double t, double2* __restrict__ dz) {
  const DevMember& d = X.d;
  const int N = d.N, C = d.C;
  double2* A = X.buf;
  double2* Bf = X.buf2;
  const double2* ZE = d.zs;
  const double2* ZU = d.zs + N;
  double2* PE = d.sc[0];   // physical (eta, u)           [breaking only]
  double2* PM = d.sc[1];   // physical (., Hilbert eta)   [breaking only]
  double2* AE = d.sc[2];   // adjusted nonlinear eta term [breaking force live only]
  double2* AU = d.sc[3];   // adjusted nonlinear u term   [breaking force live only]
  double2* DE = d.sc[4];   // FFT(damping eta)
  double2* DU = d.sc[5];   // FFT(damping u)              [breaking force live only]
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

  // (0)-(1) stage input (spectral, cyclic) and its Hermitian packing for the first
  // dual inverse transform: A <- eta^ + i u^, B <- M0 u^ + i H(eta)^ (real parts
  // only, as the reference).  Every exit of this function leaves the slices unread
  // by the other CTAs (a barrier follows the last partner reads), so they can be
  // written at once.
  if (brk) breaking_reset(X);
  auto packed = [&](int p, int pp, double2 e, double2 ep, double2 w, double2 wp, double2& a, double2& b) {
    a = pack(herm(e, ep), herm(w, wp), d.invN);
    const double2 m0 = mul_ik(d.M0im[p], w), m0p = mul_ik(d.M0im[pp], wp);
    const double2 s2 = brk ? herm(hilbert_hat(d.k[p], e), hilbert_hat(d.k[pp], ep)) : make_double2(0.0, 0.0);
    b = pack(herm(m0, m0p), s2, d.invN);
  };
  if (X.stg) {
    // during a step the stage input is formed here from y and the k's (and kept in
    // zs for the assembly).  Each Hermitian pair {k, N - k} is formed once, by one
    // thread: CTA c takes the first half of its slice, i < M / 2, with the partners
    // (CTA (C - c) mod C, index M - 1 - i, or (M - i) mod M in CTA 0), which lie in the
    // partner CTA's second half; CTA 0's positions 0 and M / 2 are their own partners.
    // The thread writes both packed values, the partner's into the partner CTA's slices
    // (its shared memory through the cluster when that is another CTA).
    double2* zw = d.zs;
    constexpr int T = Ctx<M>::T;
    const int c = X.c, cq = (C - c) & (C - 1);
    double2* Aq = A;
    double2* Bq = Bf;
    if (cq != c) {
      cg::cluster_group cl = cg::this_cluster();
      Aq = cl.map_shared_rank(A, cq);
      Bq = cl.map_shared_rank(Bf, cq);
    }
    const StageSrc& st = *X.stg;
    auto pair = [&](int i, int j) {
      const int p = c * M + i, pp = cq * M + j;
      const double2 e = stage_val(st, p), w = stage_val(st, N + p);
      if (p == pp) {
        zw[p] = e;
        zw[N + p] = w;
        double2 a, b;
        packed(p, p, e, e, w, w, a, b);
        A[pidx(i)] = a;
        Bf[pidx(i)] = b;
        return;
      }
      const double2 ep = stage_val(st, pp), wp = stage_val(st, N + pp);
      zw[p] = e;
      zw[N + p] = w;
      zw[pp] = ep;
      zw[N + pp] = wp;
      double2 a, b;
      packed(p, pp, e, ep, w, wp, a, b);
      A[pidx(i)] = a;
      Bf[pidx(i)] = b;
      packed(pp, p, ep, e, wp, w, a, b);
      Aq[pidx(j)] = a;
      Bq[pidx(j)] = b;
    };
#pragma unroll
    for (int u = 0; u < kPts / 2; ++u) {
      const int i = X.tid + u * T;
      pair(i, c == 0 ? ((M - i) & (M - 1)) : (M - 1 - i));
    }
    if (c == 0 && X.tid == 0) pair(M / 2, M / 2);
    if (C > 1) cg::this_cluster().sync();   // the partners' slices are written
  } else {
    // zs written by the caller: the partner values come through the slices
    HW_FOREACH(X) {
      A[pidx(idx)] = ZE[p];
      Bf[pidx(idx)] = ZU[p];
    }
    member_sync(C);
    HW_FOREACH(X) {
      const int jp = jpart(idx), pp = partner_pos(X, idx);
      packed(p, pp, A[pidx(idx)], Ap[pidx(jp)], Bf[pidx(idx)], Bp[pidx(jp)], va[u], vb[u]);
    }
    member_sync(C);
    HW_FOREACH(X) {
      (void)p;
      A[pidx(idx)] = va[u];
      Bf[pidx(idx)] = vb[u];
    }
  }
  // (2) products in physical space (1d/functions.c:1486-1498); the damping of u
  // waits in the member's scratch for the adjustment's transform
  const bool fused = C == 2 || C == 4 || C == 8;
  double* du = damp_u_field(d);
  if (fused) {
    fft_local2<M>(A, Bf, d.tw, C, +1);
    cross_products_any<M>(X, A, Bf, brk, PE, PM);
    fft_local2<M>(A, Bf, d.tw, C, -1);
  } else {
    fft_inverse2<M>(A, Bf, d.tw, N, C, X.c);
    HW_FOREACH(X) {
      const double2 e = A[pidx(idx)], m = Bf[pidx(idx)];
      if (brk) {
        PE[p] = e;
        PM[p].y = m.y;
      }
      du[p] = (d.dcoef[p] * e.y) * d.dchar[p];
      A[pidx(idx)] = make_double2(e.x * e.y, e.x * m.x);
      Bf[pidx(idx)] = make_double2(e.y * e.y - m.x * m.x, (d.dcoef[p] * e.x) * d.dchar[p]);
    }
    fft_forward2<M>(A, Bf, d.tw, N, C, X.c);
  }
  // breaking criterion (1d/breaking.c:36-95) on eta, u, H(eta): the transform's
  // barriers made PE / PM complete member-wide
  if (brk) breaking_scan(X, PE, &PM[0].y, 2);
  // (3) spectra of the products, H2 terms (1d/rhs.c:141-147) and, in the same
  // pass, the Hermitian packing of the nonlinear adjustment (1d/rhs.c:695-715):
  // each thread forms the terms at its wavenumber k and at N - k from the pair of
  // transformed values it holds, so no exchange separates the two steps
  member_sync(C);
  HW_FOREACH(X) {
    const int jp = jpart(idx), pp = partner_pos(X, idx);
    const double2 z1 = A[pidx(idx)], z1p = Ap[pidx(jp)], z2 = Bf[pidx(idx)], z2p = Bp[pidx(jp)];
    DE[p] = split_im(z2, z2p);
    const double kp = d.k[p], kq = d.k[pp];
    // at k
    const double2 ah = split_re(z1, z1p), bh = split_im(z1, z1p), ch = split_re(z2, z2p);
    const double2 lem = cscale(bh, d.L[p]), ik = mul_ik(kp, ah), ikc = mul_ik(kp, ch);
    const double2 te = make_double2(-lem.x - ik.x, -lem.y - ik.y);
    const double2 tu = make_double2(-ikc.x / 2, -ikc.y / 2);
    // at N - k (the partner's pair is (z1p, z1))
    const double2 ahq = split_re(z1p, z1), bhq = split_im(z1p, z1), chq = split_re(z2p, z2);
    const double2 lemq = cscale(bhq, d.L[pp]), ikq = mul_ik(kq, ahq), ikcq = mul_ik(kq, chq);
    const double2 teq = make_double2(-lemq.x - ikq.x, -lemq.y - ikq.y);
    const double2 tuq = make_double2(-ikcq.x / 2, -ikcq.y / 2);
    va[u] = pack(herm(te, teq), herm(tu, tuq), d.invN);
  }
  if (brk) breaking_lead(X, t, PE, &PM[0].y, 2);
  member_sync(C);
  HW_FOREACH(X) {
    (void)p;
    A[pidx(idx)] = va[u];
  }
  if (fused) {
    fft_local<M>(A, d.tw, C, +1);
    cross_adjust_any<M>(X, A, Bf);
    fft_local2<M>(A, Bf, d.tw, C, -1);
  } else {
    fft_inverse<M>(A, d.tw, N, C, X.c);
    HW_FOREACH(X) {
      const double2 v = A[pidx(idx)];
      const double ch = d.chi[p];
      A[pidx(idx)] = make_double2(v.x * ch, v.y * ch);
      Bf[pidx(idx)] = make_double2(du[p], 0.0);
    }
    fft_forward2<M>(A, Bf, d.tw, N, C, X.c);
  }
  double pv = 0.0, ps = 0.0;
  if (d.has_influx) {
    pv = spline_eval(d.tt, d.ins, d.insc, d.n_in, t);
    ps = spline_eval(d.tt, d.skw, d.skwc, d.n_in, t);
  }
  member_sync(C);
  // the leader's node count is visible member-wide after the transforms' barriers
  const bool rb_live = brk && d.bk->npk > 0;
  if (!rb_live) {
    // (6) assembly (1d/rhs.c:217-228) straight from the adjusted spectra
    HW_FOREACH(X) {
      const int jp = jpart(idx);
      const double2 z = A[pidx(idx)], zp = Ap[pidx(jp)], zb = Bf[pidx(idx)], zbp = Bp[pidx(jp)];
      assemble_flat(d, p, split_re(z, zp), split_im(z, zp), make_double2(0.0, 0.0), DE[p], split_re(zb, zbp), pv, ps,
                    dz);
    }
    member_sync(C);   // the partner reads of the slices are done
    return;
  }
  HW_FOREACH(X) {
    const int jp = jpart(idx);
    const double2 z = A[pidx(idx)], zp = Ap[pidx(jp)], zb = Bf[pidx(idx)], zbp = Bp[pidx(jp)];
    AE[p] = split_re(z, zp);
    AU[p] = split_im(z, zp);
    DU[p] = split_re(zb, zbp);
  }
  member_sync(C);
  // (5) kinematic breaking: eddy-viscosity force on the u-equation
  breaking_force<M>(X, PE, AE, RB);
  // (6) assembly with the force
  member_sync(C);
  HW_FOREACH(X) {
    (void)idx;
    assemble_flat(d, p, AE[p], AU[p], RB[p], DE[p], DU[p], pv, ps, dz);
  }
}

}  // namespace hwdev
