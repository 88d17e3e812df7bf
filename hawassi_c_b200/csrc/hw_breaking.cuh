// hw_breaking.cuh -- kinematic breaking on the device (1d/breaking.c:36-449 and
// rhs_breaking, 1d/rhs.c:617-657), run inside every RHS evaluation exactly as
// the reference does (the state machine sees every call, rejected stages too).
//
//  * criterion (parallel): eta above MaxEtaInit in the breaking window, the
//    local maxima above it (findpeaks) and, at each of them, the local wavenumber
//    from the Hilbert transform and the u > KBC * c test, evaluated by the thread
//    that found the maximum; the passing crests are collected with global atomics;
//  * crest state machine (one leader thread of the member): the passing crests in
//    ascending grid order (findpeaks' order), crest tracking with the
//    CrestBreak / New / Prev records, the U*(t) ramp and B in [0, 1] along each
//    breaking crest, and the breaking.dat record once per output interval;
//  * eddy-viscosity force (parallel): Flux = -B delb^2 (h + eta) (d_t eta)^2,
//    R_b = d_x Flux / (h + eta) with centred differences, then its spectrum.
#pragma once

#include "hw_rhs.cuh"

namespace hwdev {

__device__ __forceinline__ double phase_velocity_dev(double k, double d) {  // 1d/functions.c:1415
  if (k == 0) return sqrt(kG * d);
  const double s = k < 0 ? -1.0 : 1.0;
  return s * sqrt(kG * k * tanh(d * k)) / k;
}

__device__ __forceinline__ void crest_clear(Crest* a, int n) {  // set_init_CB (BindexNow untouched)
  for (int j = 0; j < n; ++j) {
    a[j].Bindex = 0;
    a[j].Ucrest = 0;
    a[j].DirProp = 0;
    a[j].Bposition = 0;
    a[j].Btime = 0;
    a[j].Bcount = 0;
  }
}

// breaking_criterion's test at a local maximum J (1d/breaking.c:72-95): local
// wavenumber K = (eta dH/dx - H deta/dx) / (eta^2 + H^2) from the Hilbert transform
// H of eta (centred differences, 1d/functions.c:1850), crest speed c(K, h + eta),
// breaking if |u| > KBC |c|.  Products and sums are rounded one by one (no fused
// multiply-add), in the reference's order, as the reference's x86-64 build rounds.
__device__ __forceinline__ bool crest_breaks(const DevMember& d, const double2* PE, const double* Heta, int hs,
                                             int J) {
  const double eJ = PE[J].x, hJ = Heta[size_t(hs) * J];
  const double dx2 = 2 * d.dx;
  const double gH = __ddiv_rn(__dsub_rn(Heta[size_t(hs) * (J + 1)], Heta[size_t(hs) * (J - 1)]), dx2);
  const double ge = __ddiv_rn(__dsub_rn(PE[J + 1].x, PE[J - 1].x), dx2);
  const double KxJ = __ddiv_rn(__dsub_rn(__dmul_rn(eJ, gH), __dmul_rn(hJ, ge)),
                               __dadd_rn(__dmul_rn(eJ, eJ), __dmul_rn(hJ, hJ)));
  const double Cc = phase_velocity_dev(KxJ, __dadd_rn(d.depth[J], eJ));
  return fabs(PE[J].y) > __dmul_rn(d.KBC, fabs(Cc));
}

// the sequential part of breaking_process, run by one thread
static __device__ __noinline__ void breaking_leader(const DevMember& d, BrkDev* bk, double t, const double2* PE, const double* Heta,
                                int hs) {
  const int N = d.N, cap = bk->cap;
  double* B = bk->B;
  // B <- 0 (only the nodes set by the previous call can be nonzero)
  if (bk->n_touched > N) {
    for (int i = 0; i < N; ++i) B[i] = 0.0;
  } else {
    for (int i = 0; i < bk->n_touched; ++i) B[bk->touched[i]] = 0.0;
  }
  bk->n_touched = 0;
  Crest* cb = bk->cb;
  Crest* cbn = bk->cbn;
  Crest* cbp = bk->cbp;
  // ---- breaking_criterion (1d/breaking.c:63): the crests that passed the test ----
  const int npk = bk->npk;
  if (bk->any_above && npk > 0) {
    int* pk = bk->pk;
    for (int i = 1; i < npk; ++i) {   // findpeaks yields ascending indices
      const int v = pk[i];
      int j = i - 1;
      while (j >= 0 && pk[j] > v) { pk[j + 1] = pk[j]; --j; }
      pk[j + 1] = v;
    }
    int itCB = 0;
    for (int i = 0; i < npk; ++i) {
      const int J = pk[i];
      const double Up = PE[J].y;
      if (itCB < cap) {
        Crest& r = cb[itCB];
        r.Bindex = J;
        r.BindexNow = J;
        r.Ucrest = fabs(Up);
        r.DirProp = int(Up / fabs(Up));
        r.Bposition = 0.0;
        r.Btime = t;
        ++itCB;
      }
    }
    for (int j = 0; j < itCB; ++j) cb[j].Bcount = itCB;
    if (itCB > bk->dirty_cb) bk->dirty_cb = itCB;
  } else {
    crest_clear(cb, bk->dirty_cb);
    bk->dirty_cb = 0;
  }
  // ---- breaking_process (1d/breaking.c:200-449) ----
  const int NCB = cb[0].Bcount;
  int* ID = bk->id_node_end;
  if (NCB > 0 && bk->flag == 0) {
    bk->flag = 1;
    for (int j = 0; j < NCB; ++j) cbn[j] = cb[j];
    if (NCB > bk->dirty_cbn) bk->dirty_cbn = NCB;
  } else if (NCB == 0 && bk->flag == 2) {
    const int NCBprev = cbp[0].Bcount;
    for (int j = 0; j < NCBprev; ++j) cbn[j] = cbp[j];
    if (NCBprev > bk->dirty_cbn) bk->dirty_cbn = NCBprev;
  } else if (NCB > 0 && bk->flag == 2) {
    const int NCBprev = cbp[0].Bcount;
    for (int j = 0; j < NCBprev; ++j) cbn[j] = cbp[j];
    if (NCBprev > bk->dirty_cbn) bk->dirty_cbn = NCBprev;
    int add = 0;
    for (int kk = 0; kk < NCB; ++kk) {
      bool isnew = true;
      for (int l = 0; l < NCBprev; ++l) {
        const int dleft = abs(ID[l] - cbp[l].BindexNow);
        if (cbp[l].DirProp == 1) {
          if (cb[kk].Bindex >= (cbp[l].BindexNow - 3 * dleft) && cb[kk].Bindex <= ID[l]) { isnew = false; break; }
        } else {
          if (cb[kk].Bindex >= cbp[l].BindexNow && cb[kk].Bindex <= (ID[l] + 3 * dleft)) { isnew = false; break; }
        }
      }
      if (isnew && NCBprev + add < cap) {
        Crest& r = cbn[NCBprev + add];
        r.Bindex = cb[kk].Bindex;
        r.BindexNow = cb[kk].Bindex;
        ID[NCBprev + add] = cb[kk].Bindex;
        r.Ucrest = cb[kk].Ucrest;
        r.Bposition = cb[kk].Bposition;
        r.Btime = cb[kk].Btime;
        r.DirProp = cb[kk].DirProp;
        r.Bcount = cb[kk].Bcount;
        ++add;
        if (NCBprev + add > bk->dirty_cbn) bk->dirty_cbn = NCBprev + add;
      }
    }
    int j = 0;
    while (j < bk->dirty_cbn && cbn[j].Bindex > 0) ++j;
    for (int i = 0; i < j; ++i) cbn[i].Bcount = j;
  }
  if (bk->flag == 1 || bk->flag == 2) {
    const int NCBnow = cbn[0].Bcount;
    int it_indexb = 0, iterNprev = 0;
    bool any_keep = false;
    crest_clear(cbp, bk->dirty_cbp);
    bk->dirty_cbp = 0;
    int prevNow = -1;
    for (int lx = 0; lx < NCBnow; ++lx) {
      int indxMaxNow;
      if (bk->flag == 1) {
        indxMaxNow = cbn[lx].Bindex;
      } else {
        const int st = cbn[lx].BindexNow;
        const int lenloc = abs(ID[lx] - st);
        int best = 0;
        if (lenloc > 0) {
          double tv = PE[st].x;
          for (int q = 0; q < lenloc; ++q) {
            const double v = PE[st + q * cbn[lx].DirProp].x;
            if (v > tv) { tv = v; best = q; }
          }
        }
        indxMaxNow = st + best * cbn[lx].DirProp;
      }
      cbn[lx].BindexNow = indxMaxNow;
      if (lx != 0 && indxMaxNow == prevNow) { prevNow = indxMaxNow; continue; }   // IDTerminate = 0
      prevNow = indxMaxNow;
      const double tbreak = cbn[lx].Btime, U_I = cbn[lx].Ucrest, U_F = d.TC * U_I;
      double U_star;
      if ((t - tbreak) >= d.Tstar) U_star = U_F;
      else if ((t - tbreak) >= 0 && (t - tbreak) < d.Tstar) U_star = U_I + ((t - tbreak) / d.Tstar) * (U_F - U_I);
      else U_star = U_I;
      const int dir = cbn[lx].DirProp;
      const int indEND = dir == 1 ? d.xbend : d.xbstart;
      int Node_end = indxMaxNow;
      bool fh = false;
      for (int ly = indxMaxNow; ly < indEND && dir != 0; ly += dir) {
        const double au = fabs(PE[ly].y);
        if (au < U_F) { Node_end = ly; break; }
        double bv;
        if (au > (2 * U_star)) bv = 1;
        else if (au <= U_star) bv = 0;
        else bv = (au / U_star) - 1;
        B[ly] = bv;
        if (bk->n_touched < N) bk->touched[bk->n_touched] = ly;
        ++bk->n_touched;
        if (au >= U_star) fh = true;
        if (it_indexb < N) bk->nodes[it_indexb] = ly;
        ++it_indexb;
      }
      if (fh) {
        any_keep = true;
        ID[iterNprev] = Node_end;
        cbp[iterNprev] = cbn[lx];
        ++iterNprev;
        if (iterNprev > bk->dirty_cbp) bk->dirty_cbp = iterNprev;
      }
    }
    int j = 0;
    while (j < bk->dirty_cbp && cbp[j].Bindex > 0) ++j;
    for (int i = 0; i < j; ++i) cbp[i].Bcount = j;
    // flag: 2 if any crest keeps breaking, else 0 (the reference loop over IDTerminate)
    if (NCBnow > 0) bk->flag = any_keep ? 2 : 0;
    if (t > (bk->ITERbdt * d.dt_in) && it_indexb > 0) {
      const long long need = 2 + it_indexb;
      if (bk->log_len + need <= bk->log_cap) {
        double* lg = bk->log + bk->log_len;
        lg[0] = t;
        lg[1] = it_indexb;
        for (int q = 0; q < it_indexb && q < N; ++q) lg[2 + q] = bk->nodes[q];
        bk->log_len += need;
      }
      ++bk->ITERbn;
    }
  }
  if (t > (bk->ITERbdt * d.dt_in)) ++bk->ITERbdt;
  crest_clear(cbn, bk->dirty_cbn);
  crest_clear(cb, bk->dirty_cb);
  bk->dirty_cbn = 0;
  bk->dirty_cb = 0;
  // nodes touched by this call (zero: the breaking force is identically zero)
  bk->npk = bk->n_touched;
}

// The parts of one RHS's breaking work, so that a caller can place them between
// its own phases:
//   breaking_reset  (leader) before a barrier that precedes the scan;
//   breaking_scan   (all threads) once eta, u and H(eta) are complete member-wide;
//   breaking_lead   (leader) after a barrier that follows the scan; it leaves the
//                   count of nodes with B != 0 in bk->npk (0: no force);
//   breaking_force  (all threads) after a barrier that follows the leader.
template <int M>
__device__ __forceinline__ void breaking_reset(Ctx<M>& X) {
  if (X.c == 0 && X.tid == 0) {
    X.d.bk->npk = 0;
    X.d.bk->any_above = 0;
  }
}

// criterion scan over this CTA's physical points (1d/breaking.c:36-61,72)
template <int M>
__device__ __forceinline__ void breaking_scan(Ctx<M>& X, const double2* PE, const double* Heta, int hs) {
  const DevMember& d = X.d;
  BrkDev* bk = d.bk;
  const int N = d.N;
  const int w0 = d.xbstart, w1 = d.xbstart + d.lenIF;   // window [w0, w1)
  bool above = false;
  HW_FOREACH(X) {
    (void)idx;
    if (p >= w0 && p < w1) {
      const double e = PE[p].x;
      if (e > d.MaxEtaInit) above = true;
      if (p >= w0 + 1 && p <= w1 - 2 && !(e < d.MaxEtaInit) && e > PE[p + 1].x && e > PE[p - 1].x &&
          crest_breaks(d, PE, Heta, hs, p)) {
        const int slot = atomicAdd(&bk->npk, 1);
        if (slot < N) bk->pk[slot] = p;
      }
    }
  }
  // one flag update per warp
  if (__any_sync(0xffffffffu, above) && (X.tid & 31) == 0) atomicOr(&bk->any_above, 1);
}

template <int M>
__device__ __forceinline__ void breaking_lead(Ctx<M>& X, double t, const double2* PE, const double* Heta, int hs) {
  if (X.c == 0 && X.tid == 0) {
    BrkDev* bk = X.d.bk;
    if (bk->npk > X.d.N) bk->npk = X.d.N;
    breaking_leader(X.d, bk, t, PE, Heta, hs);
    __threadfence();
  }
}

// eddy-viscosity force (rhs_breaking, 1d/rhs.c:617-657): Rb = F(d_x Flux / (h + eta)),
// Flux = -B delb^2 (h + eta) (d_t eta)^2, d_t eta = Re F^-1(dH1_eta + AEadj)
template <int M>
__device__ __noinline__ void breaking_force(Ctx<M>& X, const double2* PE, const double2* AEadj, double2* Rb) {
  const DevMember& d = X.d;
  BrkDev* bk = d.bk;
  const int N = d.N;
  const double2* ZU = d.zs + N;
  const double2* HS = d.sc[6];
  auto teta = [&](int q) -> double2 {
    double2 h1;
    if (d.flat) {
      const double c1 = d.c1[q];
      h1 = make_double2(c1 * ZU[q].y, -c1 * ZU[q].x);
    } else {
      const double kq = d.k[q];
      h1 = make_double2((HS[q].y / kG) * kq, -(HS[q].x / kG) * kq);
    }
    return cadd(h1, AEadj[q]);
  };
  HW_FOREACH(X) {
    const int pp = partner_pos(X, idx);
    X.buf[pidx(idx)] = cscale(herm(teta(p), teta(pp)), d.invN);
  }
  double2* FL = d.sc[8];   // flux (physical), reused scratch
  fft_inverse_then(X, [&](int, int, int p, double2 v) {
    const double dte = v.x;
    const double e = PE[p].x;
    FL[p].x = -bk->B[p] * (kDelb * kDelb) * (d.depth[p] + e) * dte * dte;
  });
  member_sync(d.C);
  // gradient (1d/functions.c:1850) and R_b = d_x Flux / (h + eta)
  HW_FOREACH(X) {
    (void)idx;
    double g;
    if (p == 0) g = (FL[1].x - FL[0].x) / d.dx;
    else if (p == N - 1) g = (FL[N - 1].x - FL[N - 2].x) / d.dx;
    else g = (FL[p + 1].x - FL[p - 1].x) / (2 * d.dx);
    const double rb = 1 / (d.depth[p] + PE[p].x) * g;
    X.buf[pidx(idx)] = make_double2(rb, 0.0);
  }
  fft_forward_split(X, [&](int, int, int p, double2 z, double2 zp) { Rb[p] = split_re(z, zp); });
}

// The whole breaking step of one RHS, after the adjusted nonlinear terms: returns
// false (Rb untouched) when no node breaks: the force is then identically zero, as
// the reference's FFT of a zero flux gives, and the assembly skips it
template <int M>
__device__ __noinline__ bool breaking_rhs(Ctx<M>& X, double t, const double2* PE, const double* Heta, int hs,
                                          const double2* AEadj, double2* Rb) {
  breaking_reset(X);
  member_sync(X.d.C);
  breaking_scan(X, PE, Heta, hs);
  member_sync(X.d.C);
  breaking_lead(X, t, PE, Heta, hs);
  member_sync(X.d.C);
  if (X.d.bk->npk == 0) return false;   // B identically zero: FFT(0) = 0, as the reference computes it
  breaking_force(X, PE, AEadj, Rb);
  return true;
}

}  // namespace hwdev
