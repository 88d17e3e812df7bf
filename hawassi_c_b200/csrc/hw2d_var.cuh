// hw2d_var.cuh -- HAWASSI 2D RHS on a varying bottom with two reference depths
// (rhs_AB2_2DB_uv, 2d/fun_odesolver.c:4542-4626; fun_termshat_AB1_2DB_uv :2874,
// fun_termshat_AB2_2DB_uv :3327; HSSgen_2depth :500).  The two-depth operator
//   HSS(phi; O) = [F(gam_min Re F^-1 S(O_min phi^)) + O_min F(gam_min phi)
//                 + F(gam_plus Re F^-1 S(O_plus phi^)) + O_plus F(gam_plus phi)] / 2
// needs a round trip through physical space per application, so one RHS is nine
// fused passes (the last two, adjust + source and assembly, are the flat path's
// k2_colD and k2_rowE):
//   A row:  stage input -> E(eta^)+iE(u^), E(v^)+iE(Cm S u^), E(Cp S u^)+iE(Cm S v^), E(Cp S v^) -> inverse rows
//   B col:  inverse cols -> eta, u, v (kept), Cm/Cp applied u, v -> damping and gam products -> forward cols
//   C row:  forward rows -> split -> damping spectra, Csqr u^, Csqr v^ -> delu H1^, delv H1^ (kept)
//           -> E(M0u^)+iE(M0v^), E(L phi^) -> inverse rows
//   D col:  inverse cols -> M0u, M0v, L phi -> eta M0u, eta u, eta M0v, eta v, deletaH2 -> forward cols
//   E row:  forward rows -> split -> (eta u)^, (eta v)^, deletaH2^ (kept), E(Om (eta M0u)^)... -> inverse rows
//   F col:  inverse cols -> gam products of eta M0u, eta M0v and their Om images -> forward cols
//   G row:  forward rows -> split -> L(eta M0u)^, L(eta M0v)^ -> H2 terms -> S -> inverse rows (adjust)
#pragma once

#include "hw2d.cuh"

namespace hw2d {

// E or S of (table o) * S(a) at every point of a quad
__device__ __forceinline__ void op_sym(const double2 a[2][2], const Pair& P, const int cc[2], int r0, int r1, int Nx,
                                       int Ny, const double* __restrict__ o, double2 out[2][2]) {
  double2 sa[2][2];
#pragma unroll
  for (int k = 0; k < 2; ++k)
#pragma unroll
    for (int s = 0; s < 2; ++s) sa[k][s] = sym_at(a, P, k, s, cc[s], Nx, Ny, false);
#pragma unroll
  for (int k = 0; k < 2; ++k)
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const double t = o[(size_t)(k ? r1 : r0) * Nx + cc[s]];
      out[k][s] = make_double2(t * sa[k][s].x, t * sa[k][s].y);
    }
}

__device__ __forceinline__ double2 packc(double2 X, double2 Y) { return make_double2(X.x - Y.y, X.y + Y.x); }

// load a quad (columns j, cm of both rows) of slices s0 (row 0), s0 + 1 (row 1)
template <int M>
__device__ __forceinline__ void quad_load(double2* sm, int s0, const int cc[2], double2 z[2][2]) {
#pragma unroll
  for (int k = 0; k < 2; ++k)
#pragma unroll
    for (int s = 0; s < 2; ++s) z[k][s] = slot(sm, M, s0 + k, cc[s]);
}

// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2v_rowA(Tab2 tb, Work2 w, RK2 rk, const Ctl2* __restrict__ ctl, Ctl2* ctlw, int mode, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const size_t n = (size_t)tb.n;
  const Pair P = row_pair(blockIdx.x, Ny);
  const int r0 = P.r[0], r1 = P.r[1];
  const double ts = stage_time(ctl, mode);
  if (blockIdx.x == 0 && threadIdx.x == 0 && ctlw) ctlw->rhs += 1;
  if (tb.has_src && threadIdx.x < 2) {
    const int r = P.r[threadIdx.x];
    const size_t o = (size_t)r * tb.nt;
    w.insig[r] = spline2(tb.tsig, tb.sig + o, tb.sigc + o, tb.nt, ts);
    w.insigs[r] = spline2(tb.tsig, tb.sigs + o, tb.sigsc + o, tb.nt, ts);
  }
  for (int j = threadIdx.x; j <= Nx / 2; j += blockDim.x) {
    const int cm = (Nx - j) % Nx;
    const int cc[2] = {j, cm};
    // one pair of output slices at a time keeps the quad's live values few
    double2 a[2][2], b[2][2];
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const size_t q = (size_t)P.r[k] * Nx + cc[s];
        a[k][s] = w.z[q];
        b[k][s] = w.z[n + q];
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        put(sm, M, 0 + k, c, packc(sym_at(a, P, k, s, c, Nx, Ny, true), sym_at(b, P, k, s, c, Nx, Ny, true)));
      }
    double2 t[2][2];
    op_sym(b, P, cc, r0, r1, Nx, Ny, tb.cmin, t);        // Cm S(u^)
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) a[k][s] = w.z[2 * n + (size_t)P.r[k] * Nx + cc[s]];   // v^
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        put(sm, M, 2 + k, c, packc(sym_at(a, P, k, s, c, Nx, Ny, true), sym_at(t, P, k, s, c, Nx, Ny, true)));
      }
    op_sym(b, P, cc, r0, r1, Nx, Ny, tb.cplus, t);       // Cp S(u^)
    op_sym(a, P, cc, r0, r1, Nx, Ny, tb.cmin, b);        // Cm S(v^)
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        put(sm, M, 4 + k, c, packc(sym_at(t, P, k, s, c, Nx, Ny, true), sym_at(b, P, k, s, c, Nx, Ny, true)));
      }
    op_sym(a, P, cc, r0, r1, Nx, Ny, tb.cplus, t);       // Cp S(v^)
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        put(sm, M, 6 + k, c, packc(sym_at(t, P, k, s, c, Nx, Ny, true), make_double2(0.0, 0.0)));
      }
  }
  fft_slices<M>(sm, 8, tb.twx, +1);
  for (int s = 0; s < 8; ++s) {
    const int f = s >> 1, k = s & 1;
    double2* dst = w.R + f * n + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) dst[j] = slot(sm, M, s, j);
  }
}

// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2v_colB(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx;
  const size_t n = (size_t)tb.n;
  const int c = blockIdx.x;
  for (int f = 0; f < 4; ++f) col_load<M>(sm, 2 * f, w.R + f * n, Nx, c);
  fft_slices<M>(sm, 8, tb.twy, +1);
  const double invN = 1.0 / ((double)tb.n);
  for (int y = threadIdx.x; y < M; y += blockDim.x) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const size_t q = (size_t)y * Nx + 2 * c + k;
      const double2 P1 = slot(sm, M, 0 + k, y), P2 = slot(sm, M, 2 + k, y);
      const double2 P3 = slot(sm, M, 4 + k, y), P4 = slot(sm, M, 6 + k, y);
      const double eta = P1.x * invN, u = P1.y * invN, v = P2.x * invN;
      const double lmu = P2.y * invN, lpu = P3.x * invN, lmv = P3.y * invN, lpv = P4.x * invN;
      w.phys[q] = eta;
      w.phys[n + q] = u;
      w.phys[2 * n + q] = v;
      const double dmp = tb.damp[q], gm = tb.gmin[q], gp = tb.gplus[q];
      put(sm, M, 0 + k, y, make_double2(dmp * eta, dmp * u));
      put(sm, M, 2 + k, y, make_double2(dmp * v, gm * u));
      put(sm, M, 4 + k, y, make_double2(gp * u, gm * lmu));
      put(sm, M, 6 + k, y, make_double2(gp * lpu, gm * v));
      put(sm, M, 8 + k, y, make_double2(gp * v, gm * lmv));
      put(sm, M, 10 + k, y, make_double2(gp * lpv, 0.0));
    }
  }
  fft_slices<M>(sm, 12, tb.twy, -1);
  for (int f = 0; f < 6; ++f) col_store<M>(sm, 2 * f, w.Q + f * n, Nx, c);
}

// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2v_rowC(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const size_t n = (size_t)tb.n;
  const Pair P = row_pair(blockIdx.x, Ny);
  for (int s = 0; s < 12; ++s) {
    const int f = s >> 1, k = s & 1;
    const double2* src = w.Q + f * n + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) put(sm, M, s, j, src[j]);
  }
  fft_slices<M>(sm, 12, tb.twx, -1);
  for (int j = threadIdx.x; j <= Nx / 2; j += blockDim.x) {
    const int cm = (Nx - j) % Nx;
    const int cc[2] = {j, cm};
    double2 z[2][2], au[2][2], tu[2][2], av[2][2], tv[2][2];
    auto q_of = [&](int k, int s) { return (size_t)P.r[k] * Nx + cc[s]; };
    // Q1: damping of eta, u
    quad_load<M>(sm, 0, cc, z);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        double2 a, b;
        split2(z[k][s], z[P.mr[k]][s ^ 1], a, b);
        w.D[q_of(k, s)] = a;
        w.D[n + q_of(k, s)] = b;
      }
    // Q2: damping of v, F(gm u)
    quad_load<M>(sm, 2, cc, z);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double2 a, b;
        split2(z[k][s], z[P.mr[k]][s ^ 1], a, b);
        if (s == 0 || cm != j) w.D[2 * n + q_of(k, s)] = a;
        const double cmn = tb.cmin[q_of(k, s)];
        tu[k][s] = make_double2(cmn * b.x, cmn * b.y);   // Cm F(gm u)
      }
    // Q3: F(gp u), F(gm Lm u)
    quad_load<M>(sm, 4, cc, z);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double2 a, b;
        split2(z[k][s], z[P.mr[k]][s ^ 1], a, b);
        au[k][s] = make_double2(b.x + tu[k][s].x, b.y + tu[k][s].y);   // F(gm Lm u) + Cm F(gm u)
        const double cpl = tb.cplus[q_of(k, s)];
        tu[k][s] = make_double2(cpl * a.x, cpl * a.y);                   // Cp F(gp u)
      }
    // Q4: F(gp Lp u), F(gm v)
    quad_load<M>(sm, 6, cc, z);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double2 a, b;
        split2(z[k][s], z[P.mr[k]][s ^ 1], a, b);
        au[k][s] = make_double2((au[k][s].x + a.x + tu[k][s].x) / 2, (au[k][s].y + a.y + tu[k][s].y) / 2);
        const double cmn = tb.cmin[q_of(k, s)];
        tv[k][s] = make_double2(cmn * b.x, cmn * b.y);
      }
    // Q5: F(gp v), F(gm Lm v)
    quad_load<M>(sm, 8, cc, z);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double2 a, b;
        split2(z[k][s], z[P.mr[k]][s ^ 1], a, b);
        av[k][s] = make_double2(b.x + tv[k][s].x, b.y + tv[k][s].y);
        const double cpl = tb.cplus[q_of(k, s)];
        tv[k][s] = make_double2(cpl * a.x, cpl * a.y);
      }
    // Q6: F(gp Lp v)
    quad_load<M>(sm, 10, cc, z);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double2 a, b;
        split2(z[k][s], z[P.mr[k]][s ^ 1], a, b);
        av[k][s] = make_double2((av[k][s].x + a.x + tv[k][s].x) / 2, (av[k][s].y + a.y + tv[k][s].y) / 2);
      }
    // delu H1^ = -i kx Csqr u^ / g, delv H1^ = -i ky Csqr v^ / g (2d/fun_odesolver.c:2943-2946)
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const double kxv = tb.kx[cc[s]], kyv = tb.ky[P.r[k]];
        const double2 cu = au[k][s], cv = av[k][s];
        au[k][s] = make_double2(cu.y / kGrav * kxv, -cu.x / kGrav * kxv);
        av[k][s] = make_double2(cv.y / kGrav * kyv, -cv.x / kGrav * kyv);
        tu[k][s] = make_double2(au[k][s].x + av[k][s].x, au[k][s].y + av[k][s].y);   // L phi^
        if (s == 0 || cm != j) {
          w.H1[q_of(k, s)] = au[k][s];
          w.H1[n + q_of(k, s)] = av[k][s];
        }
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        put(sm, M, 0 + k, c, packc(sym_at(au, P, k, s, c, Nx, Ny, true), sym_at(av, P, k, s, c, Nx, Ny, true)));
        put(sm, M, 2 + k, c, packc(sym_at(tu, P, k, s, c, Nx, Ny, true), make_double2(0.0, 0.0)));
      }
  }
  fft_slices<M>(sm, 4, tb.twx, +1);
  for (int s = 0; s < 4; ++s) {
    const int f = s >> 1, k = s & 1;
    double2* dst = w.R + f * n + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) dst[j] = slot(sm, M, s, j);
  }
}

// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2v_colD(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx;
  const size_t n = (size_t)tb.n;
  const int c = blockIdx.x;
  for (int f = 0; f < 2; ++f) col_load<M>(sm, 2 * f, w.R + f * n, Nx, c);
  fft_slices<M>(sm, 4, tb.twy, +1);
  const double invN = 1.0 / ((double)tb.n);
  for (int y = threadIdx.x; y < M; y += blockDim.x) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const size_t q = (size_t)y * Nx + 2 * c + k;
      const double2 P1 = slot(sm, M, 0 + k, y), P2 = slot(sm, M, 2 + k, y);
      const double m0u = P1.x * invN, m0v = P1.y * invN, lphi = P2.x * invN;
      const double eta = w.phys[q], u = w.phys[n + q], v = w.phys[2 * n + q];
      const double wc = tb.wallchar ? tb.wallchar[q] : 1.0;   // H2 products x wallchar (:3416-3430)
      const double em = eta * m0u * wc, evm = eta * m0v * wc;
      w.pe[q] = em;
      w.pe[n + q] = evm;
      put(sm, M, 0 + k, y, make_double2(em, eta * u * wc));
      put(sm, M, 2 + k, y, make_double2(evm, eta * v * wc));
      put(sm, M, 4 + k, y, make_double2(0.5 * ((u * u + v * v) - lphi * lphi) * wc, 0.0));
    }
  }
  fft_slices<M>(sm, 6, tb.twy, -1);
  for (int f = 0; f < 3; ++f) col_store<M>(sm, 2 * f, w.Q + f * n, Nx, c);
}

// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2v_rowE(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const size_t n = (size_t)tb.n;
  const Pair P = row_pair(blockIdx.x, Ny);
  const int r0 = P.r[0], r1 = P.r[1];
  for (int s = 0; s < 6; ++s) {
    const int f = s >> 1, k = s & 1;
    const double2* src = w.Q + f * n + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) put(sm, M, s, j, src[j]);
  }
  fft_slices<M>(sm, 6, tb.twx, -1);
  for (int j = threadIdx.x; j <= Nx / 2; j += blockDim.x) {
    const int cm = (Nx - j) % Nx;
    const int cc[2] = {j, cm};
    double2 z1[2][2], z2[2][2], z3[2][2], em[2][2], ev[2][2];
    quad_load<M>(sm, 0, cc, z1);
    quad_load<M>(sm, 2, cc, z2);
    quad_load<M>(sm, 4, cc, z3);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double2 a, b, c2, d2, dh, zero;
        split2(z1[k][s], z1[P.mr[k]][s ^ 1], a, b);
        split2(z2[k][s], z2[P.mr[k]][s ^ 1], c2, d2);
        split2(z3[k][s], z3[P.mr[k]][s ^ 1], dh, zero);
        em[k][s] = a;
        ev[k][s] = c2;
        if (s == 0 || cm != j) {
          const size_t q = (size_t)P.r[k] * Nx + cc[s];
          w.EU[q] = b;
          w.EU[n + q] = d2;
          w.EU[2 * n + q] = dh;
        }
      }
    // E(Om_min (eta M0u)^) + i E(Om_plus (eta M0u)^); the same for v.  The spectra are
    // products of the tables with unsymmetrised transforms (HSSgen_2depth :516-526).
    double2 xm[2][2], xp[2][2];
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const size_t q = (size_t)(k ? r1 : r0) * Nx + cc[s];
        xm[k][s] = make_double2(tb.omin[q] * em[k][s].x, tb.omin[q] * em[k][s].y);
        xp[k][s] = make_double2(tb.oplus[q] * em[k][s].x, tb.oplus[q] * em[k][s].y);
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        put(sm, M, 0 + k, cc[s], packc(sym_at(xm, P, k, s, cc[s], Nx, Ny, true), sym_at(xp, P, k, s, cc[s], Nx, Ny, true)));
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const size_t q = (size_t)(k ? r1 : r0) * Nx + cc[s];
        xm[k][s] = make_double2(tb.omin[q] * ev[k][s].x, tb.omin[q] * ev[k][s].y);
        xp[k][s] = make_double2(tb.oplus[q] * ev[k][s].x, tb.oplus[q] * ev[k][s].y);
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        put(sm, M, 2 + k, cc[s], packc(sym_at(xm, P, k, s, cc[s], Nx, Ny, true), sym_at(xp, P, k, s, cc[s], Nx, Ny, true)));
      }
  }
  fft_slices<M>(sm, 4, tb.twx, +1);
  for (int s = 0; s < 4; ++s) {
    const int f = s >> 1, k = s & 1;
    double2* dst = w.R + f * n + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) dst[j] = slot(sm, M, s, j);
  }
}

// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2v_colF(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx;
  const size_t n = (size_t)tb.n;
  const int c = blockIdx.x;
  for (int f = 0; f < 2; ++f) col_load<M>(sm, 2 * f, w.R + f * n, Nx, c);
  fft_slices<M>(sm, 4, tb.twy, +1);
  const double invN = 1.0 / ((double)tb.n);
  for (int y = threadIdx.x; y < M; y += blockDim.x) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const size_t q = (size_t)y * Nx + 2 * c + k;
      const double2 P1 = slot(sm, M, 0 + k, y), P2 = slot(sm, M, 2 + k, y);
      const double lmu = P1.x * invN, lpu = P1.y * invN, lmv = P2.x * invN, lpv = P2.y * invN;
      const double em = w.pe[q], ev = w.pe[n + q];
      const double gm = tb.gmin[q], gp = tb.gplus[q];
      put(sm, M, 0 + k, y, make_double2(gm * em, gp * em));
      put(sm, M, 2 + k, y, make_double2(gm * lmu, gp * lpu));
      put(sm, M, 4 + k, y, make_double2(gm * ev, gp * ev));
      put(sm, M, 6 + k, y, make_double2(gm * lmv, gp * lpv));
    }
  }
  fft_slices<M>(sm, 8, tb.twy, -1);
  for (int f = 0; f < 4; ++f) col_store<M>(sm, 2 * f, w.Q + f * n, Nx, c);
}

// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2v_rowG(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const size_t n = (size_t)tb.n;
  const Pair P = row_pair(blockIdx.x, Ny);
  for (int s = 0; s < 8; ++s) {
    const int f = s >> 1, k = s & 1;
    const double2* src = w.Q + f * n + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) put(sm, M, s, j, src[j]);
  }
  fft_slices<M>(sm, 8, tb.twx, -1);
  for (int j = threadIdx.x; j <= Nx / 2; j += blockDim.x) {
    const int cm = (Nx - j) % Nx;
    const int cc[2] = {j, cm};
    auto q_of = [&](int k, int s) { return (size_t)P.r[k] * Nx + cc[s]; };
    double2 z[2][2], acc[2][2], t2[2][2], a1[2][2], a2[2][2];
    // L (eta M0u)^ = [F(gm Lm) + Om_min F(gm .) + F(gp Lp) + Om_plus F(gp .)] / 2
    quad_load<M>(sm, 0, cc, z);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double2 a, b;
        split2(z[k][s], z[P.mr[k]][s ^ 1], a, b);
        const size_t q = q_of(k, s);
        acc[k][s] = make_double2(tb.omin[q] * a.x, tb.omin[q] * a.y);
        t2[k][s] = make_double2(tb.oplus[q] * b.x, tb.oplus[q] * b.y);
      }
    quad_load<M>(sm, 2, cc, z);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double2 a, b;
        split2(z[k][s], z[P.mr[k]][s ^ 1], a, b);
        const double2 L = make_double2((a.x + acc[k][s].x + b.x + t2[k][s].x) / 2,
                                       (a.y + acc[k][s].y + b.y + t2[k][s].y) / 2);
        const size_t q = q_of(k, s);
        const double2 eu = w.EU[q];
        const double kxv = tb.kx[cc[s]];
        a1[k][s] = make_double2(kxv * eu.y - L.x / kGrav, -kxv * eu.x - L.y / kGrav);   // delu H2^
      }
    quad_load<M>(sm, 4, cc, z);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double2 a, b;
        split2(z[k][s], z[P.mr[k]][s ^ 1], a, b);
        const size_t q = q_of(k, s);
        acc[k][s] = make_double2(tb.omin[q] * a.x, tb.omin[q] * a.y);
        t2[k][s] = make_double2(tb.oplus[q] * b.x, tb.oplus[q] * b.y);
      }
    quad_load<M>(sm, 6, cc, z);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double2 a, b;
        split2(z[k][s], z[P.mr[k]][s ^ 1], a, b);
        const double2 L = make_double2((a.x + acc[k][s].x + b.x + t2[k][s].x) / 2,
                                       (a.y + acc[k][s].y + b.y + t2[k][s].y) / 2);
        const size_t q = q_of(k, s);
        const double2 ev = w.EU[n + q];
        const double kyv = tb.ky[P.r[k]];
        a2[k][s] = make_double2(kyv * ev.y - L.x / kGrav, -kyv * ev.x - L.y / kGrav);   // delv H2^
      }
    // i kx deletaH2^, i ky deletaH2^
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const double2 dh = w.EU[2 * n + q_of(k, s)];
        acc[k][s] = mul_pi(dh, tb.kx[cc[s]]);
        t2[k][s] = mul_pi(dh, tb.ky[P.r[k]]);
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        put(sm, M, 0 + k, c, sym_at(acc, P, k, s, c, Nx, Ny, false));
        put(sm, M, 2 + k, c, sym_at(t2, P, k, s, c, Nx, Ny, false));
        put(sm, M, 4 + k, c, sym_at(a1, P, k, s, c, Nx, Ny, false));
        put(sm, M, 6 + k, c, sym_at(a2, P, k, s, c, Nx, Ny, false));
      }
  }
  __syncthreads();
  double2* dst = tb.chi_one ? w.V : w.W;
  if (!tb.chi_one) fft_slices<M>(sm, 8, tb.twx, +1);
  for (int s = 0; s < 8; ++s) {
    const int f = s >> 1, k = s & 1;
    double2* d = dst + f * n + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) d[j] = slot(sm, M, s, j);
  }
}

}  // namespace hw2d
