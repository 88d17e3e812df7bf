// hw2d_hs3.cuh -- HS3 on the flat bottom (rhs_AB3_2DF_uv, 2d/fun_odesolver.c:4628-4734,
// with fun_termshat_AB3_2DF_uv :3512-3897).  The cubic terms
//   deluH3^ = L (eta L(eta M0u))^ + L (eta^2 dx u)^ / 2 - kx^2 (eta^2 M0u)^ / 2
//   delvH3^ = L (eta L(eta M0v))^ + L (eta^2 dy v)^ / 2 - ky^2 (eta^2 M0v)^ / 2
//   deletaH3 = Lphi eta div(grad phi) + Lphi L(eta Lphi)      (i kx, i ky of its spectrum)
// need one more round trip through physical space after the HS2 products.  The
// HS2 passes A, D, E stay; B and C are replaced by four passes:
//   B3 (col)  as B, plus eta^2 M0u + i eta^2 M0v (ten slices); eta and L phi kept in
//             physical space
//   C3 (row)  forward rows, split: damping spectra, the four HS2 terms and
//             (eta^2 M0u)^, (eta^2 M0v)^ kept unsymmetrised; E(S(L(eta M0u)^)) +
//             i E(S(L(eta M0v)^)), E(S(i kx u^)) + i E(S(i ky v^)) -> inverse rows
//   H3 (col)  inverse columns -> L(eta M0u), L(eta M0v), dx u, dy v -> the five cubic
//             products packed in three fields -> forward columns
//   I3 (row)  forward rows, split, the cubic terms added to the HS2 terms, S ->
//             inverse rows into pass D's input (or, with ChiAdj = 1, pass E's)
// The reference adjusts each of the eight terms on its own and sums the results;
// fun_adjust is linear, so the sums are adjusted here (four adjusted fields, as HS2).
// div(grad phi) and L(eta Lphi), which the reference transforms from the summed
// spectra, are the sums dx u + dy v and L(eta M0u) + L(eta M0v) in physical space.
#pragma once

#include "hw2d.cuh"

namespace hw2d {

template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2_colB3(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx;
  const size_t n = (size_t)tb.n;
  const int c = blockIdx.x;
  for (int f = 0; f < 3; ++f) col_load<M>(sm, 2 * f, w.R + f * n, Nx, c);
  fft_slices<M>(sm, 6, tb.twy, +1);
  const double invN = 1.0 / ((double)tb.n);
  for (int y = threadIdx.x; y < M; y += blockDim.x) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const size_t q = (size_t)y * Nx + 2 * c + k;
      const double2 P1 = slot(sm, M, 0 + k, y), P2 = slot(sm, M, 2 + k, y), P3 = slot(sm, M, 4 + k, y);
      const double eta = P1.x * invN, lphi = P1.y * invN;
      const double u = P2.x * invN, m0u = P2.y * invN;
      const double v = P3.x * invN, m0v = P3.y * invN;
      if (w.phys) {   // kept for the breaking kernels
        w.phys[q] = eta;
        w.phys[n + q] = u;
        w.phys[2 * n + q] = v;
      }
      w.p3[q] = eta;
      w.p3[n + q] = lphi;
      const double dmp = tb.damp[q];
      const double wc = tb.wallchar ? tb.wallchar[q] : 1.0;   // dominfo.wallchar (1 without walls)
      put(sm, M, 0 + k, y, make_double2(dmp * eta, dmp * u));
      put(sm, M, 2 + k, y, make_double2(dmp * v, 0.5 * ((u * u + v * v) - lphi * lphi) * wc));
      put(sm, M, 4 + k, y, make_double2(eta * m0u * wc, eta * u * wc));
      put(sm, M, 6 + k, y, make_double2(eta * m0v * wc, eta * v * wc));
      put(sm, M, 8 + k, y, make_double2(eta * eta * m0u * wc, eta * eta * m0v * wc));
    }
  }
  fft_slices<M>(sm, 10, tb.twy, -1);
  for (int f = 0; f < 5; ++f) col_store<M>(sm, 2 * f, w.Q + f * n, Nx, c);
}

// T3 fields: 0 i kx deletaH2^, 1 i ky deletaH2^, 2 deluH2^, 3 delvH2^,
// 4 (eta^2 M0u)^, 5 (eta^2 M0v)^ (all unsymmetrised)
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2_rowC3(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const size_t n = (size_t)tb.n;
  const Pair P = row_pair(blockIdx.x, Ny);
  for (int s = 0; s < 10; ++s) {
    const int f = s >> 1, k = s & 1;
    const double2* src = w.Q + f * n + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) put(sm, M, s, j, src[j]);
  }
  fft_slices<M>(sm, 10, tb.twx, -1);
  // One thread reads and rewrites each quad at its own positions only; slices 0..3
  // receive the packed inverse inputs after all ten of the quad's values are read.
  for (int j = threadIdx.x; j <= Nx / 2; j += blockDim.x) {
    const int cm = (Nx - j) % Nx;
    const int cc[2] = {j, cm};
    double2 z[2][2], lu[2][2], lv[2][2], dxu[2][2], dyv[2][2];
    // Q1 -> damping spectra of eta and u
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) z[k][s] = slot(sm, M, 0 + k, cc[s]);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        double2 de, du;
        split2(z[k][s], z[P.mr[k]][s ^ 1], de, du);
        const size_t q = (size_t)P.r[k] * Nx + cc[s];
        w.D[q] = de;
        w.D[n + q] = du;
      }
    // Q2 -> damping spectrum of v; i kx deletaH2^, i ky deletaH2^
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) z[k][s] = slot(sm, M, 2 + k, cc[s]);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        double2 dv, dH;
        split2(z[k][s], z[P.mr[k]][s ^ 1], dv, dH);
        const int r = P.r[k], c = cc[s];
        const size_t q = (size_t)r * Nx + c;
        w.D[2 * n + q] = dv;
        w.T3[q] = mul_pi(dH, tb.kx[c]);
        w.T3[n + q] = mul_pi(dH, tb.ky[r]);
      }
    // Q3 -> deluH2^ = -L (eta M0u)^ - i kx (eta u)^ ; L (eta M0u)^
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) z[k][s] = slot(sm, M, 4 + k, cc[s]);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double2 em, eu;
        split2(z[k][s], z[P.mr[k]][s ^ 1], em, eu);
        const int r = P.r[k], c = cc[s];
        const size_t q = (size_t)r * Nx + c;
        const double L = tb.l2d[q], kxv = tb.kx[c];
        lu[k][s] = make_double2(L * em.x, L * em.y);
        if (s == 0 || cm != j) w.T3[2 * n + q] = make_double2(-lu[k][s].x + kxv * eu.y, -lu[k][s].y - kxv * eu.x);
      }
    // Q4 -> delvH2^ = -L (eta M0v)^ - i ky (eta v)^ ; L (eta M0v)^
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) z[k][s] = slot(sm, M, 6 + k, cc[s]);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double2 em, ev;
        split2(z[k][s], z[P.mr[k]][s ^ 1], em, ev);
        const int r = P.r[k], c = cc[s];
        const size_t q = (size_t)r * Nx + c;
        const double L = tb.l2d[q], kyv = tb.ky[r];
        lv[k][s] = make_double2(L * em.x, L * em.y);
        if (s == 0 || cm != j) w.T3[3 * n + q] = make_double2(-lv[k][s].x + kyv * ev.y, -lv[k][s].y - kyv * ev.x);
      }
    // Q5 -> (eta^2 M0u)^, (eta^2 M0v)^
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) z[k][s] = slot(sm, M, 8 + k, cc[s]);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        double2 a, b;
        split2(z[k][s], z[P.mr[k]][s ^ 1], a, b);
        const size_t q = (size_t)P.r[k] * Nx + cc[s];
        w.T3[4 * n + q] = a;
        w.T3[5 * n + q] = b;
      }
    // i kx u^, i ky v^ of the stage input (dxu_hat, dyv_hat)
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const int r = P.r[k], c = cc[s];
        const size_t q = (size_t)r * Nx + c;
        const double2 zu = w.z[n + q], zv = w.z[2 * n + q];
        const double kxv = tb.kx[c], kyv = tb.ky[r];
        dxu[k][s] = make_double2(-kxv * zu.y, kxv * zu.x);
        dyv[k][s] = make_double2(-kyv * zv.y, kyv * zv.x);
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        const double2 a = sym_at(lu, P, k, s, c, Nx, Ny, true), b = sym_at(lv, P, k, s, c, Nx, Ny, true);
        const double2 e = sym_at(dxu, P, k, s, c, Nx, Ny, true), f = sym_at(dyv, P, k, s, c, Nx, Ny, true);
        put(sm, M, 0 + k, c, make_double2(a.x - b.y, a.y + b.x));
        put(sm, M, 2 + k, c, make_double2(e.x - f.y, e.y + f.x));
      }
  }
  fft_slices<M>(sm, 4, tb.twx, +1);
  for (int s = 0; s < 4; ++s) {
    const int f = s >> 1, k = s & 1;
    double2* dst = w.R + f * n + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) dst[j] = slot(sm, M, s, j);
  }
}

template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2_colH3(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx;
  const size_t n = (size_t)tb.n;
  const int c = blockIdx.x;
  col_load<M>(sm, 0, w.R, Nx, c);
  col_load<M>(sm, 2, w.R + n, Nx, c);
  fft_slices<M>(sm, 4, tb.twy, +1);
  const double invN = 1.0 / ((double)tb.n);
  for (int y = threadIdx.x; y < M; y += blockDim.x) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const size_t q = (size_t)y * Nx + 2 * c + k;
      const double2 a = slot(sm, M, 0 + k, y), b = slot(sm, M, 2 + k, y);
      const double lmu = a.x * invN, lmv = a.y * invN, dxu = b.x * invN, dyv = b.y * invN;
      const double eta = w.p3[q], lphi = w.p3[n + q];
      const double wc = tb.wallchar ? tb.wallchar[q] : 1.0;
      const double divg = dxu + dyv, lel = lmu + lmv;
      put(sm, M, 0 + k, y, make_double2(eta * lmu, eta * lmv));
      put(sm, M, 2 + k, y, make_double2(eta * eta * dxu * wc, eta * eta * dyv * wc));
      put(sm, M, 4 + k, y, make_double2(lphi * eta * divg + lphi * lel, 0.0));
    }
  }
  fft_slices<M>(sm, 6, tb.twy, -1);
  for (int f = 0; f < 3; ++f) col_store<M>(sm, 2 * f, w.Q + f * n, Nx, c);
}

template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2_rowI3(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const size_t n = (size_t)tb.n;
  const Pair P = row_pair(blockIdx.x, Ny);
  for (int s = 0; s < 6; ++s) {
    const int f = s >> 1, k = s & 1;
    const double2* src = w.Q + f * n + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) put(sm, M, s, j, src[j]);
  }
  fft_slices<M>(sm, 6, tb.twx, -1);
  for (int j = threadIdx.x; j <= Nx / 2; j += blockDim.x) {
    const int cm = (Nx - j) % Nx;
    const int cc[2] = {j, cm};
    double2 y1[2][2], y2[2][2], y3[2][2];
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        y1[k][s] = slot(sm, M, 0 + k, cc[s]);
        y2[k][s] = slot(sm, M, 2 + k, cc[s]);
        y3[k][s] = slot(sm, M, 4 + k, cc[s]);
      }
    double2 f0[2][2], f1[2][2], f2[2][2], f3[2][2];
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const int r = P.r[k], c = cc[s];
        const size_t q = (size_t)r * Nx + c;
        double2 au, av, bu, bv, h3, zero;
        split2(y1[k][s], y1[P.mr[k]][s ^ 1], au, av);   // (eta L(eta M0u))^, (eta L(eta M0v))^
        split2(y2[k][s], y2[P.mr[k]][s ^ 1], bu, bv);   // (eta^2 dx u)^, (eta^2 dy v)^
        split2(y3[k][s], y3[P.mr[k]][s ^ 1], h3, zero); // deletaH3^
        const double L = tb.l2d[q], kxv = tb.kx[c], kyv = tb.ky[r];
        const double2 cu = w.T3[4 * n + q], cv = w.T3[5 * n + q];
        const double hl = 0.5 * L, kx2 = kxv * kxv, ky2 = kyv * kyv;
        const double2 du3 = make_double2(L * au.x + hl * bu.x - 0.5 * (kx2 * cu.x),
                                         L * au.y + hl * bu.y - 0.5 * (kx2 * cu.y));
        const double2 dv3 = make_double2(L * av.x + hl * bv.x - 0.5 * (ky2 * cv.x),
                                         L * av.y + hl * bv.y - 0.5 * (ky2 * cv.y));
        const double2 ix3 = mul_pi(h3, kxv), iy3 = mul_pi(h3, kyv);
        const double2 ix2 = w.T3[q], iy2 = w.T3[n + q], du2 = w.T3[2 * n + q], dv2 = w.T3[3 * n + q];
        f0[k][s] = make_double2(ix2.x + ix3.x, ix2.y + ix3.y);
        f1[k][s] = make_double2(iy2.x + iy3.x, iy2.y + iy3.y);
        f2[k][s] = make_double2(du2.x + du3.x, du2.y + du3.y);
        f3[k][s] = make_double2(dv2.x + dv3.x, dv2.y + dv3.y);
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        put(sm, M, 0 + k, c, sym_at(f0, P, k, s, c, Nx, Ny, false));
        put(sm, M, 2 + k, c, sym_at(f1, P, k, s, c, Nx, Ny, false));
        put(sm, M, 4 + k, c, sym_at(f2, P, k, s, c, Nx, Ny, false));
        put(sm, M, 6 + k, c, sym_at(f3, P, k, s, c, Nx, Ny, false));
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
