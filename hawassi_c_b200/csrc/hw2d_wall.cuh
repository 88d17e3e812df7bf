// hw2d_wall.cuh -- harbour walls on the flat bottom: fun_delphiH1hat's branch for
// refl_coef < 1 (2d/fun_odesolver.c:2172-2219).  With walls the flat RHS takes
// delphiH1^ = -i (kx (C/g) F(wallchar Re F^-1 S(C u^)) + ky (C/g) F(wallchar Re F^-1 S(C v^)))
// instead of -i (kx C^2/g u^ + ky C^2/g v^): one round trip of the pair (C u^, C v^)
// through physical space, packed as one complex transform each way.
//   W1 (row pass)  E(S(C u^)) + i E(S(C v^)) -> inverse row FFT
//   W2 (col pass)  inverse column FFT, x wallchar / N (both real fields), forward column FFT
//   W3 (row pass)  forward row FFT, split, x C/g, -i (kx . + ky .) -> delphiH1^ (w.H1)
// The H2 products of the column pass carry wallchar as well (:3239-3249).
//
// With refl_coef == 1 the branch at :2105-2170 runs instead: Flux = Re F^-1 S(C^2/g u^)
// (both components), divC2u from the symmetrised spectra, and
// delphiH1^ = F(divC2u wallchar) - F(Flux . grad wallchar):
//   V1 (row pass)  E(S(C^2/g u^)) + i E(S(C^2/g v^)), E(S(D)) with D = -i(kx S(.) + ky S(.))
//                  -> inverse row FFT (four slices)
//   V2 (col pass)  inverse column FFT -> Flux, divC2u -> divC2u wallchar + i Flux . grad
//                  wallchar -> forward column FFT
//   V3 (row pass)  forward row FFT, split, difference -> delphiH1^ (w.H1)
#pragma once

#include "hw2d.cuh"

namespace hw2d {

template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2w_row1(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const size_t n = (size_t)tb.n;
  const Pair P = row_pair(blockIdx.x, Ny);
  for (int j = threadIdx.x; j <= Nx / 2; j += blockDim.x) {
    const int cm = (Nx - j) % Nx;
    const int cc[2] = {j, cm};
    double2 A[2][2], B[2][2];
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const size_t q = (size_t)P.r[k] * Nx + cc[s];
        const double C = tb.c2d[q];
        const double2 zu = w.z[n + q], zv = w.z[2 * n + q];
        A[k][s] = make_double2(C * zu.x, C * zu.y);
        B[k][s] = make_double2(C * zv.x, C * zv.y);
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        const double2 ea = sym_at(A, P, k, s, c, Nx, Ny, true), eb = sym_at(B, P, k, s, c, Nx, Ny, true);
        put(sm, M, k, c, make_double2(ea.x - eb.y, ea.y + eb.x));
      }
  }
  fft_slices<M>(sm, 2, tb.twx, +1);
  for (int k = 0; k < 2; ++k) {
    double2* dst = w.WP + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) dst[j] = slot(sm, M, k, j);
  }
}

template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2w_col2(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx;
  const int c = blockIdx.x;
  col_load<M>(sm, 0, w.WP, Nx, c);
  fft_slices<M>(sm, 2, tb.twy, +1);
  const double invN = 1.0 / ((double)tb.n);
  for (int y = threadIdx.x; y < M; y += blockDim.x)
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const size_t q = (size_t)y * Nx + 2 * c + k;
      const double2 v = slot(sm, M, k, y);
      const double wc = tb.wallchar[q];
      put(sm, M, k, y, make_double2(v.x * invN * wc, v.y * invN * wc));
    }
  fft_slices<M>(sm, 2, tb.twy, -1);
  col_store<M>(sm, 0, w.WP, Nx, c);
}

template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2w_row3(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const Pair P = row_pair(blockIdx.x, Ny);
  for (int k = 0; k < 2; ++k) {
    const double2* src = w.WP + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) put(sm, M, k, j, src[j]);
  }
  fft_slices<M>(sm, 2, tb.twx, -1);
  for (int k = 0; k < 2; ++k) {
    const int r = P.r[k];
    const double kyv = tb.ky[r];
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) {
      const size_t q = (size_t)r * Nx + j;
      double2 X, Y;   // F(wallchar C u), F(wallchar C v)
      split2(slot(sm, M, k, j), slot(sm, M, P.mr[k], (Nx - j) % Nx), X, Y);
      const double cg = tb.c2d[q] / kGrav;
      const double2 du = make_double2(cg * X.x, cg * X.y), dv = make_double2(cg * Y.x, cg * Y.y);
      const double kxv = tb.kx[j];
      w.H1[q] = make_double2(kxv * du.y + kyv * dv.y, -kxv * du.x - kyv * dv.x);
    }
  }
}

template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2w_rowV1(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const size_t n = (size_t)tb.n;
  const Pair P = row_pair(blockIdx.x, Ny);
  for (int j = threadIdx.x; j <= Nx / 2; j += blockDim.x) {
    const int cm = (Nx - j) % Nx;
    const int cc[2] = {j, cm};
    double2 A[2][2], B[2][2], D[2][2];
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const size_t q = (size_t)P.r[k] * Nx + cc[s];
        const double cg = tb.c2g[q];
        const double2 zu = w.z[n + q], zv = w.z[2 * n + q];
        A[k][s] = make_double2(cg * zu.x, cg * zu.y);
        B[k][s] = make_double2(cg * zv.x, cg * zv.y);
      }
    // divC2u^ from the symmetrised spectra at every point of the quad
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const int c = cc[s];
        const double2 sa = sym_at(A, P, k, s, c, Nx, Ny, false), sb = sym_at(B, P, k, s, c, Nx, Ny, false);
        const double kxv = tb.kx[c], kyv = tb.ky[P.r[k]];
        D[k][s] = make_double2(-(-kxv * sa.y - kyv * sb.y), -(kxv * sa.x + kyv * sb.x));
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        const double2 ea = sym_at(A, P, k, s, c, Nx, Ny, true), eb = sym_at(B, P, k, s, c, Nx, Ny, true);
        put(sm, M, k, c, make_double2(ea.x - eb.y, ea.y + eb.x));
        put(sm, M, 2 + k, c, sym_at(D, P, k, s, c, Nx, Ny, true));
      }
  }
  fft_slices<M>(sm, 4, tb.twx, +1);
  for (int f = 0; f < 2; ++f)
    for (int k = 0; k < 2; ++k) {
      double2* dst = w.WP + f * n + (size_t)P.r[k] * Nx;
      for (int j = threadIdx.x; j < Nx; j += blockDim.x) dst[j] = slot(sm, M, 2 * f + k, j);
    }
}

template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2w_colV2(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx;
  const size_t n = (size_t)tb.n;
  const int c = blockIdx.x;
  col_load<M>(sm, 0, w.WP, Nx, c);
  col_load<M>(sm, 2, w.WP + n, Nx, c);
  fft_slices<M>(sm, 4, tb.twy, +1);
  const double invN = 1.0 / ((double)tb.n);
  for (int y = threadIdx.x; y < M; y += blockDim.x)
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const size_t q = (size_t)y * Nx + 2 * c + k;
      const double2 fl = slot(sm, M, k, y), dv = slot(sm, M, 2 + k, y);
      const double fx = fl.x * invN, fy = fl.y * invN, div = dv.x * invN;
      put(sm, M, k, y, make_double2(div * tb.wallchar[q], fx * tb.gwx[q] + fy * tb.gwy[q]));
    }
  fft_slices<M>(sm, 2, tb.twy, -1);
  col_store<M>(sm, 0, w.WP, Nx, c);
}

template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2w_rowV3(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const Pair P = row_pair(blockIdx.x, Ny);
  for (int k = 0; k < 2; ++k) {
    const double2* src = w.WP + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) put(sm, M, k, j, src[j]);
  }
  fft_slices<M>(sm, 2, tb.twx, -1);
  for (int k = 0; k < 2; ++k) {
    const int r = P.r[k];
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) {
      double2 X, Y;   // F(divC2u wallchar), F(Flux . grad wallchar)
      split2(slot(sm, M, k, j), slot(sm, M, P.mr[k], (Nx - j) % Nx), X, Y);
      w.H1[(size_t)r * Nx + j] = make_double2(X.x - Y.x, X.y - Y.y);
    }
  }
}

}  // namespace hw2d
