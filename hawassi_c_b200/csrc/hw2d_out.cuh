// hw2d_out.cuh -- the output stage of the 2D time loop (ode_solver_uv,
// 2d/fun_odesolver.c:2646-2664): eta, u and v in physical space at an output time.
// Each is ifftw_2d_c2r of a copy of its spectrum (2d/functions1.c:523-557): the
// fftwcomplex-style symmetrisation S, the backward 2D transform, the real part
// divided by Nx Ny.  The real part of the inverse transform of S(A) is the inverse
// transform of E(S(A)), the Hermitian part, so two fields share one complex
// transform:
//   O1 (row pass)  E(S(eta^)) + i E(S(u^)), E(S(v^)) -> inverse row FFT (four slices)
//   O2 (col pass)  inverse column FFT, / (Nx Ny) -> eta, u, v in FP64 and the FP32
//                  copies the field files hold (fwrite of float(eta), :2705-2722)
//   gauge          eta, u, v at the gauges' grid points (print_data_gauges_uv, :427-476)
// d(eta)/dt, which the loop also transforms, feeds only the 2D kinematics module.
#pragma once

#include "hw2d.cuh"

namespace hw2d {

template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2o_row(Tab2 tb, const double2* __restrict__ z, double2* __restrict__ P) {
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const size_t n = (size_t)tb.n;
  const Pair pr = row_pair(blockIdx.x, Ny);
  for (int j = threadIdx.x; j <= Nx / 2; j += blockDim.x) {
    const int cm = (Nx - j) % Nx;
    const int cc[2] = {j, cm};
    double2 A[2][2], B[2][2], C[2][2];
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const size_t q = (size_t)pr.r[k] * Nx + cc[s];
        A[k][s] = z[q];
        B[k][s] = z[n + q];
        C[k][s] = z[2 * n + q];
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        const double2 ea = sym_at(A, pr, k, s, c, Nx, Ny, true), eb = sym_at(B, pr, k, s, c, Nx, Ny, true);
        put(sm, M, k, c, make_double2(ea.x - eb.y, ea.y + eb.x));
        put(sm, M, 2 + k, c, sym_at(C, pr, k, s, c, Nx, Ny, true));
      }
  }
  fft_slices<M>(sm, 4, tb.twx, +1);
  for (int f = 0; f < 2; ++f)
    for (int k = 0; k < 2; ++k) {
      double2* dst = P + f * n + (size_t)pr.r[k] * Nx;
      for (int j = threadIdx.x; j < Nx; j += blockDim.x) dst[j] = slot(sm, M, 2 * f + k, j);
    }
}

// phys: eta, u, v (3 n doubles); f32: the same as floats (nullptr: not kept)
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2o_col(Tab2 tb, const double2* __restrict__ P, double* __restrict__ phys, float* __restrict__ f32) {
  extern __shared__ double2 sm[];
  const int Nx = tb.nx;
  const size_t n = (size_t)tb.n;
  const int c = blockIdx.x;
  col_load<M>(sm, 0, P, Nx, c);
  col_load<M>(sm, 2, P + n, Nx, c);
  fft_slices<M>(sm, 4, tb.twy, +1);
  const double invN = 1.0 / ((double)tb.n);
  for (int y = threadIdx.x; y < M; y += blockDim.x)
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const size_t q = (size_t)y * Nx + 2 * c + k;
      const double2 a = slot(sm, M, k, y), b = slot(sm, M, 2 + k, y);
      const double eta = a.x * invN, u = a.y * invN, v = b.x * invN;
      phys[q] = eta;
      phys[n + q] = u;
      phys[2 * n + q] = v;
      if (f32) {
        f32[q] = (float)eta;
        f32[n + q] = (float)u;
        f32[2 * n + q] = (float)v;
      }
    }
}

// out[3 g + f] = field f at gauge g (pt[g] = iy nx + ix, checked on the host)
__global__ void k2o_gauge(const double* __restrict__ phys, const int* __restrict__ pt, int ng, size_t n,
                          double* __restrict__ out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ng) return;
  const size_t q = (size_t)pt[g];
#pragma unroll
  for (int f = 0; f < 3; ++f) out[3 * g + f] = phys[f * n + q];
}

}  // namespace hw2d
