// hw2d_influx.cu -- the directional JONSWAP line signal of the 2D set-up on the device:
// jonswap_influx (2d/functions.c:2310-2446) adds, for every time sample and every point
// of a vertical influx line, one cosine per spectral component (Nt/2 components, one
// direction each) -- Nt x lines x Nt/2 terms, the set-up's dominant cost (4.6e9 terms
// for 300 s at 0.1 s on 1024 lines).  Here one thread owns 16 consecutive samples of
// one line point: per component one sincos at the first sample, then the phase steps
// back by w dt per sample as a rotation by exp(-i w dt) (cos / sin of w dt computed
// once per component), accumulating the cosine (the elevation) and the sine (its
// quadrature, the skew signal of the source) of the same phase.  Components are staged
// through shared memory in chunks.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/hawassi_b200.h"

namespace {

constexpr int kSamplesPerThread = 16;
constexpr int kThreads = 128;
constexpr int kChunk = 256;   // components staged in shared memory at a time

// per component: amplitude, w, cross-line wavenumber k sin(theta + mdir), phase,
// cos(w dt), sin(w dt)
__global__ void k_component_table(int nc, const double* __restrict__ a, const double* __restrict__ w,
                                  const double* __restrict__ k, const double* __restrict__ theta,
                                  const double* __restrict__ phi, double mdir, double dt, double* __restrict__ tab) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double sw, cw;
  sincos(w[c] * dt, &sw, &cw);
  tab[6 * c + 0] = a[c];
  tab[6 * c + 1] = w[c];
  tab[6 * c + 2] = k[c] * sin(theta[c] + mdir);
  tab[6 * c + 3] = phi[c];
  tab[6 * c + 4] = cw;
  tab[6 * c + 5] = sw;
}

// eta[j][i], skew[j][i] (line j, sample i) for a line of points y[j], times t0 + i dt
__global__ void __launch_bounds__(kThreads) k_line_signal(int nt, double t0, double dt, const double* __restrict__ y,
                                                          double y0, int nc, const double* __restrict__ tab,
                                                          const double* __restrict__ ramp_t,
                                                          const double* __restrict__ ramp_y, double* __restrict__ eta,
                                                          double* __restrict__ skew) {
  __shared__ double st[6 * kChunk];
  const int j = blockIdx.y;
  const int i0 = (blockIdx.x * kThreads + threadIdx.x) * kSamplesPerThread;
  const double yj = y[j] - y0;
  const double ti0 = t0 + i0 * dt;
  double ac[kSamplesPerThread], as[kSamplesPerThread];
#pragma unroll
  for (int q = 0; q < kSamplesPerThread; ++q) ac[q] = as[q] = 0.0;
  for (int c0 = 0; c0 < nc; c0 += kChunk) {
    const int n = min(kChunk, nc - c0);
    __syncthreads();
    for (int e = threadIdx.x; e < 6 * n; e += kThreads) st[e] = tab[6 * c0 + e];
    __syncthreads();
    if (i0 < nt) {
      for (int c = 0; c < n; ++c) {
        const double* p = st + 6 * c;
        const double amp = p[0], cw = p[4], sw = p[5];
        double s, co;
        sincos(-p[1] * ti0 + p[3] + p[2] * yj, &s, &co);
#pragma unroll
        for (int q = 0; q < kSamplesPerThread; ++q) {
          ac[q] = fma(amp, co, ac[q]);
          as[q] = fma(amp, s, as[q]);
          const double cn = co * cw + s * sw;   // exp(i (psi - w dt))
          s = s * cw - co * sw;
          co = cn;
        }
      }
    }
  }
  if (i0 >= nt) return;
  const double ry = ramp_y[j];
#pragma unroll
  for (int q = 0; q < kSamplesPerThread; ++q) {
    const int i = i0 + q;
    if (i < nt) {
      const double r = ramp_t[i] * ry;
      eta[(size_t)j * nt + i] = ac[q] * r;
      skew[(size_t)j * nt + i] = as[q] * r;
    }
  }
}

std::string g_err;

}  // namespace

extern "C" {

const char* hw2d_influx_last_error() { return g_err.c_str(); }

int hw2d_directional_influx(int nt, double t0, double dt, int nlines, const double* y, double y0, int nc,
                            const double* a, const double* w, const double* k, const double* theta,
                            const double* phi, double mdir, const double* ramp_t, const double* ramp_y, double* eta,
                            double* skew, int device) {
  if (nt <= 0 || nlines <= 0 || nc <= 0 || nlines > 65535 || !y || !a || !w || !k || !theta || !phi || !ramp_t ||
      !ramp_y || !eta || !skew || !(dt > 0)) {
    g_err = "hw2d_directional_influx: invalid arguments";
    return 1;
  }
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) {
    g_err = "hw2d_directional_influx: cannot select the CUDA device";
    return 1;
  }
  const size_t nsig = (size_t)nt * nlines;
  double *d_in = nullptr, *d_tab = nullptr, *d_out = nullptr;
  cudaError_t e = cudaMalloc(&d_in, sizeof(double) * (5 * (size_t)nc + nlines + nt + nlines));
  if (e == cudaSuccess) e = cudaMalloc(&d_tab, sizeof(double) * 6 * (size_t)nc);
  if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(double) * 2 * nsig);
  double* d_a = d_in;
  double* d_w = d_a + nc;
  double* d_k = d_w + nc;
  double* d_th = d_k + nc;
  double* d_ph = d_th + nc;
  double* d_y = d_ph + nc;
  double* d_rt = d_y + nlines;
  double* d_ry = d_rt + nt;
  const struct { double* dst; const double* src; size_t n; } up[] = {
      {d_a, a, (size_t)nc}, {d_w, w, (size_t)nc}, {d_k, k, (size_t)nc}, {d_th, theta, (size_t)nc},
      {d_ph, phi, (size_t)nc}, {d_y, y, (size_t)nlines}, {d_rt, ramp_t, (size_t)nt}, {d_ry, ramp_y, (size_t)nlines}};
  for (const auto& u : up)
    if (e == cudaSuccess) e = cudaMemcpy(u.dst, u.src, sizeof(double) * u.n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_component_table<<<(nc + 255) / 256, 256>>>(nc, d_a, d_w, d_k, d_th, d_ph, mdir, dt, d_tab);
    const int per_block = kThreads * kSamplesPerThread;
    k_line_signal<<<dim3((nt + per_block - 1) / per_block, nlines), kThreads>>>(nt, t0, dt, d_y, y0, nc, d_tab, d_rt,
                                                                                d_ry, d_out, d_out + nsig);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(eta, d_out, sizeof(double) * nsig, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(skew, d_out + nsig, sizeof(double) * nsig, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) g_err = std::string("hw2d_directional_influx: ") + cudaGetErrorString(e);
  cudaFree(d_in);
  cudaFree(d_tab);
  cudaFree(d_out);
  cudaSetDevice(prev);
  return e == cudaSuccess ? 0 : 1;
}

}  // extern "C"
