// hw_influx.cu -- seeded JONSWAP influx signals of many ensemble members in one
// launch (jonswap_influx, 1d/influx_lib.c:137-255, with fun_jonswap :137-181).
//
// One CTA per member: the spectrum on the Nt/2 lines of freqspace's grid (with
// the reference's integer exponent 5/4 == 1 and its phase off-by-one: line i+1
// takes phase[i], phase[0] = 0), the zeroth moment by the trapezoid rule, the
// Hermitian coefficient vector (the mirror writes last, as the reference's loop
// leaves it), the inverse DFT of length Nt (any length: a direct sum with exact
// twiddle arguments (j q mod Nt) / Nt), the start/end ramps and the normalisation
// to Hs / (4 sqrt(variance)).  The phases are the seeded splitmix64 stream that
// stands in for rand(): draw r is a function of seed + (r + 1) * golden, so every
// line's phase is computed independently.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/hawassi_b200.h"

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kG = 9.80665;   // 1d/header.h:27
constexpr int kThreads = 512;

struct JsDev {
  double T0, lenT, dt, Tp, Hs, gam, nTramp;
  unsigned long long seed;
  int Nt;
  long long off;      // offset of the member's samples in the concatenated buffers
};

__device__ __forceinline__ double splitmix_draw(unsigned long long seed, unsigned long long r) {
  unsigned long long z = seed + (r + 1ULL) * 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    red[32] = s;
  }
  __syncthreads();
  return red[32];
}

// freqspace (1d/functions.c:1173-1197) value at index i < N/2
__device__ __forceinline__ double freq_at(double len, int N, int i) {
  const double delta = 2 * kPi / len;
  const double fmin = -0.5 * 2 * kPi / (len / (N - 1));
  const double fmax = ((N / 2) * 2 == N) ? -fmin - delta : -fmin;
  const double d = (fmax - fmin) / (N - 1);
  return fmin + (N / 2 + i) * d;
}

__device__ __forceinline__ double js_line(const JsDev& p, int i) {
  if (i == 0) return 0.0;   // JS[0] is never set by the reference's loop (0 here)
  const double omgp = 2 * kPi / p.Tp;
  const double om = freq_at(p.lenT, p.Nt, i);
  const double sigma = om <= omgp ? 0.07 : 0.09;
  const double alpha = 0.0081, f_p = omgp / (2 * kPi);
  const double f = om / (2 * kPi);
  const double gp = exp(-0.5 * pow(((f / f_p - 1) / sigma), 2));
  return alpha * pow(kG, 2) * pow((2 * kPi), (-4)) * pow(f, (-5)) * exp(-(5 / 4) * pow((f / f_p), (-4))) *
         pow(p.gam, gp);
}

__global__ void __launch_bounds__(kThreads) k_jonswap(const JsDev* __restrict__ ps, double2* __restrict__ X,
                                                      double* __restrict__ js, double* __restrict__ out) {
  __shared__ double red[33];
  const JsDev p = ps[blockIdx.x];
  const int Nt = p.Nt, Nomg = Nt / 2;
  double2* Xm = X + p.off;
  double* jm = js + p.off;
  double* om = out + p.off;
  // spectrum and its zeroth moment (trapz, 1d/functions.c:1822)
  double part = 0.0;
  for (int i = threadIdx.x; i < Nomg; i += blockDim.x) {
    const double v = js_line(p, i);
    jm[i] = v;
    part += (i == 0 || i == Nomg - 1) ? v / 2 : v;
  }
  const double m0 = block_sum(part, red) * (freq_at(p.lenT, Nt, 1) - freq_at(p.lenT, Nt, 0));
  // coefficient vector: lines 1..Nomg, then their mirrors Nt-1-i (written last)
  for (int q = threadIdx.x; q < Nt; q += blockDim.x) {
    double2 v = make_double2(0.0, 0.0);
    int i = -1;
    bool mirror = false;
    if (q >= Nt - Nomg && q >= 1) { i = Nt - 1 - q; mirror = true; }
    else if (q >= 1 && q <= Nomg) i = q - 1;
    if (i >= 0) {
      const double spec = (pow(p.Hs, 2) / 16) * jm[i] / m0;
      const double ph = (i == 0) ? 0.0 : 2 * kPi * splitmix_draw(p.seed, (unsigned long long)(i - 1));
      const double re = (sqrt(spec) * cos(ph)) / p.dt * 2 * pow(kPi, 2);
      const double im = -(sqrt(spec) * sin(ph)) / p.dt * 2 * pow(kPi, 2);
      v = mirror ? make_double2(re, -im) : make_double2(re, im);
    }
    Xm[q] = v;
  }
  __syncthreads();
  // inverse DFT (real part over Nt), ramps, mean
  double msum = 0.0;
  for (int j = threadIdx.x; j < Nt; j += blockDim.x) {
    double acc = 0.0;
    unsigned long long r = 0;   // (j q) mod Nt, advanced by j per term
    for (int q = 0; q < Nt; ++q) {
      double s, c;
      sincospi(2.0 * (double)r / (double)Nt, &s, &c);
      const double2 x = Xm[q];
      acc += x.x * c - x.y * s;
      r += (unsigned long long)j;
      if (r >= (unsigned long long)Nt) r -= (unsigned long long)Nt;
    }
    const double raw = acc / Nt;
    auto ramp = [&](int jj) {
      const double tin = p.T0 + jj * p.dt;
      const double A = ((tin - p.T0) - p.nTramp * p.Tp);
      const double B1 = A / fabs(A);
      const double B2 = (1 - cos((tin - p.T0) * kPi / p.nTramp / p.Tp)) / 2;
      return B1 > B2 ? B1 : B2;
    };
    const double ins = ramp(j) * raw * ramp(Nt - 1 - j);
    om[j] = ins;
    msum += ins;
  }
  const double mean = block_sum(msum, red) / Nt;
  double vsum = 0.0;
  for (int j = threadIdx.x; j < Nt; j += blockDim.x) vsum += pow(om[j] - mean, 2);
  const double var = block_sum(vsum, red) / Nt;
  for (int j = threadIdx.x; j < Nt; j += blockDim.x) om[j] = om[j] * p.Hs / (4 * sqrt(var));
}

}  // namespace

extern "C" int hw_jonswap_influx(const hw_jonswap* specs, int n, double* eta_out, long long cap, int device) {
  if (!specs || n <= 0) return -1;
  std::vector<JsDev> ps((size_t)n);
  long long total = 0;
  for (int m = 0; m < n; ++m) {
    const hw_jonswap& s = specs[m];
    JsDev& d = ps[(size_t)m];
    d.T0 = s.T0; d.lenT = s.Tend - s.T0; d.dt = s.dt; d.Tp = s.Tp; d.Hs = s.Hs; d.gam = s.gamma;
    d.nTramp = s.nTramp; d.seed = s.seed;
    d.Nt = (int)((d.lenT) / d.dt + 1);   // 1d/influx_lib.c:83
    if (!(d.dt > 0) || d.Nt < 4 || d.Nt > (1 << 22)) return -1;
    d.off = total;
    total += d.Nt;
  }
  if (total > 0x7fffffffLL) return -1;   // the count must fit the return value
  if (!eta_out || cap < total) return (int)total;
  if (cudaSetDevice(device) != cudaSuccess) return -1;
  JsDev* dps = nullptr;
  double2* X = nullptr;
  double *js = nullptr, *out = nullptr;
  bool ok = cudaMalloc(&dps, sizeof(JsDev) * (size_t)n) == cudaSuccess &&
            cudaMalloc(&X, sizeof(double2) * (size_t)total) == cudaSuccess &&
            cudaMalloc(&js, sizeof(double) * (size_t)total) == cudaSuccess &&
            cudaMalloc(&out, sizeof(double) * (size_t)total) == cudaSuccess;
  ok = ok && cudaMemcpy(dps, ps.data(), sizeof(JsDev) * (size_t)n, cudaMemcpyHostToDevice) == cudaSuccess;
  if (ok) {
    k_jonswap<<<n, kThreads>>>(dps, X, js, out);
    ok = cudaGetLastError() == cudaSuccess &&
         cudaMemcpy(eta_out, out, sizeof(double) * (size_t)total, cudaMemcpyDeviceToHost) == cudaSuccess;
  }
  cudaFree(dps);
  cudaFree(X);
  cudaFree(js);
  cudaFree(out);
  return ok ? (int)total : -1;
}
