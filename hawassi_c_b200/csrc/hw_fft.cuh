// hw_fft.cuh -- FP64 complex FFT of one member's grid, distributed over the C
// CTAs of a thread-block cluster.  Each CTA owns a slice of M = N / C points in
// shared memory (T = M / 8 threads, 8 points per thread).
//
// Layouts (index i within the CTA of cluster rank c):
//   physical ("block"):  global grid index n = c*M + i
//   spectral ("cyclic"): global wavenumber index kk = c + C*i
// Forward transform (block -> cyclic) is a decimation-in-frequency four-step:
// a C-point DFT across the cluster (read from the peers' shared memory through
// DSMEM) times the twiddle W_N^(i*c), then a local M-point Stockham FFT.  The
// inverse (cyclic -> block) is the transpose: local M-point inverse FFT, then
// the twiddle and the C-point DFT across the cluster.  With C == 1 the cross
// step vanishes.  Sign convention and scaling follow FFTW (unnormalised,
// forward exponent -1).
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

namespace hwdev {

namespace cg = cooperative_groups;

constexpr int kPts = 8;  // points per thread

// bank swizzle: position i of a slice is stored at i with its low three bits XORed
// by bits 3-5 (a permutation inside each group of 8 double2 = 128 bytes = all 32
// banks), which keeps the stride-8 stores of the first Stockham pass conflict-free
// while unit-stride accesses stay conflict-free; unlike a pad slot per 8 points it
// costs no shared memory, which the SM gives to L1 instead
__device__ __forceinline__ int pidx(int i) { return i ^ ((i >> 3) & 7); }
__host__ __device__ constexpr int padded(int m) { return m; }

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// twiddle exp(sign * 2 pi i q / N) from the table tw[q] = exp(-2 pi i q / N)
__device__ __forceinline__ double2 twd(const double2* __restrict__ tw, int q, int sign) {
  double2 w = __ldg(tw + q);
  return sign > 0 ? make_double2(w.x, -w.y) : w;
}

// multiply by exp(sign * i pi / 2) = sign * i
__device__ __forceinline__ double2 mul_pm_i(double2 a, int sign) {
  return sign > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

template <int R>
__device__ __forceinline__ void dft_small(double2* v, int sign);

template <>
__device__ __forceinline__ void dft_small<2>(double2* v, int) {
  double2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <>
__device__ __forceinline__ void dft_small<4>(double2* v, int sign) {
  double2 d0 = cadd(v[0], v[2]), d2 = csub(v[0], v[2]);
  double2 d1 = cadd(v[1], v[3]), d3 = mul_pm_i(csub(v[1], v[3]), sign);
  v[0] = cadd(d0, d1);
  v[2] = csub(d0, d1);
  v[1] = cadd(d2, d3);
  v[3] = csub(d2, d3);
}

template <>
__device__ __forceinline__ void dft_small<8>(double2* v, int sign) {
  const double r = 0.70710678118654752440084436210485;  // sqrt(1/2)
  double2 b[8];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    b[i] = cadd(v[i], v[i + 4]);
    b[i + 4] = csub(v[i], v[i + 4]);
  }
  // b5 *= w^1, b6 *= w^2, b7 *= w^3 with w = exp(sign * 2 pi i / 8)
  {
    double2 a = b[5];
    b[5] = make_double2(r * (a.x - sign * a.y), r * (a.y + sign * a.x));
    b[6] = mul_pm_i(b[6], sign);
    a = b[7];
    b[7] = make_double2(r * (-a.x - sign * a.y), r * (-a.y + sign * a.x));
  }
  double2 e[4] = {b[0], b[1], b[2], b[3]}, o[4] = {b[4], b[5], b[6], b[7]};
  dft_small<4>(e, sign);
  dft_small<4>(o, sign);
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    v[2 * m] = e[m];
    v[2 * m + 1] = o[m];
  }
}


// w^1..w^(R-1) from w^1: one table load per butterfly, powers by short products
// (w^2 = w w, w^3 = w^2 w, w^4 = w^2 w^2, w^5 = w^4 w, w^6 = w^4 w^2, w^7 = w^4 w^3)
template <int R>
__device__ __forceinline__ void twiddle_powers(double2 w1, double2* w) {
  w[1] = w1;
  if constexpr (R > 2) {
    w[2] = cmul(w1, w1);
    w[3] = cmul(w[2], w1);
  }
  if constexpr (R > 4) {
    w[4] = cmul(w[2], w[2]);
    w[5] = cmul(w[4], w1);
    w[6] = cmul(w[4], w[2]);
    w[7] = cmul(w[4], w[3]);
  }
}

// One in-place Stockham radix-R pass over the M-point slice in shared memory.
// tw_stride converts an index in units of 1/M of a turn to the N-point table.
template <int M, int R>
__device__ __forceinline__ void stockham_pass(double2* buf, int Ns, const double2* __restrict__ tw,
                                              int tw_stride, int sign) {
  constexpr int T = M / kPts;
  constexpr int NB = M / R;
  constexpr int BPT = kPts / R;
  double2 v[BPT][R];
  const int tid = threadIdx.x;
#pragma unroll
  for (int u = 0; u < BPT; ++u) {
    const int j = tid + u * T;
#pragma unroll
    for (int r = 0; r < R; ++r) v[u][r] = buf[pidx(j + r * NB)];
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < BPT; ++u) {
    const int j = tid + u * T;
    const int jm = j & (Ns - 1);
    if (Ns > 1) {
      const int qb = jm * (M / (Ns * R));
      double2 w[R];
      twiddle_powers<R>(twd(tw, qb * tw_stride, sign), w);
#pragma unroll
      for (int r = 1; r < R; ++r) v[u][r] = cmul(v[u][r], w[r]);
    }
    dft_small<R>(v[u], sign);
    const int idxD = (j - jm) * R + jm;
#pragma unroll
    for (int r = 0; r < R; ++r) buf[pidx(idxD + r * Ns)] = v[u][r];
  }
  __syncthreads();
}

// Local M-point FFT, natural order in and out.
template <int M>
__device__ __forceinline__ void local_fft(double2* buf, const double2* __restrict__ tw, int tw_stride, int sign) {
  int Ns = 1;
  constexpr int L8 = (M >= 512) ? 3 : (M >= 64 ? 2 : 1);
  // radix-8 passes while they divide, then one radix-4 or radix-2 pass
  constexpr int rem = M / (1 << (3 * L8));
#pragma unroll
  for (int p = 0; p < L8; ++p) {
    stockham_pass<M, 8>(buf, Ns, tw, tw_stride, sign);
    Ns *= 8;
  }
  if constexpr (rem == 8) {
    stockham_pass<M, 8>(buf, Ns, tw, tw_stride, sign);
  } else if constexpr (rem == 4) {
    stockham_pass<M, 4>(buf, Ns, tw, tw_stride, sign);
  } else if constexpr (rem == 2) {
    stockham_pass<M, 2>(buf, Ns, tw, tw_stride, sign);
  }
}


// Cross-CTA step of the distributed transform, as gather / C-point DFT / scatter:
// the M positions of the slice are shared out over the C*T threads of the cluster;
// the thread owning position i gathers the C values at i from every CTA's slice,
// applies the C-point DFT (forward: then the twiddles W_N^(i k1); inverse: the
// twiddles W_N^-(i k1) first) and stores output j into CTA j's slice at i.
// Every position is owned by exactly one thread of the cluster, which reads and
// then rewrites it in every CTA, so the scatter needs no barrier after the gather:
// one cluster barrier before (the slices are complete) and one after.
template <int M, int C, int NBUF>
__device__ __forceinline__ void cross_gs(double2* A, double2* B, const double2* __restrict__ tw, int c, int sign) {
  constexpr int T = M / kPts;
  constexpr int PER = kPts / C;   // positions per thread
  cg::cluster_group cl = cg::this_cluster();
  double2 va[PER][C], vb[PER][C];
  cl.sync();
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int i = c * T + threadIdx.x + q * (C * T);
#pragma unroll
    for (int r = 0; r < C; ++r) {
      va[q][r] = cl.map_shared_rank(A, r)[pidx(i)];
      if constexpr (NBUF == 2) vb[q][r] = cl.map_shared_rank(B, r)[pidx(i)];
    }
  }
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int i = c * T + threadIdx.x + q * (C * T);
    double2 w[C > 1 ? C : 2];
    if (sign > 0) {   // inverse: twiddle by W_N^(+i k1) before the DFT over k1
      twiddle_powers<C>(twd(tw, i, +1), w);
#pragma unroll
      for (int r = 1; r < C; ++r) {
        va[q][r] = cmul(va[q][r], w[r]);
        if constexpr (NBUF == 2) vb[q][r] = cmul(vb[q][r], w[r]);
      }
    }
    dft_small<C>(va[q], sign);
    if constexpr (NBUF == 2) dft_small<C>(vb[q], sign);
    if (sign < 0) {   // forward: output k1 gets W_N^(-i k1)
      twiddle_powers<C>(twd(tw, i, -1), w);
#pragma unroll
      for (int r = 1; r < C; ++r) {
        va[q][r] = cmul(va[q][r], w[r]);
        if constexpr (NBUF == 2) vb[q][r] = cmul(vb[q][r], w[r]);
      }
    }
#pragma unroll
    for (int r = 0; r < C; ++r) {
      cl.map_shared_rank(A, r)[pidx(i)] = va[q][r];
      if constexpr (NBUF == 2) cl.map_shared_rank(B, r)[pidx(i)] = vb[q][r];
    }
  }
  cl.sync();
}

// dispatch on the cluster size (2, 4, 8); returns false for other sizes
template <int M, int NBUF>
__device__ __forceinline__ bool cross_fast(double2* A, double2* B, const double2* __restrict__ tw, int C, int c,
                                           int sign) {
  if (C == 2) { cross_gs<M, 2, NBUF>(A, B, tw, c, sign); return true; }
  if (C == 4) { cross_gs<M, 4, NBUF>(A, B, tw, c, sign); return true; }
  if (C == 8) { cross_gs<M, 8, NBUF>(A, B, tw, c, sign); return true; }
  return false;
}

// cluster-wide barrier (block barrier when the member is a single CTA)
__device__ __forceinline__ void member_sync(int C) {
  if (C > 1) cg::this_cluster().sync();
  else __syncthreads();
}

// Forward FFT: physical block slice in buf -> spectral cyclic slice in buf.
template <int M>
__device__ __noinline__ void fft_forward(double2* buf, const double2* __restrict__ tw, int N, int C, int c) {
  if (C == 1) __syncthreads();
  if (C > 1 && cross_fast<M, 1>(buf, buf, tw, C, c, -1)) {
    local_fft<M>(buf, tw, C, -1);
    return;
  }
  if (C > 1) {
    constexpr int T = M / kPts;
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    double2 acc[kPts];
    const int NC = N / C;
#pragma unroll
    for (int u = 0; u < kPts; ++u) {
      const int i = threadIdx.x + u * T;
      double2 s = make_double2(0.0, 0.0);
      for (int n1 = 0; n1 < C; ++n1) {
        const double2* pb = cl.map_shared_rank(buf, n1);
        double2 x = pb[pidx(i)];
        s = cadd(s, cmul(x, twd(tw, ((n1 * c) % C) * NC, -1)));
      }
      acc[u] = cmul(s, twd(tw, i * c, -1));
    }
    cl.sync();
#pragma unroll
    for (int u = 0; u < kPts; ++u) buf[pidx(threadIdx.x + u * T)] = acc[u];
    __syncthreads();
  }
  local_fft<M>(buf, tw, C, -1);
}

// Inverse FFT (unnormalised): spectral cyclic slice in buf -> physical block slice in buf.
template <int M>
__device__ __noinline__ void fft_inverse(double2* buf, const double2* __restrict__ tw, int N, int C, int c) {
  __syncthreads();
  local_fft<M>(buf, tw, C, +1);
  if (C > 1 && cross_fast<M, 1>(buf, buf, tw, C, c, +1)) {
    __syncthreads();
    return;
  }
  if (C > 1) {
    constexpr int T = M / kPts;
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    double2 acc[kPts];
    const int NC = N / C;
#pragma unroll
    for (int u = 0; u < kPts; ++u) {
      const int i = threadIdx.x + u * T;
      double2 s = make_double2(0.0, 0.0);
      for (int k1 = 0; k1 < C; ++k1) {
        const double2* pb = cl.map_shared_rank(buf, k1);
        double2 z = cmul(pb[pidx(i)], twd(tw, i * k1, +1));
        s = cadd(s, cmul(z, twd(tw, ((c * k1) % C) * NC, +1)));
      }
      acc[u] = s;
    }
    cl.sync();
#pragma unroll
    for (int u = 0; u < kPts; ++u) buf[pidx(threadIdx.x + u * T)] = acc[u];
    __syncthreads();
  }
}

}  // namespace hwdev

namespace hwdev {

// ---------------------------------------------------------------------------
// Dual transforms: two M-point slices (A and B) in one sweep -- twice the
// independent work per thread, one set of twiddle loads and barriers for both.
// ---------------------------------------------------------------------------
template <int M, int R>
__device__ __forceinline__ void stockham_pass2(double2* A, double2* B, int Ns, const double2* __restrict__ tw,
                                               int tw_stride, int sign) {
  constexpr int T = M / kPts;
  constexpr int NB = M / R;
  constexpr int BPT = kPts / R;
  double2 va[BPT][R], vb[BPT][R];
  const int tid = threadIdx.x;
#pragma unroll
  for (int u = 0; u < BPT; ++u) {
    const int j = tid + u * T;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      va[u][r] = A[pidx(j + r * NB)];
      vb[u][r] = B[pidx(j + r * NB)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < BPT; ++u) {
    const int j = tid + u * T;
    const int jm = j & (Ns - 1);
    if (Ns > 1) {
      const int qb = jm * (M / (Ns * R));
      double2 w[R];
      twiddle_powers<R>(twd(tw, qb * tw_stride, sign), w);
#pragma unroll
      for (int r = 1; r < R; ++r) {
        va[u][r] = cmul(va[u][r], w[r]);
        vb[u][r] = cmul(vb[u][r], w[r]);
      }
    }
    dft_small<R>(va[u], sign);
    dft_small<R>(vb[u], sign);
    const int idxD = (j - jm) * R + jm;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      A[pidx(idxD + r * Ns)] = va[u][r];
      B[pidx(idxD + r * Ns)] = vb[u][r];
    }
  }
  __syncthreads();
}

template <int M>
__device__ __forceinline__ void local_fft2(double2* A, double2* B, const double2* __restrict__ tw, int tw_stride,
                                           int sign) {
  int Ns = 1;
  constexpr int L8 = (M >= 512) ? 3 : (M >= 64 ? 2 : 1);
  constexpr int rem = M / (1 << (3 * L8));
#pragma unroll
  for (int p = 0; p < L8; ++p) {
    stockham_pass2<M, 8>(A, B, Ns, tw, tw_stride, sign);
    Ns *= 8;
  }
  if constexpr (rem == 8) {
    stockham_pass2<M, 8>(A, B, Ns, tw, tw_stride, sign);
  } else if constexpr (rem == 4) {
    stockham_pass2<M, 4>(A, B, Ns, tw, tw_stride, sign);
  } else if constexpr (rem == 2) {
    stockham_pass2<M, 2>(A, B, Ns, tw, tw_stride, sign);
  }
}

// cross-CTA step of the distributed transform for both slices (see fft_forward /
// fft_inverse): forward = C-point DFT then twiddle, inverse = twiddle then DFT.
template <int M>
__device__ __forceinline__ void cross_step2(double2* A, double2* B, const double2* __restrict__ tw, int N, int C,
                                            int c, int sign) {
  constexpr int T = M / kPts;
  cg::cluster_group cl = cg::this_cluster();
  cl.sync();
  double2 sa[kPts], sb[kPts];
  const int NC = N / C;
#pragma unroll
  for (int u = 0; u < kPts; ++u) {
    const int i = threadIdx.x + u * T;
    double2 a = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0);
    for (int r = 0; r < C; ++r) {
      const double2* pa = cl.map_shared_rank(A, r);
      const double2* pb = cl.map_shared_rank(B, r);
      double2 xa = pa[pidx(i)], xb = pb[pidx(i)];
      if (sign > 0) {   // inverse: peer r is the spectral class k1 = r
        const double2 w = twd(tw, i * r, +1);
        xa = cmul(xa, w);
        xb = cmul(xb, w);
      }
      const double2 wc = twd(tw, ((r * c) % C) * NC, sign);
      a = cadd(a, cmul(xa, wc));
      b = cadd(b, cmul(xb, wc));
    }
    if (sign < 0) {
      const double2 w = twd(tw, i * c, -1);
      a = cmul(a, w);
      b = cmul(b, w);
    }
    sa[u] = a;
    sb[u] = b;
  }
  cl.sync();
#pragma unroll
  for (int u = 0; u < kPts; ++u) {
    A[pidx(threadIdx.x + u * T)] = sa[u];
    B[pidx(threadIdx.x + u * T)] = sb[u];
  }
  __syncthreads();
}

template <int M>
__device__ __noinline__ void fft_forward2(double2* A, double2* B, const double2* __restrict__ tw, int N, int C,
                                          int c) {
  __syncthreads();
  if (C > 1 && !cross_fast<M, 2>(A, B, tw, C, c, -1)) cross_step2<M>(A, B, tw, N, C, c, -1);
  local_fft2<M>(A, B, tw, C, -1);
}

template <int M>
__device__ __noinline__ void fft_inverse2(double2* A, double2* B, const double2* __restrict__ tw, int N, int C,
                                          int c) {
  __syncthreads();
  local_fft2<M>(A, B, tw, C, +1);
  if (C > 1) {
    if (!cross_fast<M, 2>(A, B, tw, C, c, +1)) cross_step2<M>(A, B, tw, N, C, c, +1);
    __syncthreads();
  }
}

// The local (in-CTA) part of a distributed transform alone, for callers that do the
// cross-CTA step themselves: sign +1 is the inverse's first half, -1 the forward's
// second half.  Barrier on entry (the caller wrote the slices) and on exit.
template <int M>
__device__ __noinline__ void fft_local(double2* A, const double2* __restrict__ tw, int C, int sign) {
  __syncthreads();
  local_fft<M>(A, tw, C, sign);
}
template <int M>
__device__ __noinline__ void fft_local2(double2* A, double2* B, const double2* __restrict__ tw, int C, int sign) {
  __syncthreads();
  local_fft2<M>(A, B, tw, C, sign);
}

}  // namespace hwdev
