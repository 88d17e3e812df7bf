// hw_rhs.cuh -- the pseudo-spectral Hamiltonian RHS of one member, executed by
// the CTAs of one thread-block cluster (or one CTA).  Each FFT transforms two
// real signals at once (Hermitian packing / splitting), so the HS2 RHS takes
// 7 complex transforms where the reference takes 12 (1d/rhs.c:96-241), and the
// varying-depth operator HSS with K reference depths takes ceil(K/2)+K
// transforms where the reference takes 3K+1 (1d/functions.c:2861-2977).
// Intermediate fields live in per-member global scratch (L2 resident).
#pragma once

#include "hw_device.cuh"

namespace hwdev {

// Fehlberg coefficients (GSL rkf45)
__device__ constexpr double RK_ah[5] = {1.0 / 4.0, 3.0 / 8.0, 12.0 / 13.0, 1.0, 1.0 / 2.0};
__device__ constexpr double RK_b3[2] = {3.0 / 32.0, 9.0 / 32.0};
__device__ constexpr double RK_b4[3] = {1932.0 / 2197.0, -7200.0 / 2197.0, 7296.0 / 2197.0};
__device__ constexpr double RK_b5[4] = {8341.0 / 4104.0, -32832.0 / 4104.0, 29440.0 / 4104.0, -845.0 / 4104.0};
__device__ constexpr double RK_b6[5] = {-6080.0 / 20520.0, 41040.0 / 20520.0, -28352.0 / 20520.0, 9295.0 / 20520.0,
                                        -5643.0 / 20520.0};
__device__ constexpr double RK_c1 = 902880.0 / 7618050.0;
__device__ constexpr double RK_c3 = 3953664.0 / 7618050.0;
__device__ constexpr double RK_c4 = 3855735.0 / 7618050.0;
__device__ constexpr double RK_c5 = -1371249.0 / 7618050.0;
__device__ constexpr double RK_c6 = 277020.0 / 7618050.0;
__device__ constexpr double RK_ec1 = 1.0 / 360.0;
__device__ constexpr double RK_ec3 = -128.0 / 4275.0;
__device__ constexpr double RK_ec4 = -2197.0 / 75240.0;
__device__ constexpr double RK_ec5 = 1.0 / 50.0;
__device__ constexpr double RK_ec6 = 2.0 / 55.0;

// the stage input of an RK stage: zs = y + h sum_j b_sj k_j (s = 2..6), or zs = y
// itself (s = 1: the state a first or last derivative is evaluated at)
struct StageSrc {
  const double2* y;
  const double2* k[5];
  int s;
  double h;
};

// IEEE products and sums without fused multiply-add: the stepper's arithmetic
// rounds like GSL's (compiled without contraction)
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }

// one element of the stage input, in GSL rkf45's expression forms
__device__ __forceinline__ double2 stage_val(const StageSrc& st, int q) {
  if (st.s == 1) return st.y[q];
  const double2 y = st.y[q], a = st.k[0][q];
  const double h = st.h;
  if (st.s == 2) {
    const double f = rmul(RK_ah[0], h);
    return make_double2(radd(y.x, rmul(f, a.x)), radd(y.y, rmul(f, a.y)));
  }
  const double2 b = st.k[1][q];
  if (st.s == 3)
    return make_double2(radd(y.x, rmul(h, radd(rmul(RK_b3[0], a.x), rmul(RK_b3[1], b.x)))),
                        radd(y.y, rmul(h, radd(rmul(RK_b3[0], a.y), rmul(RK_b3[1], b.y)))));
  const double2 c3 = st.k[2][q];
  if (st.s == 4)
    return make_double2(
        radd(y.x, rmul(h, radd(radd(rmul(RK_b4[0], a.x), rmul(RK_b4[1], b.x)), rmul(RK_b4[2], c3.x)))),
        radd(y.y, rmul(h, radd(radd(rmul(RK_b4[0], a.y), rmul(RK_b4[1], b.y)), rmul(RK_b4[2], c3.y)))));
  const double2 c4 = st.k[3][q];
  if (st.s == 5)
    return make_double2(
        radd(y.x, rmul(h, radd(radd(radd(rmul(RK_b5[0], a.x), rmul(RK_b5[1], b.x)), rmul(RK_b5[2], c3.x)),
                               rmul(RK_b5[3], c4.x)))),
        radd(y.y, rmul(h, radd(radd(radd(rmul(RK_b5[0], a.y), rmul(RK_b5[1], b.y)), rmul(RK_b5[2], c3.y)),
                               rmul(RK_b5[3], c4.y)))));
  const double2 c5 = st.k[4][q];
  return make_double2(
      radd(y.x, rmul(h, radd(radd(radd(radd(rmul(RK_b6[0], a.x), rmul(RK_b6[1], b.x)), rmul(RK_b6[2], c3.x)),
                                  rmul(RK_b6[3], c4.x)),
                             rmul(RK_b6[4], c5.x)))),
      radd(y.y, rmul(h, radd(radd(radd(radd(rmul(RK_b6[0], a.y), rmul(RK_b6[1], b.y)), rmul(RK_b6[2], c3.y)),
                                  rmul(RK_b6[3], c4.y)),
                             rmul(RK_b6[4], c5.y)))));
}

template <int M>
struct Ctx {
  static constexpr int T = M / kPts;
  const DevMember& d;
  double2* buf;   // M-point FFT slice (padded) in shared memory
  double2* buf2;  // second slice for the dual transforms
  double* red;    // reduction scratch in shared memory
  int c;          // rank of this CTA in the member's cluster
  int tid;
  const StageSrc* stg = nullptr;   // set: zs is to be formed from y and the k's first
};

// dynamic shared memory of the 1D kernels of slice M: two padded FFT slices (no more:
// what the SM does not give to shared memory serves as L1 cache)
__host__ __device__ constexpr size_t slice_smem_bytes(int m) { return 2 * size_t(padded(m)) * sizeof(double2); }

template <int M>
__device__ __forceinline__ Ctx<M> make_ctx(const DevMember& d, double2* smem, double* red, int rank) {
  return Ctx<M>{d, smem, smem + padded(M), red, rank, int(threadIdx.x)};
}

#define HW_FOREACH(X)                            \
  _Pragma("unroll") for (int u = 0; u < kPts; ++u)  \
    if (const int idx = (X).tid + u * Ctx<M>::T, p = (X).c * M + idx; true)

// permuted position of the wavenumber N - kk, for the spectral entry at slice index idx
template <int M>
__device__ __forceinline__ int partner_pos(const Ctx<M>& X, int idx) {
  const DevMember& d = X.d;
  const int kk = X.c + (idx << d.logC);
  const int kp = (d.N - kk) & (d.N - 1);
  return (kp & (d.C - 1)) * M + (kp >> d.logC);
}

// Hermitian part (A[k] + conj A[N-k]) / 2: the spectrum whose inverse transform is
// the real part of the inverse transform of A (the reference keeps only the real part).
__device__ __forceinline__ double2 herm(double2 a, double2 ap) {
  return make_double2(0.5 * (a.x + ap.x), 0.5 * (a.y - ap.y));
}
// (A + i B) * s
__device__ __forceinline__ double2 pack(double2 a, double2 b, double s) {
  return make_double2((a.x - b.y) * s, (a.y + b.x) * s);
}
// spectra of the real and imaginary input parts from Z = FFT(a + i b)
__device__ __forceinline__ double2 split_re(double2 z, double2 zp) {
  return make_double2(0.5 * (z.x + zp.x), 0.5 * (z.y - zp.y));
}
__device__ __forceinline__ double2 split_im(double2 z, double2 zp) {
  return make_double2(0.5 * (z.y + zp.y), -0.5 * (z.x - zp.x));
}
// prod_1ik (1d/functions.c:297): (i a) * B
__device__ __forceinline__ double2 mul_ik(double a, double2 b) {
  return make_double2((0.0 * b.x) - (a * b.y), (0.0 * b.y) + (a * b.x));
}

// forward FFT of the physical slice in buf, then f(u, idx, p, Z, Zpartner) for each
// of this thread's spectral points (Zpartner read from the owning CTA by DSMEM)
template <int M, class F>
__device__ __forceinline__ void fft_forward_split(Ctx<M>& X, F&& f) {
  const DevMember& d = X.d;
  fft_forward<M>(X.buf, d.tw, d.N, d.C, X.c);
  const double2* pb = X.buf;
  if (d.C > 1) {
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    pb = cl.map_shared_rank(X.buf, (d.C - X.c) & (d.C - 1));
  }
  double2 Z[kPts], Zp[kPts];
  HW_FOREACH(X) {
    (void)p;
    Z[u] = X.buf[pidx(idx)];
    const int jp = X.c == 0 ? ((M - idx) & (M - 1)) : (M - 1 - idx);
    Zp[u] = pb[pidx(jp)];
  }
  member_sync(d.C);
  HW_FOREACH(X) { f(u, idx, p, Z[u], Zp[u]); }
}

// inverse FFT of the spectral slice in buf; g(u, idx, p, v) for each physical point
template <int M, class G>
__device__ __forceinline__ void fft_inverse_then(Ctx<M>& X, G&& g) {
  const DevMember& d = X.d;
  fft_inverse<M>(X.buf, d.tw, d.N, d.C, X.c);
  HW_FOREACH(X) { g(u, idx, p, X.buf[pidx(idx)]); }
}

// natural cubic spline evaluation (GSL cspline + bsearch index rule)
__device__ __forceinline__ double spline_eval(const double* __restrict__ x, const double* __restrict__ y,
                                              const double* __restrict__ c, int n, double t) {
  if (!(t >= x[0] && t <= x[n - 1])) return __longlong_as_double(0x7ff8000000000000ULL);
  const double h0 = x[1] - x[0];
  int lo = int((t - x[0]) / h0);
  lo = lo < 0 ? 0 : (lo > n - 2 ? n - 2 : lo);
  while (lo > 0 && x[lo] > t) --lo;
  while (lo < n - 2 && x[lo + 1] <= t) ++lo;
  const double xl = x[lo], h = x[lo + 1] - xl, dy = y[lo + 1] - y[lo], delx = t - xl;
  const double ci = c[lo], cp = c[lo + 1];
  const double b = dy / h - h * (cp + 2.0 * ci) / 3.0;
  const double dd = (cp - ci) / (3.0 * h);
  return y[lo] + delx * (b + delx * (ci + delx * dd));
}

// HSS (1d/functions.c:2861): out = 1/2 sum_j [ F(gam_j Re F^-1(Csq_j A)) + Csq_j F(gam_j a) ]
// with a = Re F^-1(A) supplied in physical space as aphys[2 p] (one component of a double2 field).  Reference depths are
// paired in the inverse transforms and gam_j s_j / gam_j a share one forward transform.
template <int M>
__device__ __noinline__ void hss(Ctx<M>& X, const double2* __restrict__ A, const double* __restrict__ aphys,
                                 double2* out, double2* ps) {
  const DevMember& d = X.d;
  const int N = d.N, K = d.nref;
  for (int j = 0; j < K; j += 2) {
    const double* C0 = d.Csq + size_t(j) * N;
    const double* C1 = (j + 1 < K) ? d.Csq + size_t(j + 1) * N : nullptr;
    HW_FOREACH(X) {
      const int pp = partner_pos(X, idx);
      const double2 a = A[p], ap = A[pp];
      const double2 s0 = herm(cscale(a, C0[p]), cscale(ap, C0[pp]));
      const double2 s1 = C1 ? herm(cscale(a, C1[p]), cscale(ap, C1[pp])) : make_double2(0.0, 0.0);
      X.buf[pidx(idx)] = pack(s0, s1, d.invN);
    }
    fft_inverse_then(X, [&](int, int, int p, double2 v) { ps[p] = v; });
    for (int jj = j; jj < j + 2 && jj < K; ++jj) {
      const double* g = d.gam + size_t(jj) * N;
      const double* Cj = d.Csq + size_t(jj) * N;
      HW_FOREACH(X) {
        const double s = (jj == j) ? ps[p].x : ps[p].y;
        const double gm = g[p];
        X.buf[pidx(idx)] = make_double2(gm * s, gm * aphys[2 * p]);
      }
      const bool first = (jj == 0);
      fft_forward_split(X, [&](int, int, int p, double2 z, double2 zp) {
        const double2 f1 = split_re(z, zp), f2 = split_im(z, zp);
        const double cj = Cj[p];
        const double2 v = make_double2(0.5 * (f1.x + cj * f2.x), 0.5 * (f1.y + cj * f2.y));
        out[p] = first ? v : cadd(out[p], v);
      });
    }
  }
}

// breaking hooks (implemented in hw_breaking.cuh)
template <int M>
__device__ __noinline__ bool breaking_rhs(Ctx<M>& X, double t, const double2* PE, const double* Heta, int heta_stride,
                             const double2* AEadj, double2* Rb);
template <int M>
__device__ __forceinline__ void breaking_reset(Ctx<M>& X);
template <int M>
__device__ __forceinline__ void breaking_scan(Ctx<M>& X, const double2* PE, const double* Heta, int hs);
template <int M>
__device__ __forceinline__ void breaking_lead(Ctx<M>& X, double t, const double2* PE, const double* Heta, int hs);
template <int M>
__device__ __noinline__ void breaking_force(Ctx<M>& X, const double2* PE, const double2* AEadj, double2* Rb);
// HS2 flat-bottom fast path (hw_rhs_fast.cuh)
template <int M>
__device__ __noinline__ void rhs_hs2_flat(Ctx<M>& X, double t, double2* __restrict__ dz);

// One RHS evaluation dz = f(t, zs), zs = [eta^ | u^] (permuted spectral, 2N).
template <int M>
__device__ __noinline__ void rhs_eval(Ctx<M>& X, double t, double2* __restrict__ dz) {
  const DevMember& d = X.d;
  const int N = d.N;
  const double2* z = d.zs;
  const double2* ZE = z;
  const double2* ZU = z + N;
  double2* PE = d.sc[0];   // physical (eta, u)
  double2* PM = d.sc[1];   // physical (M0 u, Hilbert eta | d_x u)
  double2* AE = d.sc[2];   // spectral eta-equation nonlinear terms, then adjusted
  double2* AU = d.sc[3];   // spectral u-equation nonlinear terms, then adjusted
  double2* DE = d.sc[4];   // FFT(damping eta)
  double2* DU = d.sc[5];   // FFT(damping u)
  double2* HS = d.sc[6];   // HSS(u^) for varying depth
  double2* PA = d.sc[7];   // physical scratch
  double2* PS = d.sc[8];   // physical scratch for HSS
  double2* S9 = d.sc[9];   // spectral scratch
  double2* S10 = d.sc[10]; // spectral scratch
  double2* RB = d.sc[11];  // FFT(breaking force)
  const bool hs2 = d.model >= 2, hs3 = d.model == 3, brk = d.brk != 0, flat = d.flat != 0;
  bool rb_live = false;   // the breaking force is nonzero (some node broke)
  if (d.model == 2 && flat) {
    rhs_hs2_flat<M>(X, t, dz);
    return;
  }
  if (X.stg) {
    for (int part = 0; part < 2; ++part) {
      const int off = part * N;
      HW_FOREACH(X) {
        (void)idx;
        d.zs[p + off] = stage_val(*X.stg, p + off);
      }
    }
  }

  member_sync(d.C);   // zs written by all CTAs of the member

  // (1) eta, u = Re F^-1(eta^), Re F^-1(u^)
  HW_FOREACH(X) {
    const int pp = partner_pos(X, idx);
    X.buf[pidx(idx)] = pack(herm(ZE[p], ZE[pp]), herm(ZU[p], ZU[pp]), d.invN);
  }
  fft_inverse_then(X, [&](int, int, int p, double2 v) { PE[p] = v; });

  if (!hs2) {
    // HS1 (1d/rhs.c:1-94): damping only
    HW_FOREACH(X) {
      const double2 v = PE[p];
      X.buf[pidx(idx)] = make_double2((d.dcoef[p] * v.x) * d.dchar[p], (d.dcoef[p] * v.y) * d.dchar[p]);
    }
    fft_forward_split(X, [&](int, int, int p, double2 zz, double2 zp) {
      DE[p] = split_re(zz, zp);
      DU[p] = split_im(zz, zp);
    });
  } else {
    // (2) varying depth: HSS(u^), a = u
    if (!flat) {
      member_sync(d.C);
      hss<M>(X, ZU, &PE[0].y, HS, PS);
      member_sync(d.C);
    }
    // (3) M0 u (and Hilbert eta for breaking, or d_x u for HS3) in physical space
    HW_FOREACH(X) {
      const int pp = partner_pos(X, idx);
      double2 m0, m0p;
      if (flat) {
        m0 = mul_ik(d.M0im[p], ZU[p]);
        m0p = mul_ik(d.M0im[pp], ZU[pp]);
      } else {
        m0 = cscale(mul_ik(d.k[p], HS[p]), -1 / kG);
        m0p = cscale(mul_ik(d.k[pp], HS[pp]), -1 / kG);
      }
      double2 s2 = make_double2(0.0, 0.0);
      if (hs3) {
        s2 = herm(mul_ik(d.k[p], ZU[p]), mul_ik(d.k[pp], ZU[pp]));
      } else if (brk) {
        const double kp = d.k[p], kq = d.k[pp];
        const double sp = kp / fabs(kp), sq = kq / fabs(kq);
        const double2 h0 = kp == 0 ? make_double2(0.0, 0.0) : make_double2(sp * ZE[p].y, -sp * ZE[p].x);
        const double2 h1 = kq == 0 ? make_double2(0.0, 0.0) : make_double2(sq * ZE[pp].y, -sq * ZE[pp].x);
        s2 = herm(h0, h1);
      }
      X.buf[pidx(idx)] = pack(herm(m0, m0p), s2, d.invN);
    }
    fft_inverse_then(X, [&](int, int, int p, double2 v) { PM[p] = v; });

    // (4) eta u and eta M0u -> spectra; L (eta M0 u)^ and the eta-equation H2 term
    HW_FOREACH(X) {
      const double2 e = PE[p];
      const double m0u = PM[p].x;
      if (!flat) PA[p].x = e.x * m0u;
      X.buf[pidx(idx)] = make_double2(e.x * e.y, e.x * m0u);
    }
    fft_forward_split(X, [&](int, int, int p, double2 zz, double2 zp) {
      const double2 ah = split_re(zz, zp), bh = split_im(zz, zp);
      if (flat) {
        const double2 lem = cscale(bh, d.L[p]);
        if (hs3) S9[p] = lem;
        const double2 ik = mul_ik(d.k[p], ah);
        AE[p] = make_double2(-lem.x - ik.x, -lem.y - ik.y);
      } else {
        S9[p] = bh;
        S10[p] = ah;
      }
    });
    if (!flat) {
      // L (eta M0u)^ = ik M1 (eta M0u)^, M1 = -(1/g) ik HSS (1d/functions.c:3393-3399)
      member_sync(d.C);
      hss<M>(X, S9, &PA[0].x, AU, PS);
      member_sync(d.C);
      HW_FOREACH(X) {
        (void)idx;
        const double kp = d.k[p];
        const double2 m1 = cscale(mul_ik(kp, AU[p]), -1 / kG);
        const double2 lem = mul_ik(kp, m1);
        if (hs3) S9[p] = lem;
        const double2 ik = mul_ik(kp, S10[p]);
        AE[p] = make_double2(-lem.x - ik.x, -lem.y - ik.y);
      }
    }
    // (5) u^2 - (M0u)^2 and damping eta -> u-equation H2 term and FFT(damp eta)
    HW_FOREACH(X) {
      const double2 e = PE[p];
      const double m0u = PM[p].x;
      X.buf[pidx(idx)] = make_double2(e.y * e.y - m0u * m0u, (d.dcoef[p] * e.x) * d.dchar[p]);
    }
    fft_forward_split(X, [&](int, int, int p, double2 zz, double2 zp) {
      const double2 ch = split_re(zz, zp);
      const double2 ik = mul_ik(d.k[p], ch);
      AU[p] = make_double2(-ik.x / 2, -ik.y / 2);
      DE[p] = split_im(zz, zp);
    });
    // (6) damping u
    HW_FOREACH(X) {
      const double2 e = PE[p];
      X.buf[pidx(idx)] = make_double2((d.dcoef[p] * e.y) * d.dchar[p], 0.0);
    }
    fft_forward_split(X, [&](int, int, int p, double2 zz, double2 zp) { DU[p] = split_re(zz, zp); });

    if (hs3) {
      // (7) L eta M0 u in physical space (and Hilbert eta for breaking)
      member_sync(d.C);
      HW_FOREACH(X) {
        const int pp = partner_pos(X, idx);
        double2 s2 = make_double2(0.0, 0.0);
        if (brk) {
          const double kp = d.k[p], kq = d.k[pp];
          const double sp = kp / fabs(kp), sq = kq / fabs(kq);
          const double2 h0 = kp == 0 ? make_double2(0.0, 0.0) : make_double2(sp * ZE[p].y, -sp * ZE[p].x);
          const double2 h1 = kq == 0 ? make_double2(0.0, 0.0) : make_double2(sq * ZE[pp].y, -sq * ZE[pp].x);
          s2 = herm(h0, h1);
        }
        X.buf[pidx(idx)] = pack(herm(S9[p], S9[pp]), s2, d.invN);
      }
      fft_inverse_then(X, [&](int, int, int p, double2 v) { PA[p] = v; });
      // (8) cubic terms (1d/functions.c:1590-1625, 3515-3540)
      HW_FOREACH(X) {
        const double e = PE[p].x, m0u = PM[p].x, dxu = PM[p].y;
        X.buf[pidx(idx)] = make_double2(e * e * m0u, m0u * (e * dxu + PA[p].x));
      }
      fft_forward_split(X, [&](int, int, int p, double2 zz, double2 zp) {
        const double2 dh = split_re(zz, zp), fh = split_im(zz, zp);
        S10[p] = dh;
        const double2 ik = mul_ik(d.k[p], fh);
        AU[p] = make_double2(AU[p].x - ik.x, AU[p].y - ik.y);
      });
      HW_FOREACH(X) {
        const double e = PE[p].x, dxu = PM[p].y, lm = PA[p].x;
        const double a3 = e * lm, b3 = e * e * dxu;
        if (!flat) PS[p].x = a3 + 0.5 * b3;   // physical A3 + B3/2 for HSS below
        X.buf[pidx(idx)] = make_double2(a3, b3);
      }
      fft_forward_split(X, [&](int, int, int p, double2 zz, double2 zp) {
        const double2 ah = split_re(zz, zp), bh = split_im(zz, zp);
        const double kp = d.k[p];
        if (flat) {
          const double Lp = d.L[p];
          const double2 dh = S10[p];
          AE[p].x += Lp * ah.x + (1 / 2.) * Lp * bh.x - (1 / 2.) * (kp * kp) * dh.x;
          AE[p].y += Lp * ah.y + (1 / 2.) * Lp * bh.y - (1 / 2.) * (kp * kp) * dh.y;
        } else {
          S9[p] = make_double2(ah.x + 0.5 * bh.x, ah.y + 0.5 * bh.y);
        }
      });
      if (!flat) {
        // ik (M0 A3^ + M0 B3^ / 2) - k^2 D3^ / 2, M0 linear: one HSS of A3^ + B3^/2
        member_sync(d.C);
        hss<M>(X, S9, &PS[0].x, RB, PM);
        member_sync(d.C);
        HW_FOREACH(X) {
          (void)idx;
          const double kp = d.k[p];
          const double2 m = cscale(mul_ik(kp, RB[p]), -1 / kG);
          const double2 ik = mul_ik(kp, m);
          const double2 dh = S10[p];
          AE[p].x += ik.x - (1 / 2.) * (kp * kp) * dh.x;
          AE[p].y += ik.y - (1 / 2.) * (kp * kp) * dh.y;
        }
      }
      member_sync(d.C);
    }
    // (9) nonlinear adjustment (1d/rhs.c:695): F(ChiAdj Re F^-1(.)) of both terms
    member_sync(d.C);
    HW_FOREACH(X) {
      const int pp = partner_pos(X, idx);
      X.buf[pidx(idx)] = pack(herm(AE[p], AE[pp]), herm(AU[p], AU[pp]), d.invN);
    }
    fft_inverse<M>(X.buf, d.tw, d.N, d.C, X.c);
    HW_FOREACH(X) {
      const double2 v = X.buf[pidx(idx)];
      const double ch = d.chi[p];
      X.buf[pidx(idx)] = make_double2(v.x * ch, v.y * ch);
    }
    fft_forward_split(X, [&](int, int, int p, double2 zz, double2 zp) {
      AE[p] = split_re(zz, zp);
      AU[p] = split_im(zz, zp);
    });
    // (10) kinematic breaking: eddy-viscosity force on the u-equation
    if (brk) {
      member_sync(d.C);
      rb_live = breaking_rhs<M>(X, t, PE, hs3 ? &PA[0].y : &PM[0].y, 2, AE, RB);
    }
  }
  // (11) assembly (1d/rhs.c:217-228, 373-385, 73-83) with the source term (1d/rhs.c:659)
  double pv = 0.0, ps = 0.0;
  if (d.has_influx) {
    pv = spline_eval(d.tt, d.ins, d.insc, d.n_in, t);
    ps = spline_eval(d.tt, d.skw, d.skwc, d.n_in, t);
  }
  member_sync(d.C);
  HW_FOREACH(X) {
    (void)idx;
    const double2 ze = ZE[p], zu = ZU[p];
    double2 h1e, h1u;
    if (flat || !hs2) {
      const double c1 = d.c1[p];
      h1e = make_double2(c1 * zu.y, -c1 * zu.x);
    } else {
      const double kp = d.k[p];
      h1e = make_double2((HS[p].y / kG) * kp, -(HS[p].x / kG) * kp);
    }
    const double gk = d.gk[p];
    h1u = make_double2(gk * ze.y, -gk * ze.x);
    double fr = 0.0, fi = 0.0;
    if (d.has_influx) {
      const double2 gx = d.gamX[p], gs = d.gamXs[p];
      if (d.prop_mode == 0) { fr = 0.5 * (pv * gx.x - ps * gs.x); fi = 0.5 * (pv * gx.y - ps * gs.y); }
      else if (d.prop_mode == 1) { fr = 0.5 * (pv * gx.x + ps * gs.x); fi = 0.5 * (pv * gx.y + ps * gs.y); }
      else if (d.prop_mode == 2) { fr = pv * gx.x; fi = pv * gx.y; }
    }
    const double al = d.aal[p];
    const double2 de = DE[p], du = DU[p];
    double2 te = h1e, tu = h1u;
    if (hs2) {
      te = cadd(te, AE[p]);
      tu = cadd(tu, AU[p]);
    }
    if (rb_live && hs2) tu = cadd(tu, RB[p]);
    dz[p] = make_double2((te.x + 2 * fr - de.x) * al, (te.y + 2 * fi - de.y) * al);
    dz[N + p] = make_double2((tu.x - du.x) * al, (tu.y - du.y) * al);
  }
}

}  // namespace hwdev
