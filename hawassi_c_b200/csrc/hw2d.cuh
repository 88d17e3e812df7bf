// hw2d.cuh -- HAWASSI 2D flat-bottom RHS (rhs_AB2_2DF_uv, 2d/fun_odesolver.c:4458)
// and its rkf45 attempt as five fused FFT passes plus stepper kernels.
//
// A 2D transform is a row pass and a column pass.  Row passes run one CTA per row
// pair {r, Ny-r} (with {0, Ny/2} sharing a CTA): that pair holds every point's
// conjugate mirror (-ky, -kx), so the Hermitian operations the reference
// performs on whole arrays (fftwcomplex_2d_sym before an inverse transform, real
// parts after it, the split of two real fields packed into one complex transform)
// are CTA-local.  Column passes run one CTA per column pair {2c, 2c+1} and do the
// physical-space products.  A CTA holds S slices (rows or columns) of M points in
// shared memory and transforms them with G groups of M/8 threads, one slice per
// group, in rounds.
//
// One RHS (HS2) = 5 kernels:
//   A row pass:    stage input z, E(eta)+iE(L phi), E(u)+iE(M0 u), E(v)+iE(M0 v), inverse row FFT
//   B column pass: inverse column FFT -> eta, Lphi, u, M0u, v, M0v -> 8 products
//                  packed into 4 complex fields -> forward column FFT
//   C row pass:    forward row FFT, split, damping spectra out, the four H2 terms
//                  symmetrised (fun_adjust's input), inverse row FFT
//   D column pass: inverse column FFT, x ChiAdj, forward column FFT; the source's
//                  column transform (its row transform is a set-up table)
//   E row pass:    forward row FFT of the adjusted terms, assembly of dt Z (x aal)
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "hw_fft.cuh"

namespace hw2d {

using hwdev::cadd;
using hwdev::cconj;
using hwdev::cmul;
using hwdev::cscale;
using hwdev::csub;
using hwdev::dft_small;
using hwdev::padded;
using hwdev::pidx;
using hwdev::twiddle_powers;
using hwdev::twd;

constexpr double kGrav = 9.80665;
constexpr int kGroups = 4;

struct Tab2 {
  int nx, ny, n, model, nt, chi_one, has_src;
  double fac_src;               // 1 (Uni+/-) or 2 (Bi)
  const double* kx;             // [nx]
  const double* ky;             // [ny]
  const double* c2g;            // C2d^2 / g
  const double* l2d;
  const double* aal;
  const double* damp;           // 7 Cpeak fbdy.charac
  const double* chi;            // ChiAdj
  const double2* gx;            // row transform of newGam
  const double2* sx;            // row transform of +-SkewGam (sign of the propagation)
  const double* tsig;           // [nt]
  const double* sig;            // [ny][nt] line signals and their spline coefficients
  const double* sigc;
  const double* sigs;
  const double* sigsc;
  const double2* twx;           // exp(-2 pi i q / nx)
  const double2* twy;           // exp(-2 pi i q / ny)
  // varying bottom, two reference depths (rhs_AB2_2DB_uv); var = 0 on a flat bottom
  int var;
  const double* gmin;           // Gam_min, Gam_plus (physical)
  const double* gplus;
  const double* cmin;           // Csqr2d_min, Csqr2d_plus (spectral)
  const double* cplus;
  const double* omin;           // Om2dSq_min, Om2dSq_plus (spectral)
  const double* oplus;
  const double* wallchar;       // dominfo.wallchar (harbour walls), nullptr: none
  const double* c2d;            // Oprt.C2d (flat bottom with walls only)
  int refl_one;                 // flat bottom, refl_coef == 1: fun_delphiH1hat's flux branch
  const double* gwx;            // fun_gradient(wallchar) (refl_one only)
  const double* gwy;
  // three reference depths (HSSgen_3depth): the middle depth's tables, nullptr: two
  const double* gmid;
  const double* cmid;
  const double* omid;
  // K reference depths (the plain K-reference and the learned operators): [K][N] weights,
  // C^2 and Omega^2 of each depth; nk = 0 when the min / plus (/ mid) tables serve
  int nk;
  const double* gk;
  const double* ck;
  const double* ok;
};

struct Work2 {
  double2* z;                   // stage input, 3 fields
  double2* R;                   // A -> B, 3 fields
  double2* Q;                   // B -> C, 4 fields
  double2* D;                   // damping spectra, 3 fields
  double2* W;                   // C -> D, 4 fields
  double2* V;                   // D -> E, 4 fields
  double2* src;                 // source spectrum
  double* insig;                // [ny] line signal at the stage time
  double* insigs;
  double* part;                 // per-block maxima of the error ratio
  // varying bottom only
  double* phys;                 // eta, u, v in physical space (3 real fields)
  double* pe;                   // eta M0u, eta M0v in physical space (2 real fields)
  double2* H1;                  // delu H1^, delv H1^ (2 fields)
  double2* EU;                  // (eta u)^, (eta v)^, deletaH2^ (3 fields)
  // kinematic breaking only: delphiH^ as the assembly forms it (nullptr: off)
  double2* dph;
  // flat bottom with walls: the round trip of (C u^, C v^) (delphiH1^ lands in H1)
  double2* WP;
  // HS3 on the flat bottom: eta, L phi in physical space (2 real fields) and the
  // HS2 terms with (eta^2 M0u)^, (eta^2 M0v)^ between passes C3 and I3 (6 fields)
  double* p3;
  double2* T3;
};

// device control block of the stepper (one per engine)
struct Ctl2 {
  double t, h, h0, t1, t_direct, eps_abs, eps_rel;
  int final_step, done, status, cur, k1i, need_k1, need_kout, attempts;
  long long rhs, acc, rej;
  // kinematic breaking on: every evolve_apply evaluates its own dydt_in and every
  // attempt its dydt_out (mode 8) before the step control, as gsl_odeiv2 does,
  // since each RHS past tprev advances the breaking state
  int brk;
};

enum { kOk = 0, kNonFinite = 1, kStepFailed = 2, kBreakCapacity = 3 };
// RHS launch conditions
enum { kAlways = 0, kIfK1 = 1, kIfStage = 2, kIfKout = 3 };

struct RK2 {
  double2* y[2];                // state, 3 fields each
  double2* kk[2];               // k1 / kout pair
  double2* ks[5];               // k2..k6
};

__device__ constexpr double A2_ah[5] = {1.0 / 4.0, 3.0 / 8.0, 12.0 / 13.0, 1.0, 1.0 / 2.0};
__device__ constexpr double A2_b3[2] = {3.0 / 32.0, 9.0 / 32.0};
__device__ constexpr double A2_b4[3] = {1932.0 / 2197.0, -7200.0 / 2197.0, 7296.0 / 2197.0};
__device__ constexpr double A2_b5[4] = {8341.0 / 4104.0, -32832.0 / 4104.0, 29440.0 / 4104.0, -845.0 / 4104.0};
__device__ constexpr double A2_b6[5] = {-6080.0 / 20520.0, 41040.0 / 20520.0, -28352.0 / 20520.0, 9295.0 / 20520.0,
                                        -5643.0 / 20520.0};
__device__ constexpr double A2_c[5] = {902880.0 / 7618050.0, 3953664.0 / 7618050.0, 3855735.0 / 7618050.0,
                                       -1371249.0 / 7618050.0, 277020.0 / 7618050.0};
__device__ constexpr double A2_ec[5] = {1.0 / 360.0, -128.0 / 4275.0, -2197.0 / 75240.0, 1.0 / 50.0, 2.0 / 55.0};

__device__ __forceinline__ bool rhs_active(const Ctl2* c, int cond) {
  if (cond == kAlways) return true;
  if (cond == kIfKout) return c->need_kout != 0;
  if (c->done) return false;
  if (cond == kIfK1) return c->need_k1 != 0;
  return true;
}

// ---------------------------------------------------------------------------
// one M-point slice in shared memory, transformed by one group of M/8 threads.
// Groups of at least a warp synchronise on their own named barrier (id 1 + g), so
// the groups of a CTA run their transforms independently; smaller groups fall
// back to the CTA barrier and keep step with each other.
// ---------------------------------------------------------------------------
template <int T>
__device__ __forceinline__ void group_sync(int g) {
  if constexpr (T >= 32) asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(T) : "memory");
  else __syncthreads();
}

template <int M, int R>
__device__ __forceinline__ void gpass(double2* buf, int Ns, const double2* __restrict__ tw, int sign, int tid,
                                      int g, bool act) {
  constexpr int T = M / 8;
  constexpr int NB = M / R;
  constexpr int BPT = 8 / R;
  double2 v[BPT][R];
  if (act) {
#pragma unroll
    for (int u = 0; u < BPT; ++u) {
      const int j = tid + u * T;
#pragma unroll
      for (int r = 0; r < R; ++r) v[u][r] = buf[pidx(j + r * NB)];
    }
  }
  group_sync<T>(g);
  if (act) {
#pragma unroll
    for (int u = 0; u < BPT; ++u) {
      const int j = tid + u * T;
      const int jm = j & (Ns - 1);
      if (Ns > 1) {
        const int qb = jm * (M / (Ns * R));
        double2 w[R];
        twiddle_powers<R>(twd(tw, qb, sign), w);
#pragma unroll
        for (int r = 1; r < R; ++r) v[u][r] = cmul(v[u][r], w[r]);
      }
      dft_small<R>(v[u], sign);
      const int idxD = (j - jm) * R + jm;
#pragma unroll
      for (int r = 0; r < R; ++r) buf[pidx(idxD + r * Ns)] = v[u][r];
    }
  }
  group_sync<T>(g);
}

template <int M>
__device__ __forceinline__ void gfft(double2* buf, const double2* __restrict__ tw, int sign, int tid, int g,
                                     bool act) {
  constexpr int L8 = (M >= 512) ? 3 : (M >= 64 ? 2 : 1);
  constexpr int rem = M / (1 << (3 * L8));
  int Ns = 1;
#pragma unroll
  for (int p = 0; p < L8; ++p) {
    gpass<M, 8>(buf, Ns, tw, sign, tid, g, act);
    Ns *= 8;
  }
  if constexpr (rem == 8) gpass<M, 8>(buf, Ns, tw, sign, tid, g, act);
  else if constexpr (rem == 4) gpass<M, 4>(buf, Ns, tw, sign, tid, g, act);
  else if constexpr (rem == 2) gpass<M, 2>(buf, Ns, tw, sign, tid, g, act);
}

// transform slices [0, ns) of the CTA's smem, kGroups at a time; CTA-wide barriers
// on entry and exit (the phases around read and write every slice)
template <int M>
__device__ __forceinline__ void fft_slices(double2* sm, int ns, const double2* __restrict__ tw, int sign) {
  constexpr int T = M / 8;
  const int g = threadIdx.x / T, tid = threadIdx.x % T;
  __syncthreads();
  for (int base = 0; base < ns; base += kGroups) {
    const int s = base + g;
    if constexpr (T >= 32) {
      if (s < ns) gfft<M>(sm + (size_t)s * padded(M), tw, sign, tid, g, true);
    } else {
      gfft<M>(sm + (size_t)s * padded(M), tw, sign, tid, g, s < ns);
    }
  }
  __syncthreads();
}

__device__ __forceinline__ double2 slot(double2* sm, int M, int s, int i) { return sm[(size_t)s * padded(M) + pidx(i)]; }
__device__ __forceinline__ void put(double2* sm, int M, int s, int i, double2 v) { sm[(size_t)s * padded(M) + pidx(i)] = v; }

// ---------------------------------------------------------------------------
// row-pair geometry and the Hermitian operators
// ---------------------------------------------------------------------------
struct Pair {
  int r[2];      // rows held (slice 2f + k holds row r[k] of field f)
  int mr[2];     // index (0/1) of the mirror row of r[k]
};

__device__ __forceinline__ Pair row_pair(int b, int Ny) {
  Pair p;
  if (b == 0) { p.r[0] = 0; p.r[1] = Ny / 2; p.mr[0] = 0; p.mr[1] = 1; }
  else { p.r[0] = b; p.r[1] = Ny - b; p.mr[0] = 1; p.mr[1] = 0; }
  return p;
}

// value of E(A) (herm) or S(A) (!herm) at (row k, column c) where S is the
// reference's fftwcomplex_2d_sym and E the Hermitian part of S(A) (what the real
// part of the inverse transform sees).  v[k][s]: A at row r[k], column (s ? cm : c)
// with cm = (Nx - c) % Nx.
__device__ __forceinline__ double2 sym_at(const double2 v[2][2], const Pair& P, int k, int s, int c, int Nx, int Ny,
                                          bool herm) {
  const int r = P.r[k];
  const double2 a = v[k][s];
  const double2 m = v[P.mr[k]][s ^ 1];
  if (c >= 1 && c < Nx / 2) return a;
  if (c > Nx / 2) return cconj(m);
  const bool selfrow = (r == 0) || (r == Ny / 2);
  if (selfrow) return make_double2(a.x, 0.0);
  if (c == 0) return (r < Ny / 2) ? a : cconj(m);
  return herm ? make_double2(0.5 * (a.x + m.x), 0.5 * (a.y - m.y)) : a;
}

// split Z = FFT(a + i b) at a point given Z there (z) and at its mirror (zm)
__device__ __forceinline__ void split2(double2 z, double2 zm, double2& A, double2& B) {
  A = make_double2(0.5 * (z.x + zm.x), 0.5 * (z.y - zm.y));
  const double2 w = make_double2(z.x - zm.x, z.y + zm.y);   // z - conj(zm)
  B = make_double2(0.5 * w.y, -0.5 * w.x);                  // w / (2i)
}

// mul by -i s: (x, y) -> (s y, -s x)
__device__ __forceinline__ double2 mul_mi(double2 a, double s) { return make_double2(s * a.y, -s * a.x); }
// mul by +i s
__device__ __forceinline__ double2 mul_pi(double2 a, double s) { return make_double2(-s * a.y, s * a.x); }

// GSL natural cubic spline evaluation with a plain binary search
__device__ __forceinline__ double spline2(const double* __restrict__ xs, const double* __restrict__ ys,
                                          const double* __restrict__ cs, int n, double x) {
  if (x < xs[0] || x > xs[n - 1]) return __longlong_as_double(0x7ff8000000000000ULL);
  int lo = 0, hi = n - 1;
  while (hi > lo + 1) {
    const int i = (hi + lo) / 2;
    if (xs[i] > x) hi = i; else lo = i;
  }
  const double xl = xs[lo], xh = xs[lo + 1], yl = ys[lo], yh = ys[lo + 1];
  const double h = xh - xl, dy = yh - yl, dx = x - xl;
  const double ci = cs[lo], cip = cs[lo + 1];
  const double bi = dy / h - h * (cip + 2.0 * ci) / 3.0;
  const double di = (cip - ci) / (3.0 * h);
  return yl + dx * (bi + dx * (ci + dx * di));
}

// modes: 0 direct RHS, 1 k1 (dydt_in), 2..6 the rkf45 stages, 7 k_out after an
// accepted step (reused as the next k1), 8 dydt_out of the attempt's candidate
// state at t + h before the step control (breaking runs)
__device__ __forceinline__ double stage_time(const Ctl2* c, int mode) {
  if (mode == 0) return c->t_direct;
  if (mode == 1 || mode == 7) return c->t;
  if (mode == 8) return c->t + c->h0;
  return c->t + A2_ah[mode - 2] * c->h0;
}

// IEEE products and sums without fused multiply-add (GSL's rounding)
__device__ __forceinline__ double rm2(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ra2(double a, double b) { return __dadd_rn(a, b); }

// stage input at element q (3n double2 per state): GSL rkf45's expression forms
__device__ __forceinline__ double2 stage_value(const RK2& B, const Ctl2* c, int mode, size_t q) {
  if (mode == 8) return B.y[c->cur ^ 1][q];
  const double2 y = B.y[c->cur][q];
  if (mode <= 1 || mode == 7) return y;
  const double h = c->h0;
  const double2 a = B.kk[c->k1i][q];
  if (mode == 2) {
    const double f = rm2(A2_ah[0], h);
    return make_double2(ra2(y.x, rm2(f, a.x)), ra2(y.y, rm2(f, a.y)));
  }
  const double2 b = B.ks[0][q];
  if (mode == 3)
    return make_double2(ra2(y.x, rm2(h, ra2(rm2(A2_b3[0], a.x), rm2(A2_b3[1], b.x)))),
                        ra2(y.y, rm2(h, ra2(rm2(A2_b3[0], a.y), rm2(A2_b3[1], b.y)))));
  const double2 c3 = B.ks[1][q];
  if (mode == 4)
    return make_double2(
        ra2(y.x, rm2(h, ra2(ra2(rm2(A2_b4[0], a.x), rm2(A2_b4[1], b.x)), rm2(A2_b4[2], c3.x)))),
        ra2(y.y, rm2(h, ra2(ra2(rm2(A2_b4[0], a.y), rm2(A2_b4[1], b.y)), rm2(A2_b4[2], c3.y)))));
  const double2 c4 = B.ks[2][q];
  if (mode == 5)
    return make_double2(
        ra2(y.x, rm2(h, ra2(ra2(ra2(rm2(A2_b5[0], a.x), rm2(A2_b5[1], b.x)), rm2(A2_b5[2], c3.x)),
                            rm2(A2_b5[3], c4.x)))),
        ra2(y.y, rm2(h, ra2(ra2(ra2(rm2(A2_b5[0], a.y), rm2(A2_b5[1], b.y)), rm2(A2_b5[2], c3.y)),
                            rm2(A2_b5[3], c4.y)))));
  const double2 c5 = B.ks[3][q];
  return make_double2(
      ra2(y.x, rm2(h, ra2(ra2(ra2(ra2(rm2(A2_b6[0], a.x), rm2(A2_b6[1], b.x)), rm2(A2_b6[2], c3.x)),
                              rm2(A2_b6[3], c4.x)),
                          rm2(A2_b6[4], c5.x)))),
      ra2(y.y, rm2(h, ra2(ra2(ra2(ra2(rm2(A2_b6[0], a.y), rm2(A2_b6[1], b.y)), rm2(A2_b6[2], c3.y)),
                              rm2(A2_b6[3], c4.y)),
                          rm2(A2_b6[4], c5.y)))));
}

// ---------------------------------------------------------------------------
// stage input z = y + h sum_j b_sj k_j of every point, a streaming pass ahead of the
// the buffer an RHS of the given mode writes
__device__ __forceinline__ double2* rhs_out(const RK2& rk, const Ctl2* ctl, int mode, double2* direct_out) {
  if (mode == 0) return direct_out;
  if (mode == 1) return rk.kk[ctl->k1i];
  if (mode == 7 || mode == 8) return rk.kk[ctl->k1i ^ 1];
  return rk.ks[mode - 2];
}

// first row pass (mode 1 and 7: z = y)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k2_stage(RK2 rk, Work2 w, const Ctl2* __restrict__ ctl, int mode, int cond, size_t n3) {
  if (!rhs_active(ctl, cond)) return;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n3; q += (size_t)gridDim.x * blockDim.x)
    w.z[q] = stage_value(rk, ctl, mode, q);
}

// ---------------------------------------------------------------------------
// A: row pass, stage input -> symmetrised spectra -> inverse row FFT
// smem slices: 2f + k = field f (0: eta|Lphi, 1: u|M0u, 2: v|M0v), row r[k]
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2_rowA(Tab2 tb, Work2 w, RK2 rk, const Ctl2* __restrict__ ctl, Ctl2* ctlw, int mode, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const size_t n = (size_t)tb.n;
  const Pair P = row_pair(blockIdx.x, Ny);
  const double ts = stage_time(ctl, mode);
  if (blockIdx.x == 0 && threadIdx.x == 0 && ctlw) ctlw->rhs += 1;
  // line signals of the two rows at the stage time
  if (tb.has_src && threadIdx.x < 2) {
    const int r = P.r[threadIdx.x];
    const size_t o = (size_t)r * tb.nt;
    w.insig[r] = spline2(tb.tsig, tb.sig + o, tb.sigc + o, tb.nt, ts);
    w.insigs[r] = spline2(tb.tsig, tb.sigs + o, tb.sigsc + o, tb.nt, ts);
  }
  for (int j = threadIdx.x; j <= Nx / 2; j += blockDim.x) {
    const int cm = (Nx - j) % Nx;
    const int cc[2] = {j, cm};
    double2 e[2][2], u[2][2], v[2][2], t1[2][2], t2[2][2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int r = P.r[k];
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const size_t q = (size_t)r * Nx + cc[s];
        const double2 ze = w.z[q], zu = w.z[n + q], zv = w.z[2 * n + q];
        e[k][s] = ze; u[k][s] = zu; v[k][s] = zv;
        // M0 u^ = -i (C^2/g) kx u^ ; M0 v^ = -i (C^2/g) ky v^
        const double cg = tb.c2g[q];
        const double kxv = tb.kx[cc[s]], kyv = tb.ky[r];
        t1[k][s] = make_double2(cg * kxv * zu.y, -cg * kxv * zu.x);
        t2[k][s] = make_double2(cg * kyv * zv.y, -cg * kyv * zv.x);
      }
    }
    // slices 2..5: E(u^) + i E(M0u^), E(v^) + i E(M0v^)
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        const double2 U1 = sym_at(u, P, k, s, c, Nx, Ny, true), U2 = sym_at(t1, P, k, s, c, Nx, Ny, true);
        const double2 V1 = sym_at(v, P, k, s, c, Nx, Ny, true), V2 = sym_at(t2, P, k, s, c, Nx, Ny, true);
        put(sm, M, 2 + k, c, make_double2(U1.x - U2.y, U1.y + U2.x));
        put(sm, M, 4 + k, c, make_double2(V1.x - V2.y, V1.y + V2.x));
      }
    // L phi^ = M0u^ + M0v^ ; slices 0, 1: E(eta^) + i E(L phi^)
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) t1[k][s] = make_double2(t1[k][s].x + t2[k][s].x, t1[k][s].y + t2[k][s].y);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        const double2 E1 = sym_at(e, P, k, s, c, Nx, Ny, true), E2 = sym_at(t1, P, k, s, c, Nx, Ny, true);
        put(sm, M, 0 + k, c, make_double2(E1.x - E2.y, E1.y + E2.x));
      }
  }
  fft_slices<M>(sm, 6, tb.twx, +1);
  for (int s = 0; s < 6; ++s) {
    const int f = s >> 1, k = s & 1;
    double2* dst = w.R + f * n + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) dst[j] = slot(sm, M, s, j);
  }
}

// column-pair load / store helpers (slice 2f + k = field f, column 2c + k)
template <int M>
__device__ __forceinline__ void col_load(double2* sm, int s0, const double2* __restrict__ F, int Nx, int c) {
  for (int y = threadIdx.x; y < M; y += blockDim.x) {
    const double2* p = F + (size_t)y * Nx + 2 * c;
    put(sm, M, s0, y, p[0]);
    put(sm, M, s0 + 1, y, p[1]);
  }
}
template <int M>
__device__ __forceinline__ void col_store(const double2* sm, int s0, double2* __restrict__ F, int Nx, int c) {
  for (int y = threadIdx.x; y < M; y += blockDim.x) {
    double2* p = F + (size_t)y * Nx + 2 * c;
    p[0] = sm[(size_t)s0 * padded(M) + pidx(y)];
    p[1] = sm[(size_t)(s0 + 1) * padded(M) + pidx(y)];
  }
}

// ---------------------------------------------------------------------------
// B: column pass, inverse column FFT -> physical products -> forward column FFT
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2_colB(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
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
      const double dmp = tb.damp[q];
      // Q1 = dampeta + i dampu, Q2 = dampv + i deletaH2, Q3 = etaM0u + i eta u, Q4 = etaM0v + i eta v
      put(sm, M, 0 + k, y, make_double2(dmp * eta, dmp * u));
      put(sm, M, 2 + k, y, make_double2(dmp * v, 0.5 * ((u * u + v * v) - lphi * lphi)));
      if (tb.wallchar) {   // the H2 products carry wallchar (2d/fun_odesolver.c:3239-3249)
        const double wc = tb.wallchar[q];
        put(sm, M, 2 + k, y, make_double2(dmp * v, 0.5 * ((u * u + v * v) - lphi * lphi) * wc));
        put(sm, M, 4 + k, y, make_double2(eta * m0u * wc, eta * u * wc));
        put(sm, M, 6 + k, y, make_double2(eta * m0v * wc, eta * v * wc));
      } else {
        put(sm, M, 4 + k, y, make_double2(eta * m0u, eta * u));
        put(sm, M, 6 + k, y, make_double2(eta * m0v, eta * v));
      }
    }
  }
  fft_slices<M>(sm, 8, tb.twy, -1);
  for (int f = 0; f < 4; ++f) col_store<M>(sm, 2 * f, w.Q + f * n, Nx, c);
}

// ---------------------------------------------------------------------------
// C: row pass, forward row FFT -> split -> damping spectra, symmetrised H2 terms
//    -> inverse row FFT (or, with ChiAdj = 1, the adjusted terms themselves)
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2_rowC(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
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
  // Each quad (columns j and Nx - j of both rows) is read and rewritten by one
  // thread at its own positions only, so no barrier separates the reads from the
  // writes.  Output slices: 0,1 S(ikx deletaH2^), 2,3 S(iky deletaH2^),
  // 4,5 S(deluH2^), 6,7 S(delvH2^); each pair of slices is written after the
  // quad's values of the field held there have been read.
  for (int j = threadIdx.x; j <= Nx / 2; j += blockDim.x) {
    const int cm = (Nx - j) % Nx;
    const int cc[2] = {j, cm};
    double2 z[2][2], a1[2][2], a2[2][2];
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
    // Q2 -> damping spectrum of v, deletaH2^ -> i kx deletaH2^, i ky deletaH2^
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) z[k][s] = slot(sm, M, 2 + k, cc[s]);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double2 dv, dH;
        split2(z[k][s], z[P.mr[k]][s ^ 1], dv, dH);
        const int r = P.r[k], c = cc[s];
        if (s == 0 || cm != j) w.D[2 * n + (size_t)r * Nx + c] = dv;
        a1[k][s] = mul_pi(dH, tb.kx[c]);
        a2[k][s] = mul_pi(dH, tb.ky[r]);
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        put(sm, M, 0 + k, c, sym_at(a1, P, k, s, c, Nx, Ny, false));
        put(sm, M, 2 + k, c, sym_at(a2, P, k, s, c, Nx, Ny, false));
      }
    // Q3 -> deluH2^ = -L (eta M0u)^ - i kx (eta u)^
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
        const double L = tb.l2d[(size_t)r * Nx + c], kxv = tb.kx[c];
        a1[k][s] = make_double2(-L * em.x + kxv * eu.y, -L * em.y - kxv * eu.x);
      }
    // Q4 -> delvH2^ = -L (eta M0v)^ - i ky (eta v)^
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
        const double L = tb.l2d[(size_t)r * Nx + c], kyv = tb.ky[r];
        a2[k][s] = make_double2(-L * em.x + kyv * ev.y, -L * em.y - kyv * ev.x);
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
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

// ---------------------------------------------------------------------------
// D: column pass, inverse column FFT -> x ChiAdj / N -> forward column FFT;
//    slices 8, 9: column transform of the source (row transform tabulated)
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2_colD(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx;
  const size_t n = (size_t)tb.n;
  const int c = blockIdx.x;
  const int nadj = tb.chi_one ? 0 : 8;
  if (!tb.chi_one) {
    for (int f = 0; f < 4; ++f) col_load<M>(sm, 2 * f, w.W + f * n, Nx, c);
    __syncthreads();
    fft_slices<M>(sm, 8, tb.twy, +1);
    const double invN = 1.0 / ((double)tb.n);
    for (int y = threadIdx.x; y < M; y += blockDim.x) {
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const double ch = tb.chi[(size_t)y * Nx + 2 * c + k];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          const double2 a = slot(sm, M, 2 * f + k, y);
          put(sm, M, 2 * f + k, y, make_double2(a.x * invN * ch, a.y * invN * ch));
        }
      }
    }
  }
  if (tb.has_src) {
    for (int y = threadIdx.x; y < M; y += blockDim.x) {
      const double a = tb.fac_src * w.insig[y], b = w.insigs[y];
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const size_t q = (size_t)y * Nx + 2 * c + k;
        const double2 g = tb.gx[q], s = tb.sx[q];
        put(sm, M, nadj + k, y, make_double2(a * g.x + b * s.x, a * g.y + b * s.y));
      }
    }
  }
  __syncthreads();
  const int ns = nadj + (tb.has_src ? 2 : 0);
  fft_slices<M>(sm, ns, tb.twy, -1);
  if (!tb.chi_one)
    for (int f = 0; f < 4; ++f) col_store<M>(sm, 2 * f, w.V + f * n, Nx, c);
  if (tb.has_src) col_store<M>(sm, nadj, w.src, Nx, c);
}

// ---------------------------------------------------------------------------
// E: row pass, forward row FFT of the adjusted terms -> dt Z
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2_rowE(Tab2 tb, Work2 w, RK2 rk, const Ctl2* __restrict__ ctl, int mode, int cond, double2* __restrict__ direct_out) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const size_t n = (size_t)tb.n;
  const Pair P = row_pair(blockIdx.x, Ny);
  for (int s = 0; s < 8; ++s) {
    const int f = s >> 1, k = s & 1;
    const double2* src = w.V + f * n + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) put(sm, M, s, j, src[j]);
  }
  __syncthreads();
  if (!tb.chi_one) fft_slices<M>(sm, 8, tb.twx, -1);
  double2* out = rhs_out(rk, ctl, mode, direct_out);
  for (int k = 0; k < 2; ++k) {
    const int r = P.r[k];
    const double kyv = tb.ky[r];
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) {
      const size_t q = (size_t)r * Nx + j;
      const double kxv = tb.kx[j];
      const double a = tb.aal[q], cg = tb.var ? 0.0 : tb.c2g[q];
      const double2 ze = w.z[q], zu = w.z[n + q], zv = w.z[2 * n + q];
      double2 dphi;
      if (tb.var) {
        // delu H1^ + delv H1^ from the two-depth operator (2d/fun_odesolver.c:4560-4563)
        const double2 h1u = w.H1[q], h1v = w.H1[n + q];
        dphi = make_double2(h1u.x + h1v.x, h1u.y + h1v.y);
      } else if (tb.wallchar) {
        dphi = w.H1[q];   // the wall branch's delphiH1^ (k2w_row3)
      } else {
        // delphiH1^ = -i (kx C^2/g u^ + ky C^2/g v^)
        const double2 du1 = make_double2(cg * zu.x, cg * zu.y), dv1 = make_double2(cg * zv.x, cg * zv.y);
        dphi = make_double2(kxv * du1.y + kyv * dv1.y, -kxv * du1.x - kyv * dv1.x);
      }
      double2 ix = slot(sm, M, 0 + k, j), iy = slot(sm, M, 2 + k, j);
      if (tb.model != 1) {   // HS2, HS3 (the cubic terms are summed into the same slices)
        const double2 au = slot(sm, M, 4 + k, j), av = slot(sm, M, 6 + k, j);
        dphi = make_double2(dphi.x + au.x + av.x, dphi.y + au.y + av.y);
      } else {
        // HS1 (rhs_AB1_2DF_uv / rhs_AB1_2DB_uv, 2d/fun_odesolver.c:4350-4456): no H2 terms
        ix = make_double2(0.0, 0.0);
        iy = make_double2(0.0, 0.0);
      }
      if (w.dph) w.dph[q] = dphi;
      const double2 S = tb.has_src ? w.src[q] : make_double2(0.0, 0.0);
      const double2 de = w.D[q], du = w.D[n + q], dv = w.D[2 * n + q];
      out[q] = make_double2((S.x + dphi.x - de.x) * a, (S.y + dphi.y - de.y) * a);
      out[n + q] = make_double2((kGrav * kxv * ze.y - ix.x - du.x) * a, (-kGrav * kxv * ze.x - ix.y - du.y) * a);
      out[2 * n + q] = make_double2((kGrav * kyv * ze.y - iy.x - dv.x) * a, (-kGrav * kyv * ze.x - iy.y - dv.y) * a);
    }
  }
}

// ---------------------------------------------------------------------------
// stepper kernels
// ---------------------------------------------------------------------------
constexpr int kCombBlocks = 592;   // 4 x 148 SMs
constexpr int kCombThreads = 256;

// y_new = y + h0 sum c_i k_i into y[cur ^ 1]; per-block max of |yerr| / D0
__global__ void __launch_bounds__(kCombThreads)
k2_combine(RK2 rk, Work2 w, const Ctl2* __restrict__ ctl, size_t n3) {
  __shared__ double red[kCombThreads / 32];
  __shared__ int badw[kCombThreads / 32];
  if (ctl->done) return;
  const double h = ctl->h0, er = ctl->eps_rel, ea = ctl->eps_abs;
  const double2* __restrict__ y = rk.y[ctl->cur];
  double2* __restrict__ yn = rk.y[ctl->cur ^ 1];
  const double2* __restrict__ k1 = rk.kk[ctl->k1i];
  double rm = 2.2250738585072014e-308;
  int bad = 0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n3; q += (size_t)gridDim.x * blockDim.x) {
    const double2 a = k1[q], c = rk.ks[1][q], e = rk.ks[2][q], f = rk.ks[3][q], g = rk.ks[4][q], yy = y[q];
    const double dix = ra2(ra2(ra2(ra2(rm2(A2_c[0], a.x), rm2(A2_c[1], c.x)), rm2(A2_c[2], e.x)), rm2(A2_c[3], f.x)),
                           rm2(A2_c[4], g.x));
    const double diy = ra2(ra2(ra2(ra2(rm2(A2_c[0], a.y), rm2(A2_c[1], c.y)), rm2(A2_c[2], e.y)), rm2(A2_c[3], f.y)),
                           rm2(A2_c[4], g.y));
    const double2 nv = make_double2(ra2(yy.x, rm2(h, dix)), ra2(yy.y, rm2(h, diy)));
    yn[q] = nv;
    const double ex = rm2(h, ra2(ra2(ra2(ra2(rm2(A2_ec[0], a.x), rm2(A2_ec[1], c.x)), rm2(A2_ec[2], e.x)),
                                     rm2(A2_ec[3], f.x)), rm2(A2_ec[4], g.x)));
    const double ey = rm2(h, ra2(ra2(ra2(ra2(rm2(A2_ec[0], a.y), rm2(A2_ec[1], c.y)), rm2(A2_ec[2], e.y)),
                                     rm2(A2_ec[3], f.y)), rm2(A2_ec[4], g.y)));
    const double rx = fabs(ex) / fabs(ra2(rm2(er, fabs(nv.x)), ea));
    const double ry = fabs(ey) / fabs(ra2(rm2(er, fabs(nv.y)), ea));
    bad |= (!(rx == rx) || !(ry == ry) || isinf(nv.x) || isinf(nv.y)) ? 1 : 0;
    rm = fmax(rm, fmax(rx, ry));
  }
  for (int o = 16; o > 0; o >>= 1) {
    rm = fmax(rm, __shfl_xor_sync(0xffffffffu, rm, o));
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5] = rm; badw[threadIdx.x >> 5] = bad; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = red[0];
    int b = badw[0];
    for (int i = 1; i < kCombThreads / 32; ++i) { m = fmax(m, red[i]); b |= badw[i]; }
    w.part[blockIdx.x] = b ? __longlong_as_double(0x7ff0000000000000ULL) : m;
  }
}

__device__ __forceinline__ void set_prologue(Ctl2* c) {
  const double dt = c->t1 - c->t;
  double h0 = c->h;
  c->final_step = 0;
  if ((dt >= 0.0 && h0 > dt) || (dt < 0.0 && h0 < dt)) { h0 = dt; c->final_step = 1; }
  c->h0 = h0;
}

// std_control_hadjust + gsl_odeiv2_evolve_apply's accept / retry decision
__global__ void k2_control(Ctl2* c, const Work2 w, int nparts) {
  __shared__ double red[32];
  if (c->done) return;
  double m = 2.2250738585072014e-308;
  bool nonfin = false;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    const double v = w.part[i];
    if (!(v <= 1.7976931348623157e308)) nonfin = true;
    m = fmax(m, v);
  }
  const int anynf = __syncthreads_or(nonfin ? 1 : 0);
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x != 0) return;
  double rmax = red[0];
  for (int i = 1; i < (int)(blockDim.x / 32); ++i) rmax = fmax(rmax, red[i]);
  c->need_k1 = 0;   // the attempt's k1 is in place
  if (anynf) { c->status = kNonFinite; c->done = 1; return; }
  const double t0 = c->t, h_old = c->h0;
  const double tn = c->final_step ? c->t1 : t0 + h_old;
  int adj = 0;
  double hn = h_old;
  if (rmax > 1.1) {
    double r = 0.9 / pow(rmax, 1.0 / 5.0);
    if (r < 0.2) r = 0.2;
    hn = r * h_old;
    adj = -1;
  } else if (rmax < 0.5) {
    double r = 0.9 / pow(rmax, 1.0 / 6.0);
    if (r > 5.0) r = 5.0;
    if (r < 1.0) r = 1.0;
    hn = r * h_old;
    adj = 1;
  }
  if (adj == -1) {
    const double t_next = tn + hn;
    if (fabs(hn) < fabs(h_old) && t_next != tn) {
      c->rej += 1;
      if (++c->attempts > 1000) { c->status = kStepFailed; c->done = 1; return; }
      c->h = hn;
      set_prologue(c);
      return;
    }
    hn = h_old;
  }
  c->acc += 1;
  c->attempts = 0;
  c->cur ^= 1;
  const double tk = t0 + h_old;
  c->t = tn;
  c->h = hn;
  if (tk == tn && !c->brk) c->need_kout = 1;
  else c->need_k1 = 1;
  if (!(c->t < c->t1)) c->done = 1;
  else set_prologue(c);
}

__global__ void k2_finalize(Ctl2* c) {
  if (c->need_kout) {
    c->k1i ^= 1;
    c->need_kout = 0;
  }
}

__global__ void k2_begin(Ctl2* c, double t1) {
  c->t1 = t1;
  c->status = kOk;
  c->attempts = 0;
  c->done = (c->t < t1) ? 0 : 1;
  if (!c->done) set_prologue(c);
}

// reference layout [Re eta | Im eta | Re u | Im u | Re v | Im v] <-> 3 double2 fields
__global__ void k2_to_internal(const double* __restrict__ yr, double2* __restrict__ yi, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < 3 * n; q += (size_t)gridDim.x * blockDim.x) {
    const size_t f = q / n, p = q - f * n;
    yi[q] = make_double2(yr[2 * f * n + p], yr[(2 * f + 1) * n + p]);
  }
}
__global__ void k2_to_reference(const double2* __restrict__ yi, double* __restrict__ yr, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < 3 * n; q += (size_t)gridDim.x * blockDim.x) {
    const size_t f = q / n, p = q - f * n;
    const double2 v = yi[q];
    yr[2 * f * n + p] = v.x;
    yr[(2 * f + 1) * n + p] = v.y;
  }
}

}  // namespace hw2d
