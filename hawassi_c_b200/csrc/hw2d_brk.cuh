// hw2d_brk.cuh -- kinematic breaking of the 2D model on the device: the
// breaking_process state machine (2d/breaking.c:505-733 with breaking_criterion
// :215-326, fun_peaks :56-136, funBr_Char :351-441, funBr_find_peak_loc :443-454,
// funBr_BreakNodes_char :456-503, fun_check_crest :328-349) and the eddy-viscosity
// force fun_sbreaking (2d/fun_odesolver.c:985-1019), as called by rhs_AB2_2DB_uv
// (:4578-4586): B is cleared on every RHS, the update runs only when the RHS's t
// exceeds tprev (the start of the current evolve_apply), and Sb_xhat / Sb_yhat keep
// their last values otherwise.
//
// Kernels, appended to the varying-bottom RHS after its assembly pass:
//   rowI  (row pass)   the update's dt eta^ with the symmetrised delphiH^ (the
//                      reference's ifftw_2d_c2r symmetrises it in place), and
//                      E(S(delphiH^)) + i E(S(HilbEta^)) -> inverse row FFT
//   colI  (col pass)   inverse column FFT -> delphi, HilbEta in physical space
//   peaks (grid)       B = 0; fun_peaks' test at every point, ranks appended
//   sort  (one CTA)    the peak ranks in fun_peaks' order (bitonic sort)
//   machine (one warp) criterion at the peaks, crest merging and tracking, break
//                      nodes and B, the breaking.dat record, ITERbdt
//   flux  (grid)       Flux = -B delb^2 (eta - bathy) delphi^2
//   sbcol (col pass)   fun_gradient, Sb = grad Flux / (eta - bathy), packed
//                      Sb_x + i Sb_y -> forward column FFT
//   sbrow (row pass)   forward row FFT, split -> Sb_xhat, Sb_yhat; dt u^, dt v^
//                      += Sb aal (also with the kept Sb when no update runs)
// A crest's scans (search sector, arg-max, break nodes) cover only the bounding
// box of its search disc: every point outside the disc contributes exactly zero.
// Node lists have no 100-entry limit (the reference's CBvar arrays overflow for
// larger crests); capacities are checked and an overflow stops the run.
#pragma once

#include "hw2d.cuh"

namespace hw2d {

constexpr int kBrkPeakCap = 16384;   // peaks sorted per update (one CTA, 64 KB of shared memory)
constexpr int kBrkCrestCap = 16384;  // records in CB, CBNew, CBPrev
constexpr int kBrkSortThreads = 1024;

struct Crest2 {
  int xindex, yindex, xNow, yNow, kwadran;
  int off, nnode;                    // break nodes of a CBPrev slot in its pool
  double Ucrest, time, theta;
};

// device state of the breaking machine (the reference's globals)
struct BrkSt {
  int flagbr, iterbdt, ncbprev, npeaks, sb_zero, bn_cur, err, nrec;
  long long nlog;
};
enum { kBrkErrPeaks = 1, kBrkErrCrests = 2, kBrkErrNodes = 4, kBrkErrLog = 8 };

struct Brk2 {
  int on;
  const double* bathy;               // dominfo.bathy.data (= -depth)
  const double* pbchar;              // pb.Char
  const double* x;                   // dominfo.x [nx]
  const double* y;                   // dominfo.y [ny]
  double dx, dy, thr, tstar, rsearch, kbc, tc, delb, cur_u, t0, dt_out;
  double* B;                         // [n]
  double* flux;                      // [n]
  double2* P;                        // [n] packed transform scratch
  double2* dh;                       // [n] (delphi, HilbEta) in physical space
  double2* sb;                       // [2n] Sb_xhat, Sb_yhat
  int* peaks;                        // [kBrkPeakCap] peak ranks
  Crest2* CB;
  Crest2* CBNew;
  Crest2* CBPrev;
  int2* bn[2];                       // break nodes of the CBPrev slots: last update / this update
  int2* bnp;                         // every crest's sector nodes of this update
  int cap_nodes;
  double* log_t;                     // breaking.dat: record times
  int* log_cnt;                      //               node pairs per record
  int2* log_nodes;
  int cap_rec;
  long long cap_log;
  BrkSt* st;
};

__device__ __forceinline__ double rs2(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ bool brk_update(const Ctl2* ctl, int mode) { return stage_time(ctl, mode) > ctl->t; }
__device__ __forceinline__ int fsign(double v) { return v < 0 ? -1 : 1; }   // fun_sign

// fun_peaks' visiting order as a rank: interior points x-major, then the edges
// x = 0, x = Nx-1 (along y) and y = 0, y = Ny-1 (along x); corners are never peaks
__device__ __forceinline__ void rank_to_xy(int r, int Nx, int Ny, int& x, int& y) {
  const int I = (Nx - 2) * (Ny - 2);
  if (r < I) { x = r / (Ny - 2) + 1; y = r % (Ny - 2) + 1; return; }
  r -= I;
  if (r < Ny - 2) { x = 0; y = r + 1; return; }
  r -= Ny - 2;
  if (r < Ny - 2) { x = Nx - 1; y = r + 1; return; }
  r -= Ny - 2;
  if (r < Nx - 2) { y = 0; x = r + 1; return; }
  r -= Nx - 2;
  y = Ny - 1;
  x = r + 1;
}

// the search sector of a crest (funBr_Char): disc of radius Rsearch around
// (x[xNow], y[yNow]) cut to the 160-degree sector of its quadrant
struct Sector {
  double xp, yp, R2, ca, sa, cb, sbt;
  int kw;
  int i0, i1, j0, j1;                // bounding box of the disc (grid indices)
};

__device__ __forceinline__ Sector sector_of(const Brk2& b, const Crest2& r, int Nx, int Ny) {
  Sector g;
  g.xp = b.x[r.xNow];
  g.yp = b.y[r.yNow];
  g.R2 = rm2(b.rsearch, b.rsearch);
  g.kw = r.kwadran;
  const double spread = 80.0;
  const double sp = spread * M_PI / 180.0;
  double alpha, beta;
  if (r.kwadran == 1 || r.kwadran == 3) {
    alpha = rs2(r.theta, sp);
    beta = rs2(ra2(sp, r.theta), M_PI / 2.0);
  } else {
    alpha = rs2(sp, r.theta);
    beta = rs2(rs2(M_PI / 2.0, r.theta), sp);
  }
  g.ca = cos(alpha);
  g.sa = sin(alpha);
  g.cb = cos(beta);
  g.sbt = sin(beta);
  const double R = b.rsearch;
  g.j0 = max(0, (int)floor((g.xp - R - b.x[0]) / b.dx) - 2);
  g.j1 = min(Nx - 1, (int)ceil((g.xp + R - b.x[0]) / b.dx) + 2);
  g.i0 = max(0, (int)floor((g.yp - R - b.y[0]) / b.dy) - 2);
  g.i1 = min(Ny - 1, (int)ceil((g.yp + R - b.y[0]) / b.dy) + 2);
  return g;
}

// funBr_Char at (i, j): 1 inside the crest's sector, 0 elsewhere
__device__ __forceinline__ double sector_char(const Brk2& b, const Sector& g, int i, int j) {
  const double xc = rs2(b.x[j], g.xp), yc = rs2(b.y[i], g.yp);
  if (!(ra2(rm2(xc, xc), rm2(yc, yc)) <= g.R2)) return 0.0;
  const double XXr = ra2(rm2(xc, g.ca), rm2(yc, g.sa));
  const double YYr = rs2(rm2(yc, g.cb), rm2(xc, g.sbt));
  switch (g.kw) {
    case 1: if ((XXr < 0) || (YYr < 0)) return 0.0; break;
    case 2: if ((XXr > 0) || (YYr < 0)) return 0.0; break;
    case 3: if ((XXr > 0) || (YYr > 0)) return 0.0; break;
    default: if ((XXr < 0) || (YYr > 0)) return 0.0; break;
  }
  return 1.0;
}

__device__ __forceinline__ int fun_kwadran(double ux, double uy) {
  if ((ux >= 0) && (uy >= 0)) return 1;
  if ((ux < 0) && (uy >= 0)) return 2;
  if ((ux < 0) && (uy < 0)) return 3;
  return 4;
}

// gradient2D at one point (one-sided at the edges)
__device__ __forceinline__ double gxat(const double* a, int st, int Nx, int i, int j, double dx) {
  const size_t r = (size_t)i * Nx;
  if (j == 0) return rs2(a[(r + 1) * st], a[r * st]) / dx;
  if (j == Nx - 1) return rs2(a[(r + Nx - 1) * st], a[(r + Nx - 2) * st]) / dx;
  return rs2(a[(r + j + 1) * st], a[(r + j - 1) * st]) / (2 * dx);
}
__device__ __forceinline__ double gyat(const double* a, int st, int Nx, int Ny, int i, int j, double dy) {
  if (i == 0) return rs2(a[((size_t)Nx + j) * st], a[(size_t)j * st]) / dy;
  if (i == Ny - 1) return rs2(a[((size_t)(Ny - 1) * Nx + j) * st], a[((size_t)(Ny - 2) * Nx + j) * st]) / dy;
  return rs2(a[((size_t)(i + 1) * Nx + j) * st], a[((size_t)(i - 1) * Nx + j) * st]) / (2 * dy);
}

// ---------------------------------------------------------------------------
// rowI: S(delphiH^) into dt eta^, and E(S(delphiH^)) + i E(S(HilbEta^)) -> inverse rows
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2b_rowI(Tab2 tb, Work2 w, Brk2 b, RK2 rk, const Ctl2* __restrict__ ctl, int mode, int cond,
         double2* __restrict__ direct_out) {
  if (!rhs_active(ctl, cond) || !brk_update(ctl, mode)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const Pair P = row_pair(blockIdx.x, Ny);
  double2* out = rhs_out(rk, ctl, mode, direct_out);
  for (int j = threadIdx.x; j <= Nx / 2; j += blockDim.x) {
    const int cm = (Nx - j) % Nx;
    const int cc[2] = {j, cm};
    double2 D[2][2], H[2][2];
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const int r = P.r[k];
        const size_t q = (size_t)r * Nx + cc[s];
        D[k][s] = w.dph[q];
        const double2 e = w.z[q];
        const double sg = (double)fsign(tb.kx[cc[s]] + tb.ky[r]);
        H[k][s] = make_double2(e.y * sg, -e.x * sg);   // HilbEta^ (2d/breaking.c:252-259)
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (s == 1 && cm == j) continue;
        const int c = cc[s];
        const size_t q = (size_t)P.r[k] * Nx + c;
        const double2 Sd = sym_at(D, P, k, s, c, Nx, Ny, false);
        const double a = tb.aal[q];
        const double2 S = tb.has_src ? w.src[q] : make_double2(0.0, 0.0);
        const double2 de = w.D[q];
        out[q] = make_double2((S.x + Sd.x - de.x) * a, (S.y + Sd.y - de.y) * a);
        const double2 Ed = sym_at(D, P, k, s, c, Nx, Ny, true), Eh = sym_at(H, P, k, s, c, Nx, Ny, true);
        put(sm, M, k, c, make_double2(Ed.x - Eh.y, Ed.y + Eh.x));
      }
  }
  fft_slices<M>(sm, 2, tb.twx, +1);
  for (int k = 0; k < 2; ++k) {
    double2* dst = b.P + (size_t)P.r[k] * Nx;
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) dst[j] = slot(sm, M, k, j);
  }
}

// colI: inverse column FFT -> delphi (real part) and HilbEta (imaginary part) / N
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2b_colI(Tab2 tb, Brk2 b, const Ctl2* __restrict__ ctl, int mode, int cond) {
  if (!rhs_active(ctl, cond) || !brk_update(ctl, mode)) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx;
  const int c = blockIdx.x;
  if (c == 0 && threadIdx.x == 0) b.st->npeaks = 0;
  col_load<M>(sm, 0, b.P, Nx, c);
  fft_slices<M>(sm, 2, tb.twy, +1);
  const double invN = 1.0 / ((double)tb.n);
  for (int y = threadIdx.x; y < M; y += blockDim.x)
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const double2 v = slot(sm, M, k, y);
      b.dh[(size_t)y * Nx + 2 * c + k] = make_double2(v.x * invN, v.y * invN);
    }
}

// peaks: B = 0 and fun_peaks' test on EtaChecked = eta pb.Char at every point
__global__ void k2b_peaks(Tab2 tb, Work2 w, Brk2 b, const Ctl2* __restrict__ ctl, int mode, int cond) {
  if (!rhs_active(ctl, cond) || !brk_update(ctl, mode)) return;
  const int Nx = tb.nx, Ny = tb.ny;
  const size_t n = (size_t)tb.n;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    b.B[q] = 0.0;
    const int i = (int)(q / Nx), j = (int)(q % Nx);   // i: y row, j: x
    const bool ei = (i == 0 || i == Ny - 1), ej = (j == 0 || j == Nx - 1);
    if (ei && ej) continue;
    const double a0 = w.phys[q] * b.pbchar[q];
    if (!(a0 > b.thr)) continue;
    const int di0 = (i == 0) ? 0 : -1, di1 = (i == Ny - 1) ? 0 : 1;
    const int dj0 = (j == 0) ? 0 : -1, dj1 = (j == Nx - 1) ? 0 : 1;
    int cnt = 0;
    for (int di = di0; di <= di1; ++di)
      for (int dj = dj0; dj <= dj1; ++dj) {
        const size_t p = (size_t)(i + di) * Nx + (j + dj);
        cnt += (w.phys[p] * b.pbchar[p] - a0 <= 0.001) ? 1 : 0;
      }
    const int need = (ei || ej) ? 6 : 9;
    if (cnt != need) continue;
    int rank;
    const int I = (Nx - 2) * (Ny - 2);
    if (!ei && !ej) rank = (j - 1) * (Ny - 2) + (i - 1);
    else if (j == 0) rank = I + (i - 1);
    else if (j == Nx - 1) rank = I + (Ny - 2) + (i - 1);
    else if (i == 0) rank = I + 2 * (Ny - 2) + (j - 1);
    else rank = I + 2 * (Ny - 2) + (Nx - 2) + (j - 1);
    const int pos = atomicAdd(&b.st->npeaks, 1);
    if (pos < kBrkPeakCap) b.peaks[pos] = rank;
  }
}

// sort: the peak ranks in ascending order (fun_peaks' visiting order)
__global__ void __launch_bounds__(kBrkSortThreads) k2b_sort(Brk2 b, const Ctl2* __restrict__ ctl, int mode, int cond) {
  if (!rhs_active(ctl, cond) || !brk_update(ctl, mode)) return;
  extern __shared__ int s[];          // kBrkPeakCap ints
  const int np = b.st->npeaks;
  if (np > kBrkPeakCap) {
    if (threadIdx.x == 0) b.st->err |= kBrkErrPeaks;
    return;
  }
  int L = 2;
  while (L < np) L <<= 1;
  for (int i = threadIdx.x; i < L; i += blockDim.x) s[i] = (i < np) ? b.peaks[i] : 0x7fffffff;
  __syncthreads();
  for (int k = 2; k <= L; k <<= 1)
    for (int jj = k >> 1; jj > 0; jj >>= 1) {
      for (int i = threadIdx.x; i < L; i += blockDim.x) {
        const int ixj = i ^ jj;
        if (ixj > i) {
          const bool up = (i & k) == 0;
          const int a = s[i], c = s[ixj];
          if ((a > c) == up) { s[i] = c; s[ixj] = a; }
        }
      }
      __syncthreads();
    }
  for (int i = threadIdx.x; i < np; i += blockDim.x) b.peaks[i] = s[i];
}

// arg-max of eta Char pb.Char over the grid with idx_max_matrix's semantics (start
// from the value at (0,0), keep the first strictly larger value); one warp.
// Returns the row-major index or -1.
__device__ int crest_argmax(const Brk2& b, const Work2& w, const Sector& g, int Nx, int Ny) {
  const int lane = threadIdx.x & 31;
  const double temp0 = w.phys[0] * sector_char(b, g, 0, 0) * b.pbchar[0];
  const int bw = g.j1 - g.j0 + 1, nb = bw * (g.i1 - g.i0 + 1);
  double bv = -INFINITY;
  int bq = 0x7fffffff;
  for (int t = lane; t < nb; t += 32) {
    const int i = g.i0 + t / bw, j = g.j0 + t % bw;
    const size_t q = (size_t)i * Nx + j;
    const double v = w.phys[q] * sector_char(b, g, i, j) * b.pbchar[q];
    if (v > bv) { bv = v; bq = (int)q; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
    const int oq = __shfl_xor_sync(0xffffffffu, bq, o);
    if (ov > bv || (ov == bv && oq < bq)) { bv = ov; bq = oq; }
  }
  const bool whole = (g.i0 == 0 && g.j0 == 0 && g.i1 == Ny - 1 && g.j1 == Nx - 1);
  if (whole || bv > 0) return (bv > temp0) ? bq : -1;
  // every point outside the box is exactly zero: the maximum is 0
  if (!(0.0 > temp0)) return -1;
  const size_t n = (size_t)Nx * Ny;
  for (size_t base = 0; base < n; base += 32) {
    const size_t q = base + lane;
    bool z = false;
    if (q < n) {
      const int i = (int)(q / Nx), j = (int)(q % Nx);
      z = (w.phys[q] * sector_char(b, g, i, j) * b.pbchar[q]) == 0.0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, z);
    if (m) return (int)(base + __ffs(m) - 1);
  }
  return -1;
}

// ---------------------------------------------------------------------------
// machine: breaking_criterion at the sorted peaks and breaking_process; one warp
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(32) k2b_machine(Tab2 tb, Work2 w, Brk2 b, Ctl2* ctl, int mode, int cond) {
  if (!rhs_active(ctl, cond) || !brk_update(ctl, mode)) return;
  const int lane = threadIdx.x;
  const unsigned FULL = 0xffffffffu;
  const unsigned lt = (1u << lane) - 1u;
  const int Nx = tb.nx, Ny = tb.ny;
  const size_t n = (size_t)tb.n;
  BrkSt* S = b.st;
  const double t = stage_time(ctl, mode);
  const double* U2 = w.phys + n;        // u, v (scaled)
  const double* V2 = w.phys + 2 * n;
  if (S->err & (kBrkErrPeaks | kBrkErrCrests | kBrkErrNodes)) {
    if (lane == 0) { ctl->status = kBreakCapacity; ctl->done = 1; }
    return;
  }
  // breaking_criterion: candidates in peak order
  const int npk = S->npeaks;
  int ncb = 0;
  for (int base = 0; base < npk; base += 32) {
    const int p = base + lane;
    bool cand = false;
    Crest2 rec{};
    if (p < npk) {
      int ix, iy;
      rank_to_xy(b.peaks[p], Nx, Ny, ix, iy);
      const size_t q = (size_t)iy * Nx + ix;
      const double e = w.phys[q], h = b.dh[q].y;
      const double* Hy = &b.dh[0].y;
      const double gxH = gxat(Hy, 2, Nx, iy, ix, b.dx), gyH = gyat(Hy, 2, Nx, Ny, iy, ix, b.dy);
      const double gxE = gxat(w.phys, 1, Nx, iy, ix, b.dx), gyE = gyat(w.phys, 1, Nx, Ny, iy, ix, b.dy);
      const double den = ra2(rm2(e, e), rm2(h, h));
      const double Kx = rs2(rm2(e, gxH), rm2(h, gxE)) / den;
      const double Ky = rs2(rm2(e, gyH), rm2(h, gyE)) / den;
      const double Kk = sqrt(ra2(rm2(Kx, Kx), rm2(Ky, Ky)));
      const double D = ra2(-b.bathy[q], e);
      double Cc;   // fun_exact_Cp1d_val
      if (Kk == 0) Cc = ra2(sqrt(rm2(kGrav, D)), b.cur_u);
      else Cc = ra2(fsign(Kk) * sqrt(rm2(rm2(kGrav, Kk), tanh(rm2(Kk, D)))), rm2(Kk, b.cur_u)) / Kk;
      const double u = U2[q], v = V2[q];
      const double Uq = sqrt(ra2(rm2(u, u), rm2(v, v)));
      if (fabs(Uq) >= rm2(b.kbc, fabs(Cc))) {
        cand = true;
        rec.xindex = ix; rec.yindex = iy; rec.xNow = ix; rec.yNow = iy;
        rec.Ucrest = fabs(Uq);
        rec.time = t;
        rec.theta = fabs(atan(v / u));
        rec.kwadran = fun_kwadran(u, v);
      }
    }
    const unsigned m = __ballot_sync(FULL, cand);
    const int pos = ncb + __popc(m & lt);
    if (cand && pos < kBrkCrestCap) b.CB[pos] = rec;
    ncb += __popc(m);
  }
  if (ncb > kBrkCrestCap) {
    if (lane == 0) { S->err |= kBrkErrCrests; ctl->status = kBreakCapacity; ctl->done = 1; }
    return;
  }
  __syncwarp();
  int flag = S->flagbr;
  const int ncp = S->ncbprev;
  int nnew = 0;
  if (ncb > 0 && flag == 0) {
    flag = 1;
    for (int j = lane; j < ncb; j += 32) b.CBNew[j] = b.CB[j];
    nnew = ncb;
  } else if (ncb == 0 && flag == 2) {
    for (int j = lane; j < ncp; j += 32) b.CBNew[j] = b.CBPrev[j];
    nnew = ncp;
  } else if (ncb > 0 && flag == 2) {
    if (ncp + ncb > kBrkCrestCap) {
      if (lane == 0) { S->err |= kBrkErrCrests; ctl->status = kBreakCapacity; ctl->done = 1; }
      return;
    }
    for (int j = lane; j < ncp; j += 32) b.CBNew[j] = b.CBPrev[j];
    const int2* old = b.bn[S->bn_cur];
    int add = 0;
    for (int k = 0; k < ncb; ++k) {
      const int idx = b.CB[k].xindex, idy = b.CB[k].yindex;
      bool seen = false;
      for (int l = lane; l < ncp; l += 32)
        if (b.CBPrev[l].xindex == idx && b.CBPrev[l].yindex == idy) seen = true;
      for (int l = 0; l < ncp; ++l) {
        const int off = b.CBPrev[l].off, nn = b.CBPrev[l].nnode;
        for (int m = lane; m < nn; m += 32) {
          const int2 nd = old[off + m];
          if (nd.x == idx && nd.y == idy) seen = true;
        }
      }
      seen = __any_sync(FULL, seen);
      if (!seen) {
        if (lane == 0) b.CBNew[ncp + add] = b.CB[k];
        ++add;
      }
    }
    nnew = ncp + add;
  }
  __syncwarp();
  bool any_b = false;
  if (flag == 1 || flag == 2) {
    const int wp = S->bn_cur ^ 1;
    int2* pool = b.bn[wp];
    int itpp = 0, itp = 0;
    long long pp_total = 0, bn_total = 0;
    bool cont = false;
    for (int lx = 0; lx < nnew; ++lx) {
      Crest2 r = b.CBNew[lx];
      if (flag == 1) {
        r.xNow = r.xindex;
        r.yNow = r.yindex;
      } else {
        const Sector g0 = sector_of(b, r, Nx, Ny);
        const int qm = crest_argmax(b, w, g0, Nx, Ny);
        if (qm < 0) continue;                               // this crest stops breaking
        r.xNow = qm % Nx;
        r.yNow = qm / Nx;
        const double u = U2[qm], v = V2[qm];
        r.theta = fabs(atan(v / u));
        r.kwadran = fun_kwadran(u, v);
      }
      __syncwarp();
      if (lane == 0) b.CBNew[lx] = r;
      const double tbreak = r.time, UI = r.Ucrest, UF = rm2(b.tc, UI);
      double Ustar;
      const double dtb = rs2(t, tbreak);
      if (dtb >= b.tstar) Ustar = UF;
      else if ((dtb >= 0) && dtb < b.tstar) Ustar = ra2(UI, rm2(dtb / b.tstar, rs2(UF, UI)));
      else Ustar = UI;
      // funBr_BreakNodes_char over the disc's box, in row-major order
      const Sector g = sector_of(b, r, Nx, Ny);
      const int bw = g.j1 - g.j0 + 1, nb = bw * (g.i1 - g.i0 + 1);
      int nbp = 0, nbn = 0;
      for (int base = 0; base < nb; base += 32) {
        const int tt = base + lane;
        bool node = false, brk = false;
        int i = 0, j = 0;
        if (tt < nb) {
          i = g.i0 + tt / bw;
          j = g.j0 + tt % bw;
          const size_t q = (size_t)i * Nx + j;
          double ch = sector_char(b, g, i, j);
          const double uu = U2[q], vv = V2[q];
          const double Uq = sqrt(ra2(rm2(uu, uu), rm2(vv, vv)));
          if ((Uq < UF) || (w.phys[q] < 0)) ch = 0;
          ch = ch * b.pbchar[q];
          if (ch == 1) {
            node = true;
            if (b.B[q] == 0) {
              double Bq;
              if (Uq >= (2 * Ustar)) Bq = 1;
              else if (Uq <= Ustar) Bq = 0;
              else Bq = rs2(Uq / Ustar, 1.0);
              b.B[q] = Bq;
              brk = Bq > 0;
            }
          }
        }
        const unsigned m1 = __ballot_sync(FULL, node), m2 = __ballot_sync(FULL, brk);
        const long long p1 = pp_total + __popc(m1 & lt), p2 = bn_total + __popc(m2 & lt);
        if (node && p1 < b.cap_nodes) b.bnp[p1] = make_int2(j, i);
        if (brk && p2 < b.cap_nodes) pool[p2] = make_int2(j, i);
        pp_total += __popc(m1);
        bn_total += __popc(m2);
        nbp += __popc(m1);
        nbn += __popc(m2);
      }
      if (pp_total > b.cap_nodes || bn_total > b.cap_nodes) {
        if (lane == 0) { S->err |= kBrkErrNodes; ctl->status = kBreakCapacity; ctl->done = 1; }
        return;
      }
      if (nbp > 0) ++itpp;
      if (nbn > 0) {
        cont = true;
        if (lane == 0) {
          Crest2 d = r;
          d.off = (int)(bn_total - nbn);
          d.nnode = nbn;
          b.CBPrev[itp] = d;
        }
        ++itp;
      }
      __syncwarp();
    }
    if (nnew > 0) flag = cont ? 2 : 0;
    any_b = bn_total > 0;
    // breaking.dat: every crest's sector nodes, once per output interval
    if ((t > ra2(b.t0, rm2((double)S->iterbdt, b.dt_out))) && itpp > 0) {
      const int rec = S->nrec;
      const long long off = S->nlog;
      if (rec < b.cap_rec && off + pp_total <= b.cap_log) {
        for (long long m = lane; m < pp_total; m += 32) b.log_nodes[off + m] = b.bnp[m];
        if (lane == 0) {
          b.log_t[rec] = t;
          b.log_cnt[rec] = (int)pp_total;
          S->nrec = rec + 1;
          S->nlog = off + pp_total;
        }
      } else if (lane == 0) {
        S->err |= kBrkErrLog;
      }
    }
    if (lane == 0) {
      S->ncbprev = itp;
      S->bn_cur = wp;
    }
  }
  if (lane == 0) {
    if (t > ra2(b.t0, rm2((double)S->iterbdt, b.dt_out))) S->iterbdt = S->iterbdt + 1;
    S->flagbr = flag;
    S->sb_zero = any_b ? 0 : 1;
  }
}

// flux: Flux = -B delb^2 (eta - bathy) delphi^2 (only when some B > 0)
__global__ void k2b_flux(Tab2 tb, Work2 w, Brk2 b, const Ctl2* __restrict__ ctl, int mode, int cond) {
  if (!rhs_active(ctl, cond) || !brk_update(ctl, mode) || b.st->sb_zero) return;
  const size_t n = (size_t)tb.n;
  const double d2 = rm2(b.delb, b.delb);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const double dp = b.dh[q].x;
    b.flux[q] = rm2(rm2(rm2(-b.B[q], d2), rs2(w.phys[q], b.bathy[q])), rm2(dp, dp));
  }
}

// sbcol: fun_gradient (periodic forward / backward differences, clipped), Sb = grad
// Flux / (eta - bathy), Sb_x + i Sb_y -> forward column FFT
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2b_sbcol(Tab2 tb, Work2 w, Brk2 b, const Ctl2* __restrict__ ctl, int mode, int cond) {
  if (!rhs_active(ctl, cond) || !brk_update(ctl, mode) || b.st->sb_zero) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const int c = blockIdx.x;
  const double* f = b.flux;
  for (int y = threadIdx.x; y < M; y += blockDim.x)
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int x = 2 * c + k;
      const size_t q = (size_t)y * Nx + x;
      const size_t r = (size_t)y * Nx;
      double Fx = (x < Nx - 1) ? rs2(f[q + 1], f[q]) / b.dx : rs2(f[r], f[q]) / b.dx;
      double Fy = (y < Ny - 1) ? rs2(f[q + Nx], f[q]) / b.dy : rs2(f[x], f[q]) / b.dy;
      double Bx = (x > 0) ? rs2(f[q], f[q - 1]) / b.dx : rs2(f[q], f[r + Nx - 1]) / b.dx;
      double By = (y > 0) ? rs2(f[q], f[q - Nx]) / b.dy : rs2(f[q], f[(size_t)(Ny - 1) * Nx + x]) / b.dy;
      if (Fx > 0) Fx = 0;
      if (Fy > 0) Fy = 0;
      if (Bx < 0) Bx = 0;
      if (By < 0) By = 0;
      const double hq = rs2(w.phys[q], b.bathy[q]);
      put(sm, M, k, y, make_double2(ra2(Fx, Bx) / hq, ra2(Fy, By) / hq));
    }
  fft_slices<M>(sm, 2, tb.twy, -1);
  col_store<M>(sm, 0, b.P, Nx, c);
}

// sbrow: forward row FFT and split -> Sb_xhat, Sb_yhat (on an update with B > 0),
// then dt u^ += Sb_xhat aal, dt v^ += Sb_yhat aal whenever Sb is not zero
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2b_sbrow(Tab2 tb, Brk2 b, RK2 rk, const Ctl2* __restrict__ ctl, int mode, int cond, double2* __restrict__ direct_out) {
  if (!rhs_active(ctl, cond) || b.st->sb_zero) return;
  extern __shared__ double2 sm[];
  const int Nx = tb.nx, Ny = tb.ny;
  const size_t n = (size_t)tb.n;
  const Pair P = row_pair(blockIdx.x, Ny);
  const bool upd = brk_update(ctl, mode);
  if (upd) {
    for (int k = 0; k < 2; ++k) {
      const double2* src = b.P + (size_t)P.r[k] * Nx;
      for (int j = threadIdx.x; j < Nx; j += blockDim.x) put(sm, M, k, j, src[j]);
    }
    fft_slices<M>(sm, 2, tb.twx, -1);
  }
  double2* out = rhs_out(rk, ctl, mode, direct_out);
  for (int k = 0; k < 2; ++k) {
    const int r = P.r[k];
    for (int j = threadIdx.x; j < Nx; j += blockDim.x) {
      const size_t q = (size_t)r * Nx + j;
      double2 A, Bv;
      if (upd) {
        split2(slot(sm, M, k, j), slot(sm, M, P.mr[k], (Nx - j) % Nx), A, Bv);
        b.sb[q] = A;
        b.sb[n + q] = Bv;
      } else {
        A = b.sb[q];
        Bv = b.sb[n + q];
      }
      const double a = tb.aal[q];
      const double2 ou = out[n + q], ov = out[2 * n + q];
      out[n + q] = make_double2(ou.x + A.x * a, ou.y + A.y * a);
      out[2 * n + q] = make_double2(ov.x + Bv.x * a, ov.y + Bv.y * a);
    }
  }
}

}  // namespace hw2d
