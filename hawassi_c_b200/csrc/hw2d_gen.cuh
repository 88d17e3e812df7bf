// hw2d_gen.cuh -- the general 2D RHS on a varying bottom: rhs_AB1_2DB_uv,
// rhs_AB2_2DB_uv and rhs_AB3_2DB_uv (2d/fun_odesolver.c:4350-4402, 4542-4626,
// 4735-4844) with their term functions fun_termshat_AB1/AB2/AB3_2DB_uv
// (:2874-2960, 3327-3510, 4104-4296) and the two- or three-reference-depth
// operator HSSgen_2depth / HSSgen_3depth (:500-697), or its sum over K reference depths
// (the plain K-reference operator and the learned 4-depth blend, which the reference
// does not have).
//
// Unlike the fused passes of hw2d_var.cuh (two reference depths, HS1/HS2 only),
// this path runs the reference's sequence of whole-field operations one by one:
// the 2D transforms are a row kernel and a column kernel (M-point Stockham slices
// in shared memory, four slices per CTA), fftwcomplex_2d_sym is one in-place
// kernel, and every pointwise step is a grid-stride kernel over the field.  Its
// fields are full complex N = Nx Ny arrays in the reference's row-major order, in
// one pool owned by the engine.  It serves the combinations the fused passes do
// not cover (three or K reference depths; HS3 on the varying bottom) at the
// reference's own transform count.
#pragma once

#include "hw2d.cuh"

namespace hw2d {

constexpr int kGenThreads = 256;
constexpr int kGenBlocks = 4 * 148;

// ---------------------------------------------------------------------------
// 2D transform building blocks (unnormalised; sign -1 forward, +1 inverse)
// ---------------------------------------------------------------------------
// rows: one CTA per kGroups consecutive rows of field blockIdx.y (M = Nx)
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2g_rows(double2* f, int nx, int ny, const double2* __restrict__ tw, int sign, const Ctl2* __restrict__ ctl,
         int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  double2* F = f + (size_t)blockIdx.y * nx * ny;
  const int r0 = blockIdx.x * kGroups;
  for (int s = 0; s < kGroups; ++s)
    for (int j = threadIdx.x; j < nx; j += blockDim.x) put(sm, M, s, j, F[(size_t)(r0 + s) * nx + j]);
  fft_slices<M>(sm, kGroups, tw, sign);
  for (int s = 0; s < kGroups; ++s)
    for (int j = threadIdx.x; j < nx; j += blockDim.x) F[(size_t)(r0 + s) * nx + j] = slot(sm, M, s, j);
}

// columns: one CTA per two column pairs (four columns) of field blockIdx.y (M = Ny)
template <int M>
__global__ void __launch_bounds__(kGroups * (M / 8), 1)
k2g_cols(double2* f, int nx, int ny, const double2* __restrict__ tw, int sign, const Ctl2* __restrict__ ctl,
         int cond) {
  if (!rhs_active(ctl, cond)) return;
  extern __shared__ double2 sm[];
  double2* F = f + (size_t)blockIdx.y * nx * ny;
  const int c = 2 * blockIdx.x;
  col_load<M>(sm, 0, F, nx, c);
  col_load<M>(sm, 2, F, nx, c + 1);
  fft_slices<M>(sm, 4, tw, sign);
  col_store<M>(sm, 0, F, nx, c);
  col_store<M>(sm, 2, F, nx, c + 1);
}

// fftwcomplex_2d_sym (2d/functions1.c:492-521) in place: the right half of every row
// from the conjugate mirror of the left half, column 0 below row Ny/2 from its upper
// half, the imaginary parts of the four self-conjugate points cleared.  Every write
// reads only points that no write changes, so the points are independent.
__global__ void k2g_sym(double2* f, int nf, int nx, int ny, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  const size_t n = (size_t)nx * ny;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < n * nf; g += (size_t)gridDim.x * blockDim.x) {
    double2* F = f + (g / n) * n;
    const size_t q = g % n;
    const int i = int(q / nx), j = int(q % nx);
    if ((i == 0 || i == ny / 2) && (j == 0 || j == nx / 2)) {
      F[q].y = 0.0;
    } else if (j > nx / 2) {
      const double2 m = F[(size_t)((ny - i) % ny) * nx + (nx - j)];
      F[q] = make_double2(m.x, -m.y);
    } else if (j == 0 && i > ny / 2) {
      const double2 m = F[(size_t)(ny - i) * nx];
      F[q] = make_double2(m.x, -m.y);
    }
  }
}

// pointwise steps: op(q, i, j) over every point of the grid
template <class Op>
__global__ void k2g_map(Op op, size_t n, int nx, const Ctl2* __restrict__ ctl, int cond) {
  if (!rhs_active(ctl, cond)) return;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    op(q, int(q / nx), int(q % nx));
}

// the line signals at the stage time, one value per row (fun_source's INsig_t)
__global__ void k2g_signal(Tab2 tb, Work2 w, const Ctl2* __restrict__ ctl, int mode, int cond) {
  if (!rhs_active(ctl, cond)) return;
  const double ts = stage_time(ctl, mode);
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < tb.ny; r += gridDim.x * blockDim.x) {
    const size_t o = (size_t)r * tb.nt;
    w.insig[r] = spline2(tb.tsig, tb.sig + o, tb.sigc + o, tb.nt, ts);
    w.insigs[r] = spline2(tb.tsig, tb.sigs + o, tb.sigsc + o, tb.nt, ts);
  }
}

// ---------------------------------------------------------------------------
// pointwise operators, each one line of the reference's term functions
// ---------------------------------------------------------------------------
struct OpCopy {   // dst = src
  double2* dst;
  const double2* src;
  __device__ void operator()(size_t q, int, int) const { dst[q] = src[q]; }
};
struct OpScaleTable {   // dst = o src (o a real spectral table): HSSgen's Op_j phi^
  double2* dst;
  const double2* src;
  const double* o;
  __device__ void operator()(size_t q, int, int) const {
    dst[q] = make_double2(o[q] * src[q].x, o[q] * src[q].y);
  }
};
struct OpGam {   // dst = gam re(src) / N (imaginary part 0): HSSgen's gam_j phi / factIFFT
  double2* dst;
  const double2* src;
  const double* gam;
  double N;
  __device__ void operator()(size_t q, int, int) const { dst[q] = make_double2(gam[q] * src[q].x / N, 0.0); }
};
constexpr int kMaxRef2 = 16;   // reference depths of the K-reference operator
struct OpHssSum {   // result = (sum_j gL_j + O_j g_j) / 2 in the reference's order
  double2* res;
  const double2* g[kMaxRef2];
  const double2* gl[kMaxRef2];
  const double* o[kMaxRef2];
  int K;
  __device__ void operator()(size_t q, int, int) const {
    double re = gl[0][q].x + o[0][q] * g[0][q].x, im = gl[0][q].y + o[0][q] * g[0][q].y;
    for (int d = 1; d < K; ++d) {
      re = re + gl[d][q].x + o[d][q] * g[d][q].x;
      im = im + gl[d][q].y + o[d][q] * g[d][q].y;
    }
    res[q] = make_double2(re / 2, im / 2);
  }
};
struct OpDampH1 {   // damping fields and delu H1^, delv H1^ (rhs_AB2_2DB_uv, fun_termshat_AB1_2DB_uv)
  double2 *de, *du, *dv, *h1u, *h1v;
  const double2 *eta, *u, *v, *cu, *cv;
  const double *damp, *kx, *ky;
  double N, g;
  __device__ void operator()(size_t q, int i, int j) const {
    const double dm = damp[q];
    de[q] = make_double2(dm * eta[q].x / N, 0.0);
    du[q] = make_double2(dm * u[q].x / N, 0.0);
    dv[q] = make_double2(dm * v[q].x / N, 0.0);
    h1u[q] = make_double2(cu[q].y / g * kx[j], -cu[q].x / g * kx[j]);
    h1v[q] = make_double2(cv[q].y / g * ky[i], -cv[q].x / g * ky[i]);
  }
};
struct OpM0 {   // M0u = delu H1^, M0v = delv H1^, L phi = their sum (to be symmetrised)
  double2 *m0u, *m0v, *lphi;
  const double2 *h1u, *h1v;
  __device__ void operator()(size_t q, int, int) const {
    m0u[q] = h1u[q];
    m0v[q] = h1v[q];
    lphi[q] = make_double2(h1u[q].x + h1v[q].x, h1u[q].y + h1v[q].y);
  }
};
struct OpH2Products {   // the H2 products in physical space, each x wallchar, and eta u v kept
  double2 *em0u, *eu, *em0v, *ev, *dh2, *em0uh, *em0vh;
  double* phys;   // eta, u, v / N (the breaking kernels' fields), nullptr: not kept
  const double2 *eta, *u, *v, *m0u, *m0v, *lphi;
  const double* wall;
  double N, f2;
  size_t n;
  __device__ void operator()(size_t q, int, int) const {
    const double wc = wall ? wall[q] : 1.0;
    const double e = eta[q].x, uu = u[q].x, vv = v[q].x, lp = lphi[q].x;
    const double a = e * m0u[q].x / f2 * wc, b = e * m0v[q].x / f2 * wc;
    em0u[q] = make_double2(a, 0.0);
    em0uh[q] = make_double2(a, 0.0);
    eu[q] = make_double2(e * uu / f2 * wc, 0.0);
    em0v[q] = make_double2(b, 0.0);
    em0vh[q] = make_double2(b, 0.0);
    ev[q] = make_double2(e * vv / f2 * wc, 0.0);
    dh2[q] = make_double2(0.5 * ((uu * uu + vv * vv) - lp * lp) / f2 * wc, 0.0);
    if (phys) {
      phys[q] = e / N;
      phys[n + q] = uu / N;
      phys[2 * n + q] = vv / N;
    }
  }
};
struct OpScaleRe {   // re(a) *= N (fun_termshat's "for operator" rescaling)
  double2* a;
  double N;
  __device__ void operator()(size_t q, int, int) const { a[q].x = a[q].x * N; }
};
struct OpDelH2 {   // ikx, iky of deletaH2^ and delu, delv (fun_termshat_AB2_2DB_uv)
  double2 *ikx, *iky, *delu, *delv;
  const double2 *dh2, *eu, *ev, *lu, *lv;
  const double *kx, *ky;
  double g;
  __device__ void operator()(size_t q, int i, int j) const {
    const double a = kx[j], b = ky[i];
    ikx[q] = make_double2(-a * dh2[q].y, a * dh2[q].x);
    iky[q] = make_double2(-b * dh2[q].y, b * dh2[q].x);
    delu[q] = make_double2(a * eu[q].y - lu[q].x / g, -a * eu[q].x - lu[q].y / g);
    delv[q] = make_double2(b * ev[q].y - lv[q].x / g, -b * ev[q].x - lv[q].y / g);
  }
};
struct OpChi {   // fun_adjust: A ChiAdj / N after the inverse transform
  double2* a;
  const double* chi;
  double N;
  __device__ void operator()(size_t q, int, int) const {
    a[q] = make_double2(a[q].x * chi[q] / N, a[q].y * chi[q] / N);
  }
};
struct OpH3Pre {   // HS3 inputs (fun_termshat_AB3_2DB_uv): L(eta M0u)/g ..., eta^2 M0u, d_x u, d_y v
  double2 *lmu, *lmv, *lelp, *divg, *e2m0u, *e2m0v, *dxu, *dyv;
  const double2 *lu, *lv, *z, *eta, *m0u, *m0v;
  const double *kx, *ky, *wall;
  double g, f3;
  size_t n;
  __device__ void operator()(size_t q, int i, int j) const {
    const double wc = wall ? wall[q] : 1.0;
    const double2 a = make_double2(lu[q].x / g, lu[q].y / g), b = make_double2(lv[q].x / g, lv[q].y / g);
    lmu[q] = a;
    lmv[q] = b;
    lelp[q] = make_double2(a.x + b.x, a.y + b.y);
    const double2 zu = z[n + q], zv = z[2 * n + q];
    const double X = kx[j], Y = ky[i];
    divg[q] = make_double2(-X * zu.y - Y * zv.y, X * zu.x + Y * zv.x);
    const double e = eta[q].x;
    e2m0u[q] = make_double2(e * e * m0u[q].x / f3 * wc, 0.0);
    e2m0v[q] = make_double2(e * e * m0v[q].x / f3 * wc, 0.0);
    dxu[q] = make_double2(-X * zu.y, X * zu.x);
    dyv[q] = make_double2(-Y * zv.y, Y * zv.x);
  }
};
struct OpH3Products {   // the cubic products p0..p3 (and their copies for the transforms), deletaH3
  double2 *p[4], *ph[4], *dh3;
  const double2 *eta, *lmu, *lmv, *dxu, *dyv, *lphi, *divg, *lelp;
  const double* wall;
  double N, f3;
  __device__ void operator()(size_t q, int, int) const {
    const double wc = wall ? wall[q] : 1.0;
    const double e = eta[q].x;
    const double v0 = e / N * lmu[q].x / N, v1 = e / N * lmv[q].x / N;
    const double v2 = e * e * dxu[q].x / f3 * wc, v3 = e * e * dyv[q].x / f3 * wc;
    const double vals[4] = {v0, v1, v2, v3};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      p[k][q] = make_double2(vals[k], 0.0);
      ph[k][q] = make_double2(vals[k], 0.0);
    }
    dh3[q] = make_double2(lphi[q].x / N * e / N * divg[q].x / N + lphi[q].x / N * lelp[q].x / N, 0.0);
  }
};
struct OpDelH3 {   // ikx3, iky3 and delu3, delv3 (fun_termshat_AB3_2DB_uv)
  double2 *ikx, *iky, *delu, *delv;
  const double2 *dh3, *lp0, *lp1, *lp2, *lp3, *e2m0u, *e2m0v;
  const double *kx, *ky;
  double g;
  __device__ void operator()(size_t q, int i, int j) const {
    const double a = kx[j], b = ky[i];
    ikx[q] = make_double2(-a * dh3[q].y, a * dh3[q].x);
    iky[q] = make_double2(-b * dh3[q].y, b * dh3[q].x);
    delu[q] = make_double2(lp0[q].x / g + 0.5 * lp2[q].x / g - 0.5 * (a * a * e2m0u[q].x),
                           lp0[q].y / g + 0.5 * lp2[q].y / g - 0.5 * (a * a * e2m0u[q].y));
    delv[q] = make_double2(lp1[q].x / g + 0.5 * lp3[q].x / g - 0.5 * (b * b * e2m0v[q].x),
                           lp1[q].y / g + 0.5 * lp3[q].y / g - 0.5 * (b * b * e2m0v[q].y));
  }
};
struct OpSource {   // the line source after its row transform (a set-up table): fac INsig gx + INsig_skew sx
  double2* s;
  const double2 *gx, *sx;
  const double *ins, *inss;
  double fac;
  __device__ void operator()(size_t q, int i, int) const {
    const double a = fac * ins[i], b = inss[i];
    s[q] = make_double2(a * gx[q].x + b * sx[q].x, a * gx[q].y + b * sx[q].y);
  }
};
struct OpAssemble {   // dt Z of rhs_AB1/AB2/AB3_2DB_uv (the breaking force is added after)
  double2* out;       // 3 fields: the direct RHS's output (mode 0); the stepper's modes
  RK2 rk;             // write the RK buffer rhs_out selects from the control block
  const Ctl2* ctl;
  int mode;
  double2* dph;       // delphiH^ kept for the breaking kernels (nullptr: off)
  const double2 *z, *src, *h1u, *h1v, *au, *av, *au3, *av3, *ikx, *iky, *ikx3, *iky3, *de, *du, *dv;
  const double *aal, *kx, *ky;
  double g;
  int model;
  size_t n;
  __device__ void operator()(size_t q, int i, int j) const {
    double2* out = rhs_out(rk, ctl, mode, this->out);
    const double a = aal[q];
    const double2 S = src ? src[q] : make_double2(0.0, 0.0);
    const double2 ze = z[q];
    double2 dphi;
    if (model == 1) {
      dphi = make_double2(h1u[q].x + h1v[q].x, h1u[q].y + h1v[q].y);
    } else if (model == 3) {
      dphi = make_double2(h1u[q].x + h1v[q].x + au[q].x + av[q].x + au3[q].x + av3[q].x,
                          h1u[q].y + h1v[q].y + au[q].y + av[q].y + au3[q].y + av3[q].y);
    } else {
      dphi = make_double2(h1u[q].x + h1v[q].x + au[q].x + av[q].x, h1u[q].y + h1v[q].y + au[q].y + av[q].y);
    }
    if (dph) dph[q] = dphi;
    out[q] = make_double2((S.x + dphi.x - de[q].x) * a, (S.y + dphi.y - de[q].y) * a);
    const double X = kx[j], Y = ky[i];
    if (model == 1) {
      out[n + q] = make_double2((g * X * ze.y - du[q].x) * a, (-g * X * ze.x - du[q].y) * a);
      out[2 * n + q] = make_double2((g * Y * ze.y - dv[q].x) * a, (-g * Y * ze.x - dv[q].y) * a);
    } else if (model == 3) {
      out[n + q] = make_double2((g * X * ze.y - ikx[q].x - ikx3[q].x - du[q].x) * a,
                                (-g * X * ze.x - ikx[q].y - ikx3[q].y - du[q].y) * a);
      out[2 * n + q] = make_double2((g * Y * ze.y - iky[q].x - iky3[q].x - dv[q].x) * a,
                                    (-g * Y * ze.x - iky[q].y - iky3[q].y - dv[q].y) * a);
    } else {
      out[n + q] = make_double2((g * X * ze.y - ikx[q].x - du[q].x) * a, (-g * X * ze.x - ikx[q].y - du[q].y) * a);
      out[2 * n + q] = make_double2((g * Y * ze.y - iky[q].x - dv[q].x) * a, (-g * Y * ze.x - iky[q].y - dv[q].y) * a);
    }
  }
};

}  // namespace hw2d
