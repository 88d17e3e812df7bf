// hw_kin.cu -- kinematics of the 1D model on the device (kinematic_modul,
// 1d/kinematic_modul.c:1-247, with the grid of read_kinematics,
// 1d/functions.c:3555-3669).
//
// At an output sample the reference forms, from the spectral state (eta^, u^) and
// its RHS dy: eta and d eta/dt in physical space; the local depth H = eta + d and
// its two-depth weights (natural cubic splines over 101 total depths between
// Hmin = minEta + minD and Hplus = maxEta + maxD, sinhcosh2IP); then at every
// output level z four spectra (factor, dt phi, dz phi, dx phi: phi^ times the
// cosh/sinh(k (z + d)) / cosh(k H) ratios, with k and H taken at the same index
// as the reference does) and their inverse transforms; on the window it combines
// them (d phi/dt + d eta/dt factor, dx phi + dH/dx factor + dD/dx dz phi), masks
// points above the surface or below the bed with NaN, and forms the pressure
// -dt phi - g z - (dx phi^2 + 2 dz phi)/2 and the accelerations
// (velocity - 0) / (t - tprev), all as the reference writes them.
//
// Device work per sample: one packed inverse transform for eta and d eta/dt, a
// pointwise pass for H and its weights, one pass that builds every level's four
// spectra packed two per complex transform (the real part of an inverse transform
// is the transform of the Hermitian part, so E(A) + i E(B) carries two), 2 nz
// transforms in one launch (one CTA each, radix-2 Stockham through L2), and the
// output pass.  Static tables (levels, window, cosh/sinh of every level, the
// spline knots and coefficients) are built once on the host.
#include "hw_kin.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace hwkin {

namespace {

constexpr double kG = 9.80665;   // 1d/header.h:27
constexpr int kNH = 100;         // total-depth samples of the weights (kinematic_modul.c:10)
constexpr int kFftThreads = 512;

struct KinDev {
  int N, logN, nz, nxo, i1;
  double dx, inv_n;
  const double* k;         // [N] wavenumbers (FFTW order)
  const double* depth;     // [N]
  const double* gradD;     // [N] gradient(depth)
  const double* zout;      // [nz]
  const double* ch_min;    // [N] cosh(k Hmin), cosh(k Hplus), tanh(k Hmin), tanh(k Hplus)
  const double* ch_plus;
  const double* th_min;
  const double* th_plus;
  const double* cz;        // [nz][N] cosh(k (z + d)) (or its two-depth blend)
  const double* sz;        // [nz][N] sinh
  const double* Ht;        // [kNH+1] knots and natural-spline data of the weights
  const double* gm;
  const double* gp;
  const double* cm;
  const double* cp;
  const double2* tw;       // [N] exp(-2 pi i q / N)
  double2* P0;             // [N] packed eta + i dteta (spectral, then physical)
  double2* phi;            // [N] phi^
  double2* dphi;           // [N] dt phi^
  double* eta;             // [N] physical eta, d eta / dt, cosh(kH), tanh(kH), dH/dx
  double* dteta;
  double* coshH;
  double* tanhH;
  double* gradH;
  double2* spec;           // [2 nz][N] packed spectra (then physical)
  double2* scratch;        // [(2 nz + 1)][N] Stockham ping-pong
  double* out_eta;         // [nxo]
  double* out;             // [5][nxo][nz]: P, dxphi, dzphi, dtdxphi, dtdzphi
};

__device__ __forceinline__ double2 herm_pack(double2 a, double2 am, double2 b, double2 bm) {
  // E(A) + i E(B) at a point, given A, B there (a, b) and at the mirror (am, bm)
  const double2 ea = make_double2(0.5 * (a.x + am.x), 0.5 * (a.y - am.y));
  const double2 eb = make_double2(0.5 * (b.x + bm.x), 0.5 * (b.y - bm.y));
  return make_double2(ea.x - eb.y, ea.y + eb.x);
}

// the output stage's spectra (1d/functions.c:570-590): eta^ + i dteta^ packed,
// phi^ = u^ / (i k) and dt phi^ = du^ / (i k) as prod_1ik(-1/k, .)
__global__ void k_kin_prep(KinDev K, const double* __restrict__ y, const double* __restrict__ dy) {
  const int N = K.N;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const int m = (N - j) % N;
    const double2 e = make_double2(y[j], y[N + j]), em = make_double2(y[m], y[N + m]);
    const double2 d = make_double2(dy[j], dy[N + j]), dm = make_double2(dy[m], dy[N + m]);
    K.P0[j] = herm_pack(e, em, d, dm);
    const double kj = K.k[j];
    if (kj == 0) {
      K.phi[j] = make_double2(0.0, 0.0);
      K.dphi[j] = make_double2(0.0, 0.0);
    } else {
      const double ur = y[2 * N + j], ui = y[3 * N + j];
      K.phi[j] = make_double2(ui / kj, -ur / kj);
      const double a = -1 / kj;
      K.dphi[j] = make_double2(__dsub_rn(__dmul_rn(0.0, dy[2 * N + j]), __dmul_rn(a, dy[3 * N + j])),
                               __dadd_rn(__dmul_rn(0.0, dy[3 * N + j]), __dmul_rn(a, dy[2 * N + j])));
    }
  }
}

// batched inverse FFT (exponent +1, unnormalised), one CTA per transform: radix-2
// Stockham passes alternating between the data and a scratch copy in L2
__global__ void __launch_bounds__(kFftThreads) k_kin_ifft(double2* data, double2* scratch, int N, int logN,
                                                           const double2* __restrict__ tw) {
  double2* src = data + (size_t)blockIdx.x * N;
  double2* dst = scratch + (size_t)blockIdx.x * N;
  double2* base = src;
  const int half = N >> 1;
  for (int s = 0; s < logN; ++s) {
    const int Ns = 1 << s;
    const int stride = N / (2 * Ns);
    for (int j = threadIdx.x; j < half; j += blockDim.x) {
      const int kk = j & (Ns - 1);
      const double2 v0 = src[j], v1 = src[j + half];
      const double2 w = tw[kk * stride];                          // exp(-i pi kk / Ns)
      const double2 t = make_double2(v1.x * w.x + v1.y * w.y, v1.y * w.x - v1.x * w.y);   // v1 conj(w)
      const int d = ((j - kk) << 1) + kk;
      dst[d] = make_double2(v0.x + t.x, v0.y + t.y);
      dst[d + Ns] = make_double2(v0.x - t.x, v0.y - t.y);
    }
    __syncthreads();
    double2* tmp = src;
    src = dst;
    dst = tmp;
  }
  if (src != base) {
    for (int j = threadIdx.x; j < N; j += blockDim.x) base[j] = src[j];
  }
}

// GSL natural cubic spline evaluation (binary search, then the cubic); NaN outside
__device__ __forceinline__ double spline_at(const double* __restrict__ xs, const double* __restrict__ ys,
                                            const double* __restrict__ cs, int n, double x) {
  if (x < xs[0] || x > xs[n - 1]) return NAN;   // outside the knots (GSL_EDOM)
  int lo = 0, hi = n - 1;
  while (hi > lo + 1) {
    const int i = (hi + lo) / 2;
    if (xs[i] > x) hi = i; else lo = i;
  }
  const double xl = xs[lo], xh = xs[lo + 1], yl = ys[lo], yh = ys[lo + 1];
  const double h = xh - xl, dy = yh - yl, dxx = x - xl;
  const double ci = cs[lo], cip = cs[lo + 1];
  const double bi = dy / h - h * (cip + 2.0 * ci) / 3.0;
  const double di = (cip - ci) / (3.0 * h);
  return yl + dxx * (bi + dxx * (ci + dxx * di));
}

// eta, d eta/dt; H = eta + d, its weights, cosh(kH), tanh(kH) at the same index, dH/dx
__global__ void k_kin_fields(KinDev K) {
  const int N = K.N;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const double2 p = K.P0[j];
    const double e = p.x * K.inv_n;
    K.eta[j] = e;
    K.dteta[j] = p.y * K.inv_n;
    const double H = e + K.depth[j];
    const double gmv = spline_at(K.Ht, K.gm, K.cm, kNH + 1, H);
    const double gpv = spline_at(K.Ht, K.gp, K.cp, kNH + 1, H);
    K.coshH[j] = gmv * K.ch_min[j] + gpv * K.ch_plus[j];
    K.tanhH[j] = gmv * K.th_min[j] + gpv * K.th_plus[j];
    auto Hat = [&](int i) { return K.P0[i].x * K.inv_n + K.depth[i]; };
    double g;
    if (j == 0) g = (Hat(1) - Hat(0)) / K.dx;
    else if (j == N - 1) g = (Hat(N - 1) - Hat(N - 2)) / K.dx;
    else g = (Hat(j + 1) - Hat(j - 1)) / (2 * K.dx);
    K.gradH[j] = g;
  }
}

// every level's spectra, packed: spec[2 zz] = E(factor) + i E(dt phi),
// spec[2 zz + 1] = E(dz phi) + i E(dx phi)
__device__ __forceinline__ void level_spectra(const KinDev& K, int zz, int j, double2& fa, double2& ft, double2& fz,
                                              double2& fx) {
  const double kj = K.k[j], cH = K.coshH[j], tH = K.tanhH[j];
  const double cz = K.cz[(size_t)zz * K.N + j], sz = K.sz[(size_t)zz * K.N + j];
  const double ratio = cz / cH;
  const double2 ph = K.phi[j], dp = K.dphi[j];
  const double f = -kj * tH;
  fa = make_double2(ph.x * ratio * f, ph.y * ratio * f);
  ft = make_double2(dp.x * ratio, dp.y * ratio);
  fz = make_double2(ph.x * kj * sz / cH, ph.y * kj * sz / cH);
  fx = make_double2(-kj * ph.y * ratio, kj * ph.x * ratio);
}

__global__ void k_kin_spectra(KinDev K) {
  const int N = K.N;
  const int zz = blockIdx.y;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const int m = (N - j) % N;
    double2 a, b, c, d, am, bm, cm, dm;
    level_spectra(K, zz, j, a, b, c, d);
    level_spectra(K, zz, m, am, bm, cm, dm);
    K.spec[(size_t)(2 * zz) * N + j] = herm_pack(a, am, b, bm);
    K.spec[(size_t)(2 * zz + 1) * N + j] = herm_pack(c, cm, d, dm);
  }
}

// the window: combination, masks, pressure, accelerations ([nxo][nz], x-major)
__global__ void k_kin_out(KinDev K, double t, double tprev) {
  const int nz = K.nz, nxo = K.nxo, N = K.N;
  const size_t cnt = (size_t)nz * nxo, plane = cnt;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < cnt; q += (size_t)gridDim.x * blockDim.x) {
    const int xo = (int)(q / nz), zz = (int)(q % nz);
    const int j = K.i1 + xo;
    const double zo = K.zout[zz];
    const double2 A = K.spec[(size_t)(2 * zz) * N + j], B = K.spec[(size_t)(2 * zz + 1) * N + j];
    const double fac = A.x * K.inv_n, tdt = A.y * K.inv_n, tdz = B.x * K.inv_n, tdx = B.y * K.inv_n;
    double vt, vx, vz;
    if ((zo > K.eta[j]) || (zo < -K.depth[j])) {
      vt = NAN; vx = NAN; vz = NAN;
    } else {
      vt = tdt + K.dteta[j] * fac;
      vx = tdx + K.gradH[j] * fac + K.gradD[j] * tdz;
      vz = tdz;
    }
    K.out[q] = -vt - kG * zo - 0.5 * (vx * vx + 2 * vz);
    K.out[plane + q] = vx;
    K.out[2 * plane + q] = vz;
    K.out[3 * plane + q] = (vx - 0) / (t - tprev);
    K.out[4 * plane + q] = (vz - 0) / (t - tprev);
    if (zz == 0) K.out_eta[xo] = K.eta[j];
  }
}

// sinhcosh2IP (1d/functions.c:1889-1928)
void sinhcosh2ip(const std::vector<double>& D, double Dmin, double Dplus, const std::vector<double>& k, double nupeak,
                 std::vector<double>& gmin, std::vector<double>& gplus) {
  const size_t n = D.size();
  gmin.resize(n);
  gplus.resize(n);
  for (size_t j = 0; j < n; ++j) {
    const double kap = (D[j] == 0) ? k[2] : hw::linear_wavenumber(nupeak, D[j]);
    const double cmin = std::cosh(kap * Dmin), cplus = std::cosh(kap * Dplus), cD = std::cosh(kap * D[j]);
    const double smin = std::sinh(kap * Dmin), splus = std::sinh(kap * Dplus), sD = std::sinh(kap * D[j]);
    const double det = cmin * splus - cplus * smin;
    gmin[j] = (splus * cD - cplus * sD) / det;
    gplus[j] = (-(smin * cD) + cmin * sD) / det;
  }
}

}  // namespace

struct Kin {
  KinDev d{};
  double* yref = nullptr;    // [4N] state and RHS in the reference layout
  double* dyref = nullptr;
  std::vector<void*> allocs;
  std::vector<double> xo, zo;
  template <class T>
  T* alloc(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
    allocs.push_back(p);
    return static_cast<T*>(p);
  }
  template <class T>
  const T* upload(const std::vector<T>& v) {
    T* p = alloc<T>(v.size());
    if (p && cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
    return p;
  }
  ~Kin() {
    for (void* p : allocs) cudaFree(p);
  }
};

Kin* kin_create(const hw::Member& m, std::string& err) {
  const hw::Deck& dk = m.deck;
  const int N = m.Nx;
  if (dk.kinematic != "yes") { err = "the deck has kinematic no"; return nullptr; }
  if (dk.nsurf < 2 || dk.ndeep < 1) { err = "kinematics: nsurf must be >= 2 and ndeep >= 1"; return nullptr; }
  if (N < 4 || (N & (N - 1))) { err = "kinematics: Nx must be a power of two"; return nullptr; }
  for (double v : m.depth)
    if (v == 0) { err = "kinematics: runup (zero depth) is not supported"; return nullptr; }
  // read_kinematics
  double zs1, zs2;
  if (dk.min_z == "default") {
    zs1 = -2.5 * m.Hs_in;
    if (dk.initial == "user_defined") zs1 = -0.6 * m.Hs_in;
  } else {
    zs1 = std::atof(dk.min_z.c_str());
  }
  if (dk.max_z == "default") {
    zs2 = 2.5 * m.Hs_in;
    if (dk.initial == "user_defined") zs2 = 0.6 * m.Hs_in;
  } else {
    zs2 = std::atof(dk.max_z.c_str());
  }
  double maxD = m.depth[0], minD = m.depth[0];
  for (double v : m.depth) { if (v > maxD) maxD = v; if (v < minD) minD = v; }
  const int i1 = hw::closest_index(m.x, dk.xinterv1), i2 = hw::closest_index(m.x, dk.xinterv2);
  const int nxo = i2 - i1 + 1;
  if (nxo < 1) { err = "kinematics: empty overlay window"; return nullptr; }
  const int ns = dk.nsurf, nd = dk.ndeep, nz = ns + nd;
  const double maxEta = zs2, minEta = zs1;
  const double dzs = (maxEta - minEta) / (ns - 1);
  const double kpk = hw::linear_wavenumber(m.nu_peak, maxD);
  std::vector<double> zs(ns), zd(nd), z(nz);
  for (int j = 0; j < ns; ++j) zs[j] = minEta + j * dzs;
  const double Flux = 1 / (kpk * std::sinh(kpk * maxD)) * (std::cosh(kpk * (maxD + minEta)) - 1);
  const double tol = Flux / nd;
  zd[0] = -1 * (minEta - dzs);
  for (int i = 1; i < nd; ++i) zd[i] = zd[i - 1] + (tol / (std::sinh(kpk * (maxD - zd[i - 1])) / std::sinh(kpk * maxD)));
  for (int i = 0; i < ns; ++i) z[i] = zs[i];
  for (int i = ns; i < nz; ++i) z[i] = -1 * zd[i - ns];
  for (int i = 0; i < nz; ++i)
    for (int j = i + 1; j < nz; ++j)
      if (z[j] < z[i]) std::swap(z[i], z[j]);
  // kinematic_modul's static part (its tables do not depend on the state)
  const double Hplus = maxEta + maxD, Hmin = minEta + minD;
  const double dhtot = (Hplus - Hmin) / kNH;
  std::vector<double> Ht(kNH + 1), DZt(kNH + 1), gHm, gHp, gDm, gDp;
  for (int i = 0; i < kNH + 1; ++i) Ht[i] = Hmin + i * dhtot;
  sinhcosh2ip(Ht, Hmin, Hplus, m.k, m.nu_peak, gHm, gHp);
  const double DZmin0 = 0, DZplus0 = Hplus;
  for (int i = 0; i < kNH + 1; ++i) DZt[i] = DZmin0 + i * (DZplus0 - DZmin0) / kNH;
  sinhcosh2ip(DZt, DZmin0, DZplus0, m.k, m.nu_peak, gDm, gDp);
  const std::vector<double> cHm = hw::natural_spline_c(Ht, gHm), cHp = hw::natural_spline_c(Ht, gHp);
  const std::vector<double> cDm = hw::natural_spline_c(DZt, gDm), cDp = hw::natural_spline_c(DZt, gDp);
  std::vector<double> chm(N), chp(N), thm(N), thp(N), gD(N);
  for (int j = 0; j < N; ++j) {
    chm[j] = std::cosh(m.k[j] * Hmin);
    chp[j] = std::cosh(m.k[j] * Hplus);
    thm[j] = std::tanh(m.k[j] * Hmin);
    thp[j] = std::tanh(m.k[j] * Hplus);
  }
  gD[0] = (m.depth[1] - m.depth[0]) / m.dx;
  gD[N - 1] = (m.depth[N - 1] - m.depth[N - 2]) / m.dx;
  for (int j = 1; j < N - 1; ++j) gD[j] = (m.depth[j + 1] - m.depth[j - 1]) / (2 * m.dx);
  std::vector<double> cz((size_t)nz * N), sz((size_t)nz * N), DZ(N);
  const bool flatb = (minD == maxD);
  for (int zz = 0; zz < nz; ++zz) {
    double* c = cz.data() + (size_t)zz * N;
    double* s = sz.data() + (size_t)zz * N;
    const double zo = z[zz];
    bool direct = flatb;
    double DZmin = 0, DZplus = 0;
    if (!flatb) {
      for (int j = 0; j < N; ++j) { DZ[j] = m.depth[j] + zo; if (DZ[j] < 0) DZ[j] = 0; }
      DZplus = DZ[0]; DZmin = DZ[0];
      for (int j = 0; j < N; ++j) { if (DZ[j] > DZplus) DZplus = DZ[j]; if (DZ[j] < DZmin) DZmin = DZ[j]; }
      if (DZmin < 0) DZmin = 0;
      direct = (DZmin == DZplus);
    }
    for (int j = 0; j < N; ++j) {
      if (direct) {
        c[j] = std::cosh(m.k[j] * (zo + m.depth[0]));
        s[j] = std::sinh(m.k[j] * (zo + m.depth[0]));
      } else {
        double gm = hw::natural_spline_eval(DZt, gDm, cDm, DZ[j]);
        double gp = hw::natural_spline_eval(DZt, gDp, cDp, DZ[j]);
        if (DZ[j] == DZmin) { gm = 1; gp = 0; }
        if (DZ[j] == DZplus) { gm = 0; gp = 1; }
        c[j] = gm * std::cosh(m.k[j] * DZmin) + gp * std::cosh(m.k[j] * DZplus);
        s[j] = gm * std::sinh(m.k[j] * DZmin) + gp * std::sinh(m.k[j] * DZplus);
      }
    }
  }
  std::vector<double2> tw(N);
  for (int q = 0; q < N; ++q) {
    const double a = 2.0 * M_PI * double(q) / double(N);
    tw[q] = make_double2(std::cos(a), -std::sin(a));
  }
  auto* K = new Kin();
  KinDev& d = K->d;
  d.N = N;
  d.logN = 0;
  while ((1 << d.logN) < N) ++d.logN;
  d.nz = nz; d.nxo = nxo; d.i1 = i1; d.dx = m.dx; d.inv_n = 1.0 / double(N);
  d.k = K->upload(m.k); d.depth = K->upload(m.depth); d.gradD = K->upload(gD); d.zout = K->upload(z);
  d.ch_min = K->upload(chm); d.ch_plus = K->upload(chp); d.th_min = K->upload(thm); d.th_plus = K->upload(thp);
  d.cz = K->upload(cz); d.sz = K->upload(sz);
  d.Ht = K->upload(Ht); d.gm = K->upload(gHm); d.gp = K->upload(gHp); d.cm = K->upload(cHm); d.cp = K->upload(cHp);
  d.tw = K->upload(tw);
  d.P0 = K->alloc<double2>(N); d.phi = K->alloc<double2>(N); d.dphi = K->alloc<double2>(N);
  d.eta = K->alloc<double>(N); d.dteta = K->alloc<double>(N); d.coshH = K->alloc<double>(N);
  d.tanhH = K->alloc<double>(N); d.gradH = K->alloc<double>(N);
  d.spec = K->alloc<double2>((size_t)2 * nz * N);
  d.scratch = K->alloc<double2>((size_t)(2 * nz + 1) * N);
  d.out_eta = K->alloc<double>(nxo);
  d.out = K->alloc<double>((size_t)5 * nxo * nz);
  K->yref = K->alloc<double>((size_t)4 * N);
  K->dyref = K->alloc<double>((size_t)4 * N);
  const bool ok = K->yref && K->dyref && d.k && d.depth && d.gradD && d.zout && d.ch_min && d.ch_plus && d.th_min && d.th_plus && d.cz &&
                  d.sz && d.Ht && d.gm && d.gp && d.cm && d.cp && d.tw && d.P0 && d.phi && d.dphi && d.eta &&
                  d.dteta && d.coshH && d.tanhH && d.gradH && d.spec && d.scratch && d.out_eta && d.out;
  if (!ok) {
    err = "kinematics: device allocation failed";
    delete K;
    return nullptr;
  }
  K->xo.assign(m.x.begin() + i1, m.x.begin() + i1 + nxo);
  K->zo = z;
  return K;
}

void kin_destroy(Kin* k) { delete k; }

double* kin_state_buffer(Kin* k, int which) { return which ? k->dyref : k->yref; }

void kin_dims(const Kin* k, int* nx_out, int* nz_out) {
  if (nx_out) *nx_out = k->d.nxo;
  if (nz_out) *nz_out = k->d.nz;
}

void kin_grid(const Kin* k, double* x_out, double* z_out) {
  if (x_out) std::copy(k->xo.begin(), k->xo.end(), x_out);
  if (z_out) std::copy(k->zo.begin(), k->zo.end(), z_out);
}

bool kin_run(Kin* k, const double* d_y, const double* d_dy, double t, double tprev, cudaStream_t s, std::string& err) {
  KinDev& d = k->d;
  const int blocks = std::min(592, (d.N + 255) / 256);
  k_kin_prep<<<blocks, 256, 0, s>>>(d, d_y, d_dy);
  k_kin_ifft<<<1, kFftThreads, 0, s>>>(d.P0, d.scratch, d.N, d.logN, d.tw);
  k_kin_fields<<<blocks, 256, 0, s>>>(d);
  k_kin_spectra<<<dim3(std::max(1, std::min(64, (d.N + 255) / 256)), d.nz), 256, 0, s>>>(d);
  k_kin_ifft<<<2 * d.nz, kFftThreads, 0, s>>>(d.spec, d.scratch, d.N, d.logN, d.tw);
  const size_t cnt = (size_t)d.nz * d.nxo;
  k_kin_out<<<(unsigned)std::min<size_t>(592, (cnt + 255) / 256), 256, 0, s>>>(d, t, tprev);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    err = std::string("kinematics: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

bool kin_fetch(Kin* k, double* eta_cut, double* P, double* dxphi, double* dzphi, double* dtdxphi, double* dtdzphi,
               cudaStream_t s, std::string& err) {
  const KinDev& d = k->d;
  const size_t plane = (size_t)d.nxo * d.nz;
  double* outs[5] = {P, dxphi, dzphi, dtdxphi, dtdzphi};
  if (eta_cut && cudaMemcpyAsync(eta_cut, d.out_eta, sizeof(double) * d.nxo, cudaMemcpyDeviceToHost, s) != cudaSuccess) {
    err = "kinematics: copy failed";
    return false;
  }
  for (int f = 0; f < 5; ++f)
    if (outs[f] &&
        cudaMemcpyAsync(outs[f], d.out + f * plane, sizeof(double) * plane, cudaMemcpyDeviceToHost, s) != cudaSuccess) {
      err = "kinematics: copy failed";
      return false;
    }
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    err = std::string("kinematics: ") + cudaGetErrorString(cudaGetLastError());
    return false;
  }
  return true;
}

}  // namespace hwkin
