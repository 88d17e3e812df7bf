// hw_setup.cpp -- host set-up of one HAWASSI 1D member: input.txt parsing,
// influx loading/synthesis, domain and wavenumber grid, damping zones,
// influx source kernel, nonlinear-adjustment mask, dispersion operators
// (flat, or interpolated over reference depths), aliasing mask, breaking
// parameters and the initial spectral state.  Citations are to the reference
// project's 1d/ sources.
#include "hw_setup.hpp"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>

namespace hw {
namespace {

constexpr double kG = 9.80665;      // 1d/header.h:27
const double kPi = 4.0 * std::atan(1.0);  // 1d/header.h:28

using cplx = std::complex<double>;

// ----------------------------------------------------------------------------
// Host FFT: radix-2 for powers of two, recursive mixed radix otherwise,
// Bluestein for large prime factors.  Only used during set-up.
// ----------------------------------------------------------------------------
struct Twiddles {
  int n;
  std::vector<cplx> w;  // exp(+2 pi i j / n)
  explicit Twiddles(int n_) : n(n_), w(n_) {
    for (int j = 0; j < n; ++j) {
      double a = 2.0 * kPi * double(j) / double(n);
      w[j] = cplx(std::cos(a), std::sin(a));
    }
  }
  cplx at(long long e, int sign) const {
    cplx v = w[size_t(((e % n) + n) % n)];
    return sign > 0 ? v : std::conj(v);
  }
};

void dft_pow2(std::vector<cplx>& a, int sign) {
  const int n = int(a.size());
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  Twiddles tw(n);
  for (int len = 2; len <= n; len <<= 1) {
    const int half = len >> 1, step = n / len;
    for (int s = 0; s < n; s += len)
      for (int j = 0; j < half; ++j) {
        cplx w = tw.at((long long)j * step, sign);
        cplx u = a[s + j], v = a[s + j + half] * w;
        a[s + j] = u + v;
        a[s + j + half] = u - v;
      }
  }
}

void dft_any(std::vector<cplx>& a, int sign);

void dft_bluestein(std::vector<cplx>& a, int sign) {
  const int n = int(a.size());
  int m = 1;
  while (m < 2 * n - 1) m <<= 1;
  std::vector<cplx> chirp(n), A(m), B(m);
  for (int j = 0; j < n; ++j) {
    long long q = ((long long)j * j) % (2LL * n);
    double ang = kPi * double(q) / double(n);
    chirp[j] = cplx(std::cos(ang), sign > 0 ? std::sin(ang) : -std::sin(ang));
  }
  for (int j = 0; j < n; ++j) A[j] = a[j] * chirp[j];
  for (int j = 0; j < n; ++j) {
    B[j] = std::conj(chirp[j]);
    if (j) B[m - j] = std::conj(chirp[j]);
  }
  dft_pow2(A, -1);
  dft_pow2(B, -1);
  for (int j = 0; j < m; ++j) A[j] *= B[j];
  dft_pow2(A, +1);
  for (int k = 0; k < n; ++k) a[k] = (A[k] / double(m)) * chirp[k];
}

void dft_mixed(std::vector<cplx>& a, int sign) {
  const int n = int(a.size());
  int p = 0;
  for (int f = 2; f * f <= n; ++f)
    if (n % f == 0) { p = f; break; }
  if (p == 0) {
    if (n > 64) { dft_bluestein(a, sign); return; }
    Twiddles tw(n);
    std::vector<cplx> out(n);
    for (int k = 0; k < n; ++k) {
      cplx s = 0;
      for (int j = 0; j < n; ++j) s += a[j] * tw.at((long long)j * k, sign);
      out[k] = s;
    }
    a.swap(out);
    return;
  }
  const int m = n / p;
  std::vector<std::vector<cplx>> sub(p, std::vector<cplx>(m));
  for (int r = 0; r < p; ++r)
    for (int j = 0; j < m; ++j) sub[r][j] = a[size_t(j) * p + r];
  for (int r = 0; r < p; ++r) dft_any(sub[r], sign);
  Twiddles tw(n);
  for (int k = 0; k < n; ++k) {
    cplx s = 0;
    for (int r = 0; r < p; ++r) s += sub[r][k % m] * tw.at((long long)r * k, sign);
    a[k] = s;
  }
}

void dft_any(std::vector<cplx>& a, int sign) {
  const int n = int(a.size());
  if (n <= 1) return;
  if ((n & (n - 1)) == 0) dft_pow2(a, sign);
  else dft_mixed(a, sign);
}

// ----------------------------------------------------------------------------
// Reference helpers restated
// ----------------------------------------------------------------------------
double sgn(double v) { return v < 0 ? -1.0 : 1.0; }
double omega_i(double k, double d) {  // 1d/functions.c:1397
  return k == 0 ? 0.0 : sgn(k) * std::sqrt(kG * k * std::tanh(d * k));
}
double phase_velocity_i(double k, double d) {  // 1d/functions.c:1415
  return k == 0 ? std::sqrt(kG * d) : sgn(k) * std::sqrt(kG * k * std::tanh(d * k)) / k;
}
double group_velocity_i(double k, double d) {  // 1d/functions.c:1361
  if (k == 0) return std::sqrt(kG * d);
  double th = std::tanh(d * k);
  return sgn(k) * std::sqrt(kG) / 2 / std::sqrt(k * th) * (th + k * (1 - std::pow(th, 2)) * d);
}

// invers_omega (1d/functions.c:984-1020): Newton from k = 0, stopping rule
// |x - x0| < 1e-3 |x| (gsl_root_test_delta with epsabs 0, epsrel 1e-3).
double invers_omega(double w, double d) {
  double x = 0.0, value = 0.0, root = 0.0;
  double f = w - omega_i(root, d), df = -group_velocity_i(root, d);
  for (int iter = 1; iter <= 1000; ++iter) {
    if (df == 0.0) break;
    root = root - f / df;
    f = w - omega_i(root, d);
    df = -group_velocity_i(root, d);
    double x0 = x;
    x = root;
    if (std::fabs(x - x0) < 1e-3 * std::fabs(x) || x == x0) { value = x; break; }
  }
  return value;
}

// freqspace (1d/functions.c:1173-1197)
std::vector<double> freqspace(double len, int N) {
  std::vector<double> fs(N);
  double delta = 2 * kPi / len;
  double fmin = -0.5 * 2 * kPi / (len / (N - 1));
  double fmax = ((N / 2) * 2 == N) ? -fmin - delta : -fmin;
  double d = (fmax - fmin) / (N - 1);
  for (int i = 0; i < N / 2; ++i) fs[i] = fmin + (N / 2 + i) * d;
  for (int i = N / 2, Ni = 0; i < N; ++i, ++Ni) fs[i] = fmin + Ni * d;
  return fs;
}

int closest(const std::vector<double>& a, double ref) {  // 1d/functions.c:1761
  const int N = int(a.size());
  int idx = 0;
  double mn = 10 * (a[N / 2] - a[N / 2 - 1]);
  for (int i = 0; i < N; ++i)
    if (std::fabs(a[i] - ref) < mn) { mn = std::fabs(a[i] - ref); idx = i; }
  return idx;
}

std::vector<double> cf(const std::vector<double>& xi, double Xi, double del) {  // 1d/x_space.c:1
  std::vector<double> r(xi.size());
  for (size_t j = 0; j < xi.size(); ++j) {
    double a = (xi[j] - (Xi + del)) / std::fabs(xi[j] - (Xi + del));
    double b = (1 - std::cos((xi[j] - Xi) * kPi / del)) / 2;
    if (xi[j] < Xi) r[j] = 0;
    else if (xi[j] == Xi) r[j] = 0.5 * std::fmax(a, b);
    else r[j] = std::fmax(a, b);
  }
  return r;
}

double trapz_uniform(const std::vector<double>& x, const std::vector<double>& a, int N) {
  double s = 0.0;
  for (int i = 0; i < N; ++i) s += (i == 0 || i == N - 1) ? a[i] / 2 : a[i];
  return s * (x[1] - x[0]);
}

// a thin stdio cursor over input.txt reproducing the reference's positional reads
class InputFile {
 public:
  explicit InputFile(const std::string& path) : f_(std::fopen(path.c_str(), "r")) {}
  ~InputFile() { if (f_) std::fclose(f_); }
  bool ok() const { return f_ != nullptr; }
  void rewind() { std::rewind(f_); }
  bool skip_lines(int n, int width) {
    std::vector<char> line(size_t(width) + 1);
    for (int i = 0; i < n; ++i)
      if (!std::fgets(line.data(), width, f_)) return false;
    return true;
  }
  FILE* get() { return f_; }

 private:
  FILE* f_;
};

bool scan_word(FILE* f, std::string& out) {  // "%*s %*s %s \n"
  char buf[256];
  if (std::fscanf(f, "%*s %*s %255s \n", buf) != 1) return false;
  out = buf;
  return true;
}

bool read_column(const std::string& path, std::vector<double>& out, size_t n) {
  FILE* f = std::fopen(path.c_str(), "r");
  if (!f) return false;
  out.assign(n, 0.0);
  bool good = true;
  for (size_t j = 0; j < n && good; ++j) good = std::fscanf(f, "%lf \n", &out[j]) == 1;
  std::fclose(f);
  return good;
}

// 1d/read_input.c:1-60
bool parse_input(const std::string& dir, Deck& d, std::string& err) {
  InputFile in(dir + "/input.txt");
  if (!in.ok()) { err = "cannot open " + dir + "/input.txt"; return false; }
  FILE* f = in.get();
  bool ok = in.skip_lines(1, 128) && scan_word(f, d.wavename) && scan_word(f, d.initial);
  in.rewind();
  char b[256];
  ok = ok && in.skip_lines(18, 128) &&
       std::fscanf(f, "%*s %*s %255s \n %*s %*s %lf \n %*s %*s %lf \n", b, &d.depthflat, &d.adjcoef) == 3;
  if (ok) d.bath = b;
  in.rewind();
  ok = ok && in.skip_lines(23, 128) && scan_word(f, d.dynmodel) && scan_word(f, d.breaking) &&
       scan_word(f, d.friction) && scan_word(f, d.influxing) && scan_word(f, d.propagation) &&
       scan_word(f, d.kinematic) && std::fscanf(f, "%*s %*s %d \n", &d.ngauge) == 1 &&
       std::fscanf(f, "%*s %*s %d \n", &d.npartition) == 1;
  if (!ok) { err = "malformed input.txt (header blocks)"; return false; }
  // Optional blocks: a failed conversion keeps the default, as the reference's globals do.
  double xi1, xi2;
  int ns, nd, wt;
  double xw, rc, xc0, xc1, ac;
  char c1[256] = "", c2[256] = "";
  if (in.skip_lines(1, 128)) {
    if (std::fscanf(f, "%*s %*s %lf \n %*s %*s %lf %lf \n", &d.parKBC, &d.parTC, &d.parTchar) < 0) {}
  }
  if (in.skip_lines(1, 128)) {
    if (std::fscanf(f, "%*s %*s %lf \n %*s %*s %lf \n", &xi1, &xi2) == 2) { d.xinterv1 = xi1; d.xinterv2 = xi2; }
    if (std::fscanf(f, "%*s %*s %d \n %*s %*s %d \n", &ns, &nd) == 2) { d.nsurf = ns; d.ndeep = nd; }
  }
  if (in.skip_lines(1, 128)) {
    scan_word(f, d.cut_temp);
    scan_word(f, d.mid_temp);
    scan_word(f, d.min_z);
    scan_word(f, d.max_z);
    if (std::fscanf(f, "%*s %*s %255s %lf", c1, &d.nTramp) >= 1) d.rampbool = c1;
    scan_word(f, d.wall);
    if (std::fscanf(f, "%*s %*s %d %lf %lf\n", &wt, &xw, &rc) < 0) {}
  }
  if (in.skip_lines(1, 128)) {
    if (std::fscanf(f, "%*s %*s %255s %255s\n %*s %*s %lf %lf\n", c1, c2, &xc0, &xc1) >= 1) d.coupling = c1;
    if (std::fscanf(f, "%*s %*s %lf\n", &ac) < 0) {}
  }
  return true;
}

// seeded stand-in for rand()/RAND_MAX (splitmix64, 53-bit mantissa)
double splitmix_uniform(unsigned long long& s) {
  unsigned long long z = (s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return double(z >> 11) * (1.0 / 9007199254740992.0);
}

// influxlib (1d/influx_lib.c:1-109) with harmonic_influx (:217) and a seeded
// jonswap_influx (:289, including the integer exponent 5/4 == 1 of :269-270)
bool load_influx(const std::string& dir, Member& m, std::vector<double>& wt, std::vector<double>& we,
                 const SetupOptions& opt, std::string& err) {
  Deck& d = m.deck;
  InputFile in(dir + "/input.txt");
  FILE* f = in.get();
  const bool timed = d.wavename == "harmonic" || d.wavename == "jonswap" || d.wavename == "zero";
  int Nt = 0;
  double lenT = 0;
  if (timed) {
    in.skip_lines(5, 256);
    if (std::fscanf(f, "%*s %*s %lf \n %*s %*s %lf \n %*s %*s %lf\n", &d.T0, &d.Tend, &d.dt) != 3 ||
        std::fscanf(f, "%*s %*s %lf \n %*s %*s %lf \n %*s %*s %lf\n", &d.Tp, &d.Hs, &d.gamJS) != 3) {
      err = "malformed time/spectrum block in input.txt";
      return false;
    }
    in.rewind();
    lenT = d.Tend - d.T0;
    Nt = int((lenT) / d.dt + 1);
  }
  if (d.wavename == "zero") {
    wt.resize(Nt);
    we.assign(Nt, 0.0);
    for (int i = 0; i < Nt; ++i) wt[i] = d.T0 + d.dt * i;
  } else if (d.wavename == "user_defined") {
    FILE* fi = std::fopen((dir + "/influx.dat").c_str(), "r");
    if (!fi) { err = "cannot open influx file " + dir + "/influx.dat"; return false; }
    double tt, ss;
    while (std::fscanf(fi, "%lf %lf", &tt, &ss) == 2) { wt.push_back(tt); we.push_back(ss); }
    std::fclose(fi);
    if (wt.size() < 2) { err = "influx.dat holds fewer than 2 samples"; return false; }
  } else if (d.wavename == "harmonic") {
    double t = d.T0, amp = 0.5 * d.Hs;
    for (int i = 0; t <= d.Tend; ++i) {
      t = d.T0 + i * d.dt;
      double r1 = ((t - 4 * d.Tp) < 0 ? -1 : 1);
      double r2 = (1 - std::cos(t * kPi / 4 / d.Tp)) / 2;
      wt.push_back(t);
      we.push_back(amp * (r1 > r2 ? r1 : r2) * (std::sin(t * 2 * kPi / d.Tp)));
    }
  } else if (d.wavename == "jonswap" && opt.influx_eta && int(opt.influx_eta->size()) == Nt) {
    wt.resize(Nt);
    we = *opt.influx_eta;
    for (int j = 0; j < Nt; ++j) wt[j] = d.T0 + j * d.dt;
  } else if (d.wavename == "jonswap") {
    const double omgp = 2 * kPi / d.Tp;
    std::vector<double> om = freqspace(lenT, Nt);
    const int Nomg = Nt / 2;
    std::vector<double> JS(Nomg, 0.0), spec(Nomg);
    const double alpha = 0.0081, fp = omgp / (2 * kPi);
    for (int i = 1; i < Nomg; ++i) {
      double sigma = om[i] <= omgp ? 0.07 : 0.09;
      double fr = om[i] / (2 * kPi);
      double gp = std::exp(-0.5 * std::pow(((fr / fp - 1) / sigma), 2));
      JS[i] = alpha * std::pow(kG, 2) * std::pow((2 * kPi), (-4)) * std::pow(fr, (-5)) *
              std::exp(-(5 / 4) * std::pow((fr / fp), (-4))) * std::pow(d.gamJS, gp);
    }
    double m0 = trapz_uniform(om, JS, Nomg);
    for (int i = 0; i < Nomg; ++i) spec[i] = (std::pow(d.Hs, 2) / 16) * JS[i] / m0;
    std::vector<double> phase(Nomg + 1, 0.0), re(Nt, 0.0), im(Nt, 0.0);
    unsigned long long s = opt.seed;
    for (int i = 0; i < Nomg; ++i) {
      phase[i + 1] = 2 * kPi * splitmix_uniform(s);
      re[i + 1] = (std::sqrt(spec[i]) * std::cos(phase[i])) / d.dt * 2 * std::pow(kPi, 2);
      im[i + 1] = -(std::sqrt(spec[i]) * std::sin(phase[i])) / d.dt * 2 * std::pow(kPi, 2);
      re[Nt - 1 - i] = re[i + 1];
      im[Nt - 1 - i] = -im[i + 1];
    }
    re[0] = im[0] = 0;
    host_dft(re, im, +1);
    std::vector<double> ramp(Nt), sig(Nt);
    for (int j = 0; j < Nt; ++j) {
      double tin = d.T0 + j * d.dt;
      double A = ((tin - d.T0) - d.nTramp * d.Tp);
      double B1 = A / std::fabs(A);
      double B2 = (1 - std::cos((tin - d.T0) * kPi / d.nTramp / d.Tp)) / 2;
      ramp[j] = B1 > B2 ? B1 : B2;
    }
    double mean = 0;
    for (int j = 0; j < Nt; ++j) { sig[j] = ramp[j] * (re[j] / Nt) * ramp[Nt - 1 - j]; mean += sig[j]; }
    mean /= Nt;
    double var = 0;
    for (int j = 0; j < Nt; ++j) var += std::pow(sig[j] - mean, 2);
    var /= Nt;
    wt.resize(Nt);
    we.resize(Nt);
    for (int j = 0; j < Nt; ++j) { wt[j] = d.T0 + j * d.dt; we[j] = sig[j] * d.Hs / (4 * std::sqrt(var)); }
  } else {
    err = "unsupported wavename '" + d.wavename + "'";
    return false;
  }
  in.rewind();
  in.skip_lines(13, 256);
  if (std::fscanf(f, "%*s %*s %lf \n %*s %*s %lf \n %*s %*s %lf\n", &d.Xstart, &d.Xend, &d.Xinflux) != 3 ||
      std::fscanf(f, "%*s %*s %lf \n %*s %*s %lf %lf\n ", &d.dx, &d.dampL, &d.dampR) != 3) {
    err = "malformed &SPATIAL block in input.txt";
    return false;
  }
  return true;
}

bool largest_prime_ok(int number) {  // 1d/functions.c:3671
  while (number % 2 == 0) number /= 2;
  for (int i = 3; i <= std::sqrt(number); i += 2)
    while (number % i == 0) number /= i;
  return number <= 13;
}

// Up2IP / Up3IP (1d/functions.c:2195-2340) on the reference depths D, with the
// gamma coefficients fitted on 101 depth samples and natural cubic splines.
void interp_two_three(Member& m, double nu, int three, double D_min, double D_mid, double D_plus) {
  const int n = 101;
  const double dD = (D_plus - D_min) / (n - 1);
  std::vector<double> Dd(n), gm(n), gc(n), gp(n);
  for (int i = 0; i < n; ++i) {
    Dd[i] = D_min + i * dD;
    double kap = invers_omega(nu, Dd[i]);
    if (!three) {
      double Cp_min = std::pow(phase_velocity_i(kap, D_min), 2);
      double Cp_plus = std::pow(phase_velocity_i(kap, D_plus), 2);
      double Cp_D = std::pow(phase_velocity_i(kap, Dd[i]), 2);
      double Om_min = omega_i(kap, D_min), Om_plus = omega_i(kap, D_plus), Om_D = omega_i(kap, Dd[i]);
      double det = Cp_min * Om_plus - Cp_plus * Om_min;
      gm[i] = (Om_plus * Cp_D - Cp_plus * Om_D) / det;
      gp[i] = (-Om_min * Cp_D + Cp_min * Om_D) / det;
    } else {
      double C0_min = std::sqrt(kG * D_min), C0_mid = std::sqrt(kG * D_mid), C0_plus = std::sqrt(kG * D_plus),
             C0_D = std::sqrt(kG * Dd[i]);
      double Cp_min = std::pow(phase_velocity_i(kap, D_min), 2);
      double Cp_mid = std::pow(phase_velocity_i(kap, D_mid), 2);
      double Cp_plus = std::pow(phase_velocity_i(kap, D_plus), 2);
      double Cp_D = std::pow(phase_velocity_i(kap, Dd[i]), 2);
      double Om_min = omega_i(kap, D_min), Om_mid = omega_i(kap, D_mid), Om_plus = omega_i(kap, D_plus),
             Om_D = omega_i(kap, Dd[i]);
      double A = (Om_mid * Cp_plus) - (Om_plus * Cp_mid);
      double B = -(Om_min * Cp_plus) + (Om_plus * Cp_min);
      double C = (Om_min * Cp_mid) - (Om_mid * Cp_min);
      double D = -(C0_mid * Cp_plus) + (C0_plus * Cp_mid);
      double E = (C0_min * Cp_plus) - (C0_plus * Cp_min);
      double F = -(C0_min * Cp_mid) + (C0_mid * Cp_min);
      double Gg = (C0_mid * Om_plus) - (C0_plus * Om_mid);
      double H = -(C0_min * Om_plus) + (C0_plus * Om_min);
      double J = (C0_min * Om_mid) - (C0_mid * Om_min);
      double det = C0_min * A + C0_mid * B + C0_plus * C;
      gm[i] = (A * C0_D + D * Om_D + Gg * Cp_D) / det;
      gc[i] = (B * C0_D + E * Om_D + H * Cp_D) / det;
      gp[i] = (C * C0_D + F * Om_D + J * Cp_D) / det;
    }
  }
  const int Nx = m.Nx;
  const int K = three ? 3 : 2;
  m.Csq_ref.assign(K, std::vector<double>(Nx));
  m.gam_ref.assign(K, std::vector<double>(Nx));
  std::vector<double> cm = natural_spline_c(Dd, gm), cp = natural_spline_c(Dd, gp), cc;
  if (three) cc = natural_spline_c(Dd, gc);
  // reference order of the sum in HSS: min, plus, then mid (1d/functions.c:2955-2971)
  for (int i = 0; i < Nx; ++i) {
    m.Csq_ref[0][i] = std::pow(phase_velocity_i(m.k[i], D_min), 2);
    m.Csq_ref[1][i] = std::pow(phase_velocity_i(m.k[i], D_plus), 2);
    m.gam_ref[0][i] = natural_spline_eval(Dd, gm, cm, m.depth[i]);
    m.gam_ref[1][i] = natural_spline_eval(Dd, gp, cp, m.depth[i]);
    if (three) {
      m.Csq_ref[2][i] = std::pow(phase_velocity_i(m.k[i], D_mid), 2);
      m.gam_ref[2][i] = natural_spline_eval(Dd, gc, cc, m.depth[i]);
    }
  }
}

// K reference depths (K > 3, no counterpart in the reference): log-spaced between
// the shallowest and the deepest point; each point uses the two-reference system of
// Up2IP (1d/functions.c:2195-2245) on its bracketing pair, solved at its own depth.
void interp_k(Member& m, double nu, int K, double Dmin, double Dmax) {
  const int Nx = m.Nx;
  std::vector<double> D(K);
  for (int j = 0; j < K; ++j) D[j] = Dmin * std::pow(Dmax / Dmin, double(j) / double(K - 1));
  D[0] = Dmin;
  D[K - 1] = Dmax;
  m.Csq_ref.assign(K, std::vector<double>(Nx));
  m.gam_ref.assign(K, std::vector<double>(Nx, 0.0));
  for (int j = 0; j < K; ++j)
    for (int i = 0; i < Nx; ++i) m.Csq_ref[j][i] = std::pow(phase_velocity_i(m.k[i], D[j]), 2);
  for (int i = 0; i < Nx; ++i) {
    const double h = m.depth[i];
    int j = 0;
    while (j < K - 2 && h > D[j + 1]) ++j;
    const double kap = invers_omega(nu, h);
    const double Cp_a = std::pow(phase_velocity_i(kap, D[j]), 2), Cp_b = std::pow(phase_velocity_i(kap, D[j + 1]), 2);
    const double Cp_h = std::pow(phase_velocity_i(kap, h), 2);
    const double Om_a = omega_i(kap, D[j]), Om_b = omega_i(kap, D[j + 1]), Om_h = omega_i(kap, h);
    const double det = Cp_a * Om_b - Cp_b * Om_a;
    m.gam_ref[j][i] = (Om_b * Cp_h - Cp_b * Om_h) / det;
    m.gam_ref[j + 1][i] = (-Om_a * Cp_h + Cp_a * Om_h) / det;
  }
}

}  // namespace

std::vector<double> csq_row(const std::vector<double>& k, double D) {
  std::vector<double> r(k.size());
  for (size_t i = 0; i < k.size(); ++i) r[i] = std::pow(phase_velocity_i(k[i], D), 2);
  return r;
}

void host_dft(std::vector<double>& re, std::vector<double>& im, int sign) {
  std::vector<cplx> a(re.size());
  for (size_t i = 0; i < re.size(); ++i) a[i] = cplx(re[i], im[i]);
  dft_any(a, sign);
  for (size_t i = 0; i < re.size(); ++i) { re[i] = a[i].real(); im[i] = a[i].imag(); }
}

// GSL cspline (natural) init: symmetric tridiagonal system solved by LDL^T.
std::vector<double> natural_spline_c(const std::vector<double>& x, const std::vector<double>& y) {
  const int n = int(x.size());
  std::vector<double> c(n, 0.0);
  const int sys = n - 2;
  if (sys <= 0) return c;
  std::vector<double> diag(sys), off(sys), g(sys);
  for (int i = 0; i < sys; ++i) {
    double h_i = x[i + 1] - x[i], h_ip1 = x[i + 2] - x[i + 1];
    double yd_i = y[i + 1] - y[i], yd_ip1 = y[i + 2] - y[i + 1];
    double g_i = (h_i != 0.0) ? 1.0 / h_i : 0.0;
    double g_ip1 = (h_ip1 != 0.0) ? 1.0 / h_ip1 : 0.0;
    off[i] = h_ip1;
    diag[i] = 2.0 * (h_ip1 + h_i);
    g[i] = 3.0 * (yd_ip1 * g_ip1 - yd_i * g_i);
  }
  if (sys == 1) { c[1] = g[0] / diag[0]; return c; }
  std::vector<double> gamma(sys), alpha(sys), z(sys);
  alpha[0] = diag[0];
  gamma[0] = off[0] / alpha[0];
  for (int i = 1; i < sys - 1; ++i) {
    alpha[i] = diag[i] - off[i - 1] * gamma[i - 1];
    gamma[i] = off[i] / alpha[i];
  }
  alpha[sys - 1] = diag[sys - 1] - off[sys - 2] * gamma[sys - 2];
  z[0] = g[0];
  for (int i = 1; i < sys; ++i) z[i] = g[i] - gamma[i - 1] * z[i - 1];
  std::vector<double> cc(sys);
  for (int i = 0; i < sys; ++i) cc[i] = z[i] / alpha[i];
  std::vector<double> sol(sys);
  sol[sys - 1] = cc[sys - 1];
  for (int i = sys - 2; i >= 0; --i) sol[i] = cc[i] - gamma[i] * sol[i + 1];
  for (int i = 0; i < sys; ++i) c[i + 1] = sol[i];
  return c;
}

double natural_spline_eval(const std::vector<double>& x, const std::vector<double>& y,
                           const std::vector<double>& c, double t) {
  const int n = int(x.size());
  if (t < x[0] || t > x[n - 1]) return std::nan("");
  int lo = 0, hi = n - 1;
  while (hi > lo + 1) {
    int i = (hi + lo) / 2;
    if (x[i] > t) hi = i; else lo = i;
  }
  double h = x[lo + 1] - x[lo], dy = y[lo + 1] - y[lo], delx = t - x[lo];
  double b = dy / h - h * (c[lo + 1] + 2.0 * c[lo]) / 3.0;
  double d = (c[lo + 1] - c[lo]) / (3.0 * h);
  return y[lo] + delx * (b + delx * (c[lo] + delx * d));
}

bool build_member(const std::string& dir, const SetupOptions& opt, Member& m, std::string& err) {
  Deck& d = m.deck;
  if (!parse_input(dir, d, err)) return false;
  if (d.rampbool == "no") d.nTramp = 0;  // 1d/main.cc:47-49
  if (d.dynmodel != "HS1" && d.dynmodel != "HS2" && d.dynmodel != "HS3") {
    err = "unsupported dynamics '" + d.dynmodel + "'";
    return false;
  }
  if (d.friction == "yes" || d.wall == "yes" || d.coupling == "yes") {
    err = "friction, wall and coupling are outside this engine";
    return false;
  }
  m.model = d.dynmodel[2] - '0';
  m.cutfracwn = m.model == 1 ? 2 : m.model == 2 ? 4 : 6;  // 1d/influx_lib.c:186-197
  std::vector<double> wt, we;
  if (!load_influx(dir, m, wt, we, opt, err)) return false;
  // domain (1d/influx_lib.c:199-213)
  m.length = d.Xend - d.Xstart;
  int Nx = int((m.length / d.dx) + 1);
  if (Nx % 2 != 0) Nx -= 1;
  if (Nx < 4) { err = "grid too small"; return false; }
  m.Nx = Nx;
  m.x.resize(Nx);
  m.dx = m.length / (Nx - 1);
  for (int i = 0; i < Nx; ++i) m.x[i] = d.Xstart + m.dx * i;
  m.idx_inf = closest(m.x, d.Xinflux);
  m.Xinflux = m.x[m.idx_inf];
  if (!largest_prime_ok(Nx)) { err = "Nx has a largest prime factor > 13"; return false; }
  const int n = int(wt.size());
  m.n = n;
  m.ttrace = wt;
  m.dt = m.ttrace[1] - m.ttrace[0];
  // bathymetry (1d/functions.c:804-830)
  m.flat = d.bath == "flat";
  if (d.bath == "user_defined") {
    if (!read_column(dir + "/bath.dat", m.depth, size_t(Nx))) { err = "cannot read bath.dat"; return false; }
    m.depthinf = m.depth[m.idx_inf];
    for (double v : m.depth)
      if (v < 0) { err = "runup (negative depth) is outside this engine"; return false; }
  } else if (m.flat) {
    m.depth.assign(Nx, d.depthflat);
    m.depthinf = d.depthflat;
  } else {
    err = "unsupported bathymetry '" + d.bath + "'";
    return false;
  }
  if (d.ngauge > 0) {
    FILE* fg = std::fopen((dir + "/gauges.dat").c_str(), "r");
    if (!fg) { err = "cannot open gauges.dat"; return false; }
    m.gauge.assign(d.ngauge, 0.0);
    for (int j = 0; j < d.ngauge; ++j)
      if (std::fscanf(fg, "%lf \n", &m.gauge[j]) != 1) m.gauge[j] = 0.0;
    std::fclose(fg);
  }
  m.has_influx = d.wavename != "zero";
  m.insig.assign(n, 0.0);
  m.insig_skew.assign(n, 0.0);
  std::vector<double> ww, kom, GV, ins_re, ins_im;   // modified_influx's kom, GVom, insig_hat
  if (m.has_influx) {
    // set_influx / nsqrspec (1d/functions.c:1256-1329): peak of the normalised spectrum
    std::vector<double> re(we), im(n, 0.0);
    host_dft(re, im, -1);
    std::vector<double> sq(n), spin(n);
    double sum = 0;
    for (int i = 0; i < n; ++i) {
      double a = std::sqrt(std::pow(re[i], 2) + std::pow(im[i], 2));
      sq[i] = a * a;
    }
    for (int i = 0; i < n; ++i) sum += sq[i];
    for (int i = 0; i < n; ++i) spin[i] = std::sqrt(sq[i] / sum);
    ww = freqspace(wt[n - 1] - wt[0], n);
    double best = spin[0];
    int idx = 0;
    for (int i = 0; i < n / 2; ++i)
      if (spin[i] >= best) { best = spin[i]; idx = i; }
    m.nu_peak = std::fabs(ww[idx]);
    m.kp = invers_omega(m.nu_peak, m.depthinf);
    m.Tp_peak = 2 * kPi / m.nu_peak;
    if (d.wavename == "jonswap") {
      m.nu_peak = 2 * kPi / d.Tp;
      m.kp = invers_omega(m.nu_peak, m.depthinf);
    }
    m.lambda_p = 2 * kPi / m.kp;
    double avg = 0, var = 0;
    for (int i = 0; i < n; ++i) avg += we[i];
    avg /= n;
    for (int i = 0; i < n; ++i) var += std::pow(we[i] - avg, 2);
    var /= n;
    m.Hs_in = 4 * std::sqrt(var);
    m.MaxEtaInit = (m.Hs_in / 2) * 0.8;
    // modified_influx (1d/functions.c:1968-2042)
    m.insig = we;
    if (d.wavename == "user_defined") {
      std::vector<double> ramp(n);
      for (int j = 0; j < n; ++j) {
        double A = ((m.ttrace[j] - m.ttrace[0]) - d.nTramp * m.Tp_peak);
        double B1 = A / std::fabs(A);
        double B2 = (1 - std::cos((m.ttrace[j] - m.ttrace[0]) * kPi / d.nTramp / m.Tp_peak)) / 2;
        ramp[j] = B1 > B2 ? B1 : B2;
      }
      for (int j = 0; j < n; ++j) m.insig[j] = ramp[j] * m.insig[j] * ramp[n - 1 - j];
    }
    double acc = 0;
    m.insig_skew[0] = 0;
    for (int i = 1; i < n; ++i) { acc = acc + 0.5 * m.dt * (m.insig[i - 1] + m.insig[i]); m.insig_skew[i] = acc; }
    if (d.influxing == "Point" || d.influxing == "AreaShort") {
      kom.resize(n);
      GV.resize(n);
      for (int i = 0; i < n; ++i) {
        kom[i] = ww[i] == 0 ? 0 : invers_omega(ww[i], m.depthinf);
        GV[i] = group_velocity_i(kom[i], m.depthinf);
      }
    }
    if (d.influxing == "AreaShort") {
      // the signal's spectrum (insig_hat) and the group velocity scaled to the long-wave
      // speed at omega = 0, for x_space's division by the kernel's spectrum
      ins_re = m.insig;
      ins_im.assign(n, 0.0);
      host_dft(ins_re, ins_im, -1);
      const double g0 = GV[0];
      for (int j = 0; j < n; ++j) GV[j] = GV[j] * std::sqrt(kG * m.depthinf) / g0;
    } else if (d.influxing == "Point") {
      std::vector<double> a_re(m.insig), a_im(n, 0.0), s_re(m.insig_skew), s_im(n, 0.0);
      host_dft(a_re, a_im, -1);
      host_dft(s_re, s_im, -1);
      for (int i = 0; i < n; ++i) { a_re[i] *= GV[i]; a_im[i] *= GV[i]; s_re[i] *= GV[i]; s_im[i] *= GV[i]; }
      host_dft(a_re, a_im, +1);
      host_dft(s_re, s_im, +1);
      for (int j = 0; j < n; ++j) { m.insig[j] = a_re[j] / n; m.insig_skew[j] = s_re[j] / n; }
    } else if (d.influxing != "Area") {
      err = "influxing '" + d.influxing + "' is outside this engine";
      return false;
    }
  } else {
    m.Hs_in = 0;
    m.MaxEtaInit = 0;
  }
  // x_space (1d/x_space.c:18-164)
  m.dampchar.resize(Nx);
  const double Bleft = d.Xstart + d.dampL, Bright = d.Xend - d.dampR;
  for (int i = 0; i < Nx; ++i) {  // dampzone (1d/functions.c:1331)
    const double xi = m.x[i];
    double hR0 = Bright - xi < 0 ? -1 : 1;
    double hR1 = 1 + ((Bright + d.dampR - xi) < 0 ? -1 : 1);
    double hR2 = (1 + std::cos(kPi * (xi - Bright) / d.dampR)) / 2;
    double mR = hR1 < hR2 ? hR1 : hR2;
    double hhR = hR0 > mR ? hR0 : mR;
    double hL0 = 1 + ((xi - Bleft + d.dampL) < 0 ? -1 : 1);
    double hL1 = (xi - Bleft) < 0 ? -1 : 1;
    double hL2 = (1 - std::cos(kPi * (xi - Bleft + d.dampL) / d.dampL)) / 2;
    double mL = hL1 > hL2 ? hL1 : hL2;
    double hhL = hL0 < mL ? hL0 : mL;
    m.dampchar[i] = 1 - (hhR * hhL);
  }
  double CpLeft, CpRight;
  if (m.has_influx) {
    CpLeft = omega_i(m.kp, m.depth[0]) / m.kp;
    CpRight = omega_i(m.kp, m.depth[Nx - 1]) / m.kp;
  } else {
    CpLeft = std::sqrt(kG * m.depth[0]);
    CpRight = std::sqrt(kG * m.depth[Nx - 1]);
  }
  m.dampcoef.resize(Nx);
  for (int j = 0; j < Nx / 2; ++j) {
    m.dampcoef[j] = 7 * CpLeft / (0.9 * d.dampL);
    m.dampcoef[j + Nx / 2] = 7 * CpRight / (0.9 * d.dampR);
  }
  m.k = freqspace(m.length, Nx);
  m.gamX_re.assign(Nx, 0.0); m.gamX_im.assign(Nx, 0.0);
  m.gamXs_re.assign(Nx, 0.0); m.gamXs_im.assign(Nx, 0.0);
  if (m.has_influx) {
    const double fact = 1 / m.dx, cp = std::sqrt(kG * m.depthinf);
    if (d.influxing == "Point") {
      for (int i = 0; i < Nx; ++i) {
        m.gamX_re[i] = std::cos(m.k[i] * (m.Xinflux - d.Xstart)) * fact;
        m.gamX_im[i] = -std::sin(m.k[i] * (m.Xinflux - d.Xstart)) * fact;
      }
    } else {
      // Area: spatial kernel = shifted inverse transform of the group velocity
      std::vector<double> re(Nx), im(Nx, 0.0);
      for (int i = 0; i < Nx; ++i) re[i] = group_velocity_i(m.k[i], m.depthinf);
      host_dft(re, im, +1);
      std::vector<double> sp(Nx);
      const int shift = int((m.Xinflux - d.Xstart) / m.dx);
      const int s = ((shift % Nx) + Nx) % Nx;
      for (int j = 0; j < Nx; ++j) sp[(j + s) % Nx] = re[j] / Nx;
      if (d.influxing == "AreaShort") {
        // 1d/x_space.c:64-78: the kernel under a Gaussian window of +-2 peak wavelengths
        const double Lb = 2 * std::pow(0.4 * m.lambda_p, 2);
        const int ind1 = closest(m.x, m.Xinflux - 2 * m.lambda_p), ind2 = closest(m.x, m.Xinflux + 2 * m.lambda_p);
        std::vector<double> win(Nx, 0.0);
        for (int i = ind1; i < ind2 + 1; ++i) win[i] = std::exp(-std::pow((m.x[i] - m.Xinflux), 2) / Lb);
        for (int i = 0; i < Nx; ++i) sp[i] = sp[i] * win[i];
      }
      std::vector<double> gr(sp), gi(Nx, 0.0);
      host_dft(gr, gi, -1);
      // scaling_influx (1d/functions.c:1747)
      for (int i = 0; i < Nx; ++i) { gr[i] = gr[i] * fact; gi[i] = gi[i] * fact; }
      const double scale = gr[0] * m.dx;
      for (int i = 0; i < Nx; ++i) { m.gamX_re[i] = gr[i] * cp / scale; m.gamX_im[i] = gi[i] * cp / scale; }
      if (d.influxing == "AreaShort") {
        // 1d/x_space.c:86-109: the signal's spectrum times the scaled group velocity over
        // the kernel's spectral amplitude (a natural spline over the centred wavenumbers,
        // its last value beyond them), back to time; its running integral again
        const int n = m.n;
        std::vector<double> ag(Nx), kt(Nx);
        for (int i = 0; i < Nx / 2; ++i) {
          ag[i] = std::sqrt(std::pow(m.gamX_re[Nx / 2 + i], 2) + std::pow(m.gamX_im[Nx / 2 + i], 2));
          ag[Nx / 2 + i] = std::sqrt(std::pow(m.gamX_re[i], 2) + std::pow(m.gamX_im[i], 2));
          kt[i] = m.k[Nx / 2 + i];
          kt[Nx / 2 + i] = m.k[i];
        }
        const std::vector<double> cg = natural_spline_c(kt, ag);
        std::vector<double> tr(n), ti(n);
        for (int i = 0; i < n; ++i) {
          const double gom = std::fabs(kom[i]) > std::fabs(kt[Nx - 1]) ? ag[Nx - 1]
                                                                       : natural_spline_eval(kt, ag, cg, kom[i]);
          tr[i] = ins_re[i] * GV[i] / gom / m.dx;
          ti[i] = ins_im[i] * GV[i] / gom / m.dx;
        }
        host_dft(tr, ti, +1);
        for (int j = 0; j < n; ++j) m.insig[j] = tr[j] / n;
        double a = 0;
        m.insig_skew[0] = 0;
        for (int i = 1; i < n; ++i) { a = a + 0.5 * m.dt * (m.insig[i - 1] + m.insig[i]); m.insig_skew[i] = a; }
      }
    }
    for (int i = 0; i < Nx; ++i) {
      m.gamXs_re[i] = -omega_i(m.k[i], m.depthinf) * m.gamX_im[i];
      m.gamXs_im[i] = omega_i(m.k[i], m.depthinf) * m.gamX_re[i];
    }
    m.sp_c_in = natural_spline_c(m.ttrace, m.insig);
    m.sp_c_skew = natural_spline_c(m.ttrace, m.insig_skew);
  }
  // nonlinear adjustment mask (1d/x_space.c:131-163)
  if (d.propagation == "Uni+") m.prop_mode = 0;
  else if (d.propagation == "Uni-") m.prop_mode = 1;
  else if (d.propagation == "Bi") m.prop_mode = 2;
  else m.prop_mode = 3;
  if (m.model == 1 || !m.has_influx) {
    m.ChiAdj.assign(Nx, 1.0);
  } else if (m.prop_mode == 0) {
    m.ChiAdj = cf(m.x, m.Xinflux, d.adjcoef * m.lambda_p);
  } else if (m.prop_mode == 1) {
    std::vector<double> t = cf(m.x, (m.Xinflux - d.adjcoef * m.lambda_p), d.adjcoef * m.lambda_p);
    m.ChiAdj.resize(Nx);
    for (int j = 0; j < Nx; ++j) m.ChiAdj[j] = 1 - t[j];
  } else if (m.prop_mode == 2) {
    std::vector<double> L = cf(m.x, m.Xinflux, d.adjcoef * m.lambda_p);
    std::vector<double> R = cf(m.x, m.Xinflux - d.adjcoef * m.lambda_p, d.adjcoef * m.lambda_p);
    m.ChiAdj.resize(Nx);
    for (int j = 0; j < Nx; ++j) m.ChiAdj[j] = 1 - R[j] + L[j];
  } else {
    m.ChiAdj.assign(Nx, 0.0);
  }
  // initial condition (1d/main.cc:104-136)
  if (d.initial == "user_defined") {
    FILE* fi = std::fopen((dir + "/initial.dat").c_str(), "r");
    if (!fi) { err = "cannot open initial.dat"; return false; }
    m.temp_wave.assign(Nx, 0.0);
    m.temp_u.assign(Nx, 0.0);
    for (int j = 0; j < Nx; ++j)
      if (std::fscanf(fi, "%lf %lf\n", &m.temp_wave[j], &m.temp_u[j]) != 2) {
        std::fclose(fi);
        err = "initial.dat: short file";
        return false;
      }
    std::fclose(fi);
    std::vector<double> re(m.temp_wave), im(Nx, 0.0);
    host_dft(re, im, -1);
    double best = std::sqrt(std::pow(re[0], 2) + std::pow(im[0], 2));
    int idx = 0;
    for (int i = 0; i < Nx / 2; ++i) {
      double a = std::sqrt(std::pow(re[i], 2) + std::pow(im[i], 2));
      if (a >= best) { best = a; idx = i; }
    }
    m.kp = std::fabs(m.k[idx]);
    if (idx == 0) m.kp = std::fabs(m.k[1]);
    double avgD = 0;
    for (double v : m.depth) avgD += v;
    avgD /= Nx;
    m.nu_peak = omega_i(m.kp, avgD);
    double mx = m.temp_wave[0];
    for (double v : m.temp_wave) if (v > mx) mx = v;
    if (2 * mx > m.Hs_in) m.Hs_in = 2 * mx;
    m.MaxEtaInit = (m.Hs_in / 2) * 0.8;
  } else if (d.initial != "zero") {
    err = "unsupported initial '" + d.initial + "'";
    return false;
  }
  // breaking parameters (1d/breaking.c:1-34)
  m.breaking = d.breaking == "yes" && m.model >= 2;
  if (d.breaking == "yes") {
    m.KBC = d.parKBC;
    m.TC = d.parTC;
    m.Tstar = d.initial != "zero" ? 5 * std::sqrt(m.depthinf * kG) : d.parTchar * m.Tp_peak;
    const double off = 0.1 * d.adjcoef * m.lambda_p;
    if (m.prop_mode == 0) {
      m.xbstart = closest(m.x, m.Xinflux + off); m.xbend = Nx - 1; m.lenIF = m.xbend - m.xbstart;
    } else if (m.prop_mode == 1) {
      m.xbend = closest(m.x, m.Xinflux - off); m.xbstart = 0; m.lenIF = m.xbend - m.xbstart;
    } else if (m.prop_mode == 2) {
      m.xbstart = 0; m.xbendL = closest(m.x, m.Xinflux - off); m.xbstartR = closest(m.x, m.Xinflux + off);
      m.xbend = Nx - 1; m.ILL = m.xbendL - m.xbstart; m.IFF = m.xbend - m.xbstartR;
    } else {
      m.xbstart = 0; m.xbend = Nx - 1; m.lenIF = m.xbend - m.xbstart;
    }
  }
  // expert overrides read by read_kinematics (1d/functions.c:3555-3562)
  double mid1 = 0.5;
  if (!d.cut_temp.empty() && d.cut_temp != "default") m.cutfracwn = std::atoi(d.cut_temp.c_str());
  if (!d.mid_temp.empty() && d.mid_temp != "default") mid1 = std::atof(d.mid_temp.c_str());
  // operators (1d/functions.c:2828-2859, 1796-1820)
  m.Csqr.resize(Nx); m.L.resize(Nx); m.M0im.resize(Nx);
  for (int i = 0; i < Nx; ++i) m.Csqr[i] = std::pow(phase_velocity_i(m.k[i], m.depthinf), 2);
  for (int i = 0; i < Nx; ++i) {
    m.L[i] = std::pow(m.k[i], 2) * std::pow(phase_velocity_i(m.k[i], m.depthinf), 2) / kG;
    m.M0im[i] = -m.k[i] * m.Csqr[i] / kG;
  }
  m.nref = opt.nref ? opt.nref : 3;
  if (!m.flat) {
    double Dmin = m.depth[0], Dmax = m.depth[0];
    for (double v : m.depth) { Dmin = std::min(Dmin, v); Dmax = std::max(Dmax, v); }
    if (m.nref <= 3) {
      double Dmid = (Dmax + Dmin) / 2;
      if (!d.mid_temp.empty() && d.mid_temp != "default") Dmid = mid1;
      interp_two_three(m, m.nu_peak, m.nref == 3, Dmin, Dmid, Dmax);
    } else if (m.nref <= 16) {
      interp_k(m, m.nu_peak, m.nref, Dmin, Dmax);
    } else {
      err = "at most 16 reference depths";
      return false;
    }
  }
  // alias (1d/functions.c:1774)
  m.aal.resize(Nx);
  const int idk = int(Nx / double(m.cutfracwn)) - 1;
  const double k0 = m.k[idk];
  for (int i = 0; i < Nx; ++i)
    m.aal[i] = (i != idk) ? ((k0 - std::fabs(m.k[i])) / std::fabs(k0 - std::fabs(m.k[i])) + 1) / 2 : 0.5;
  // tolerances and first step (1d/functions.c:528-541)
  m.eps_abs = opt.eps_abs > 0 ? opt.eps_abs : 1e-5;
  m.eps_rel = opt.eps_rel > 0 ? opt.eps_rel : 1e-4;
  m.h0 = opt.h0 > 0 ? opt.h0 : 1e-4;
  // initial spectral state (set_initial_ode, 1d/functions.c:314-352)
  m.y0.assign(size_t(4) * Nx, 0.0);
  if (d.initial == "user_defined") {
    std::vector<double> ur(Nx), ui(Nx, 0.0), er(Nx), ei(Nx, 0.0);
    for (int j = 0; j < Nx; ++j) { ur[j] = m.temp_u[j] * (1 - m.dampchar[j]); er[j] = m.temp_wave[j] * (1 - m.dampchar[j]); }
    host_dft(ur, ui, -1);
    host_dft(er, ei, -1);
    for (int j = 0; j < Nx; ++j) {
      m.y0[j] = er[j]; m.y0[j + Nx] = ei[j]; m.y0[j + 2 * Nx] = ur[j]; m.y0[j + 3 * Nx] = ui[j];
    }
  }
  return true;
}

bool jonswap_params(const std::string& dir, bool* is_jonswap, double* T0, double* Tend, double* dt, double* Tp,
                    double* Hs, double* gamma, double* nTramp, std::string& err) {
  Deck d;
  if (!parse_input(dir, d, err)) return false;
  *is_jonswap = d.wavename == "jonswap";
  if (!*is_jonswap) return true;
  InputFile in(dir + "/input.txt");
  FILE* f = in.get();
  in.skip_lines(5, 256);
  if (std::fscanf(f, "%*s %*s %lf \n %*s %*s %lf \n %*s %*s %lf\n", T0, Tend, dt) != 3 ||
      std::fscanf(f, "%*s %*s %lf \n %*s %*s %lf \n %*s %*s %lf\n", Tp, Hs, gamma) != 3) {
    err = "malformed time/spectrum block in input.txt";
    return false;
  }
  *nTramp = d.rampbool == "no" ? 0.0 : d.nTramp;
  return true;
}

double linear_wavenumber(double w, double d) { return invers_omega(w, d); }
int closest_index(const std::vector<double>& a, double ref) { return closest(a, ref); }

}  // namespace hw
