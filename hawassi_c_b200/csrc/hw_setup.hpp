// hw_setup.hpp -- host-side deck parsing and table construction for one HAWASSI
// 1D member (a tank realisation).  Everything here runs once per member, on the
// host, before the device engine takes over; it mirrors the reference's set-up
// order in 1d/main.cc:42-205.
#pragma once

#include <string>
#include <vector>

namespace hw {

struct SetupOptions {
  double eps_abs = 0.0;   // <= 0: reference 1e-5 (1d/functions.c:529)
  double eps_rel = 0.0;   // <= 0: reference 1e-4 (1d/functions.c:530)
  double h0 = 0.0;        // <= 0: reference 1e-4 (1d/functions.c:541)
  unsigned long long seed = 0;  // phase seed for wavename = jonswap
  int nref = 0;           // 0/3: three reference depths (Up3IP); 2: Up2IP; >3: log-spaced K refs
  // wavename = jonswap: the influx signal already synthesised (on the device, for a
  // whole ensemble at once); nullptr: synthesise it here
  const std::vector<double>* influx_eta = nullptr;
};

// The time and spectrum block of a jonswap deck (1d/influx_lib.c:1-109) with the ramp
// length (0 when ramp_influx is no, 1d/main.cc:47-49).  Returns false with err on a
// malformed deck; *is_jonswap false for other wavenames.
bool jonswap_params(const std::string& dir, bool* is_jonswap, double* T0, double* Tend, double* dt, double* Tp,
                    double* Hs, double* gamma, double* nTramp, std::string& err);

// Deck values as read from input.txt (1d/read_input.c:1-60, 1d/influx_lib.c:1-109).
struct Deck {
  std::string wavename, initial, bath, dynmodel, breaking, friction, influxing, propagation,
      kinematic, wall, coupling, rampbool, cut_temp, mid_temp, min_z, max_z;
  double depthflat = 0, adjcoef = 0, parKBC = 0, parTC = 0, parTchar = 0, nTramp = 0;
  int ngauge = 0, npartition = 0;
  double T0 = 0, Tend = 0, dt = 0, Tp = 0, Hs = 0, gamJS = 0;
  double Xstart = 0, Xend = 0, Xinflux = 0, dx = 0, dampL = 0, dampR = 0;
  double xinterv1 = 0, xinterv2 = 0;   // &IF KINEMATIC block (1d/read_input.c:42-44)
  int nsurf = 0, ndeep = 0;
};

// All per-member tables in the reference's natural index order (FFTW order for
// spectral quantities, grid order for physical ones).
struct Member {
  Deck deck;
  int Nx = 0, n = 0;           // grid points, influx/output samples
  int model = 2;               // 1, 2, 3 (HS1..HS3)
  bool flat = true;
  bool has_influx = false;
  bool breaking = false;
  int prop_mode = 0;           // 0 Uni+, 1 Uni-, 2 Bi, 3 none
  int cutfracwn = 4;
  int nref = 3;                // reference depths used by the varying-depth operator
  double length = 0, dx = 0, dt = 0, depthinf = 0, nu_peak = 0, kp = 0, Tp_peak = 0,
         lambda_p = 0, Hs_in = 0, MaxEtaInit = 0, Xinflux = 0;
  double eps_abs = 1e-5, eps_rel = 1e-4, h0 = 1e-4;
  int idx_inf = 0;

  std::vector<double> x, k, depth, dampchar, dampcoef, aal, ChiAdj, Csqr, L, M0im;
  std::vector<double> gamX_re, gamX_im, gamXs_re, gamXs_im;
  std::vector<std::vector<double>> Csq_ref, gam_ref;   // [nref][Nx]
  std::vector<double> ttrace, insig, insig_skew, sp_c_in, sp_c_skew;  // influx splines
  std::vector<double> temp_wave, temp_u;               // initial.dat (if user_defined)
  std::vector<double> gauge;

  // kinematic breaking (1d/breaking.c:1-34)
  double KBC = 0, TC = 0, Tstar = 0;
  int xbstart = 0, xbend = 0, xbendL = 0, xbstartR = 0, lenIF = 0, ILL = 0, IFF = 0;

  // initial spectral state, reference layout [Re eta^|Im eta^|Re u^|Im u^]
  std::vector<double> y0;
};

// Parse <dir>/input.txt and the files it names, build every table.  Returns
// false with a message in err on malformed or unsupported input.
bool build_member(const std::string& dir, const SetupOptions& opt, Member& m, std::string& err);

// C^2(k, D) for every wavenumber of k (exact dispersion, 1d/functions.c:1415)
std::vector<double> csq_row(const std::vector<double>& k, double D);

// Host FFT used by the set-up (any length; FFTW sign convention, unnormalised).
void host_dft(std::vector<double>& re, std::vector<double>& im, int sign);

// GSL-compatible natural cubic spline second-derivative coefficients (c_i).
std::vector<double> natural_spline_c(const std::vector<double>& x, const std::vector<double>& y);
double natural_spline_eval(const std::vector<double>& x, const std::vector<double>& y,
                           const std::vector<double>& c, double t);

// invers_omega (1d/functions.c:984-1020) and closest (1d/functions.c:1761), as the
// set-up uses them, for the kinematics tables
double linear_wavenumber(double w, double d);
int closest_index(const std::vector<double>& a, double ref);

}  // namespace hw
