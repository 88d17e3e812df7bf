// hw_engine.cu -- kernels, host engine and C ABI of the B200 HAWASSI 1D engine.
//
// One member (tank realisation) is advanced by one thread-block cluster of C
// CTAs (C = N / M, slice M <= 2048 points, M / 8 threads per CTA).  One launch
// per (M, C) class advances every member of that class through its output
// samples, the whole RKF45 loop (stages, error norm, step control, retries)
// staying on the device.  Classes run concurrently on forked streams.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/hawassi_b200.h"
#include "hw_kernels.h"
#include "hw_kin.h"
#include "hw_setup.hpp"

using namespace hwdev;

namespace {

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
// clear the budget status so that a bounded launch can continue where it stopped, and
// set every member's stop index for the coming launch
__global__ void k_resume(DevMember* mems, int n, const int* __restrict__ stops) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (mems[i].status == kBudget) mems[i].status = kOk;
  mems[i].i_stop = stops[i];
}

// Longest-first order of a class's members for its next launch: the CTAs of a launch
// start roughly in block order, so the members that took the most RHS evaluations in
// the previous launch start first and the launch's tail is shorter.  The members are
// independent: their order changes no result.  One block; ties keep member order.
__global__ void k_order_class(const DevMember* __restrict__ mems, int* list, int n, long long* prev) {
  extern __shared__ long long key[];
  int* id = reinterpret_cast<int*>(key + n);
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const int m = list[j];
    id[j] = m;
    key[j] = mems[m].rhs_calls - prev[m];
  }
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const long long kj = key[j];
    const int mj = id[j];
    int r = 0;
    for (int k = 0; k < n; ++k) r += (key[k] > kj) || (key[k] == kj && id[k] < mj);
    list[r] = mj;
    prev[mj] = mems[mj].rhs_calls;
  }
}

// reference layout (4N doubles) -> internal (2N double2, spectral permuted)
__global__ void k_to_internal(const double* __restrict__ ref, double2* __restrict__ dst, int N, int logC, int M) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  const int C = 1 << logC;
  const int p = (q & (C - 1)) * M + (q >> logC);
  dst[p] = make_double2(ref[q], ref[N + q]);
  dst[N + p] = make_double2(ref[2 * N + q], ref[3 * N + q]);
}

__global__ void k_to_reference(const double2* __restrict__ src, double* __restrict__ ref, int N, int logC, int M) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  const int C = 1 << logC;
  const int p = (q & (C - 1)) * M + (q >> logC);
  const double2 e = src[p], u = src[N + p];
  ref[q] = e.x;
  ref[N + q] = e.y;
  ref[2 * N + q] = u.x;
  ref[3 * N + q] = u.y;
}

// every member's state at once: member m = blockIdx.y reads its current state
// pointer from its descriptor on the device (the stepper swaps buffers), so a whole
// ensemble moves with one host copy and one launch, without host round trips
__global__ void k_states_to_internal(DevMember* mems, const double* __restrict__ stage,
                                     const long long* __restrict__ off) {
  DevMember& d = mems[blockIdx.y];
  const double* ref = stage + off[blockIdx.y];
  const int N = d.N, C = d.C, M = d.M, logC = d.logC;
  double2* dst = d.y;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < N; q += gridDim.x * blockDim.x) {
    const int p = (q & (C - 1)) * M + (q >> logC);
    dst[p] = make_double2(ref[q], ref[N + q]);
    dst[N + p] = make_double2(ref[2 * N + q], ref[3 * N + q]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) d.k1_valid = 0;   // the state changed under the stepper
}

__global__ void k_states_to_reference(const DevMember* __restrict__ mems, double* __restrict__ stage,
                                      const long long* __restrict__ off) {
  const DevMember& d = mems[blockIdx.y];
  double* ref = stage + off[blockIdx.y];
  const int N = d.N, C = d.C, M = d.M, logC = d.logC;
  const double2* src = d.y;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < N; q += gridDim.x * blockDim.x) {
    const int p = (q & (C - 1)) * M + (q >> logC);
    const double2 e = src[p], u = src[N + p];
    ref[q] = e.x;
    ref[N + q] = e.y;
    ref[2 * N + q] = u.x;
    ref[3 * N + q] = u.y;
  }
}

// ---------------------------------------------------------------------------
// host engine
// ---------------------------------------------------------------------------
#define HW_CUDA(call)                                                                       \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) {                                                                \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);                             \
      return false;                                                                         \
    }                                                                                       \
  } while (0)

struct Arena {
  char* base = nullptr;
  size_t used = 0, cap = 0;
  template <class T>
  T* take(size_t n) {
    size_t off = (used + 255) & ~size_t(255);
    used = off + n * sizeof(T);
    return reinterpret_cast<T*>(base + off);
  }
};

struct HostMember {
  hw::Member m;
  int N = 0, C = 1, M = 0, logC = 0;
  DevMember d{};
  void* dev = nullptr;       // arena base
  size_t dev_bytes = 0;
  double* fields = nullptr;  // per-sample eta, u, phi when the member keeps fields
  double t0 = 0, h0 = 0;
  hwkin::Kin* kin = nullptr; // kinematics tables (made by the first kinematics call)
};

struct Class {
  int M, C;
  std::vector<int> members;
  int* d_list = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  cudaEvent_t t_start = nullptr, t_stop = nullptr;   // timing of the last evolve launch
  int* d_queue = nullptr;   // work-queue counter of the persistent evolve grid
  int grid = 0;             // resident clusters of the persistent grid (0: one per member)
};

}  // namespace

struct hw_ctx {
  std::vector<HostMember> mem;
  std::vector<Class> classes;
  DevMember* d_mems = nullptr;
  std::vector<std::pair<int, double2*>> tw;   // twiddle tables per N
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  int* d_single = nullptr;    // one-member list for single-member launches
  int* d_stops = nullptr;     // stop index of every member for the next launch
  long long* d_prev_rhs = nullptr;   // each member's RHS count when its class was last ordered
  double* d_ref = nullptr;    // 4*maxN staging for reference-layout transfers
  int maxN = 0;
  double* d_stage = nullptr;  // all members' states, reference layout, concatenated
  long long* d_off = nullptr; // offset of each member in d_stage
  size_t stage_doubles = 0;
  bool ensure_stage();
  int device = 0;
  std::string err;

  bool init(const std::vector<std::string>& dirs, const hw_opts* o, const int* member_slice = nullptr);
  bool upload_member(HostMember& h);
  bool launch_class(const Class& c, const int* list, int nblocks_members, int mode, cudaStream_t s);
  bool launch_member(int mi, int mode, double t_rhs);
  bool run(int i_stop_all, double t_end, bool by_time, const int* per_member = nullptr);
  bool sync_desc();
  bool reset();
  ~hw_ctx();
};

static std::string g_create_err;

// no-allocation RHS (hw_noalloc.cu)
int hw_noalloc_max_nx();
bool hw_noalloc_rhs_launch(DevMember* mems, int mi, int N, int M, int C, double t, const double* y,
                           double* dy, cudaStream_t s, int dev, std::string& err);

namespace {

std::vector<double> permute(const std::vector<double>& v, int N, int C, int M) {
  std::vector<double> r(N);
  for (int q = 0; q < N; ++q) r[(q % C) * M + q / C] = v[q];
  return r;
}

cudaError_t launch_any(int M, int mode, DevMember* mems, const int* list, int nmem, int C, double t, cudaStream_t s,
                       int* queue = nullptr, int ngrid = 0) {
  switch (M) {
    case 256: return hw_launch_256(mode, mems, list, nmem, C, t, s, queue, ngrid);
    case 512: return hw_launch_512(mode, mems, list, nmem, C, t, s, queue, ngrid);
    case 1024: return hw_launch_1024(mode, mems, list, nmem, C, t, s, queue, ngrid);
    case 2048: return hw_launch_2048(mode, mems, list, nmem, C, t, s, queue, ngrid);
    default: return cudaErrorInvalidValue;
  }
}

int max_clusters_any(int M, int C) {
  switch (M) {
    case 256: return hw_max_clusters_256(C);
    case 512: return hw_max_clusters_512(C);
    case 1024: return hw_max_clusters_1024(C);
    case 2048: return hw_max_clusters_2048(C);
    default: return 0;
  }
}

}  // namespace

bool hw_ctx::upload_member(HostMember& h) {
  const hw::Member& m = h.m;
  const int N = h.N, C = h.C, M = h.M, K = m.flat ? 0 : m.nref, n = m.n;
  // size the arena
  size_t bytes = 0;
  auto add = [&](size_t b) { bytes += ((b + 255) / 256) * 256; };
  for (int i = 0; i < 10 + 2; ++i) add(sizeof(double) * N);                 // real tables
  add(sizeof(double2) * N * 2);                                              // gamX, gamXs
  add(sizeof(double) * size_t(N) * std::max(K, 1) * 2);                      // Csq, gam
  for (int i = 0; i < 5; ++i) add(sizeof(double) * std::max(n, 2));          // splines
  add(sizeof(double2) * size_t(2 * N) * 10);                                 // y, ynew, kb[7], zs
  add(sizeof(double2) * size_t(N) * kScratch);
  const int cap = std::max(N / 4, 4);
  add(sizeof(BrkDev));
  add(sizeof(Crest) * cap * 3);
  add(sizeof(int) * (cap + 3 * N + 8));
  add(sizeof(double) * N);
  const long long log_cap = m.breaking ? (1LL << 22) : 16;
  add(sizeof(double) * log_cap);
  const int ng = int(m.gauge.size());
  add(sizeof(double) * N);                                                   // grid x
  add(sizeof(double) * std::max(ng, 1));                                     // gauge positions
  add(sizeof(int) * std::max(ng, 1));                                        // gauge intervals
  add(sizeof(double) * size_t(std::max(n, 1)) * 2 * std::max(ng, 1));        // gauge series
  add(sizeof(double) * size_t(std::max(n, 1)));                              // sample times
  bytes += 4096;
  HW_CUDA(cudaMalloc(&h.dev, bytes));
  HW_CUDA(cudaMemset(h.dev, 0, bytes));
  h.dev_bytes = bytes;
  Arena a;
  a.base = static_cast<char*>(h.dev);
  a.cap = bytes;
  DevMember& d = h.d;
  std::memset(&d, 0, sizeof d);
  d.N = N; d.C = C; d.M = M; d.logC = h.logC;
  d.model = m.model; d.flat = m.flat ? 1 : 0; d.nref = K; d.brk = m.breaking ? 1 : 0;
  d.has_influx = m.has_influx ? 1 : 0; d.prop_mode = m.prop_mode; d.n_in = n;
  d.invN = 1.0 / N; d.dx = m.dx; d.eps_abs = m.eps_abs; d.eps_rel = m.eps_rel;
  auto up = [&](const std::vector<double>& v, size_t cnt) -> double* {
    double* p = a.take<double>(cnt);
    if (!v.empty()) cudaMemcpy(p, v.data(), sizeof(double) * std::min(cnt, v.size()), cudaMemcpyHostToDevice);
    return p;
  };
  std::vector<double> c1(N), gk(N);
  for (int i = 0; i < N; ++i) {
    c1[i] = (m.Csqr[i] / hwdev::kG) * m.k[i];
    gk[i] = hwdev::kG * m.k[i];
  }
  d.k = up(permute(m.k, N, C, M), N);
  d.aal = up(permute(m.aal, N, C, M), N);
  d.c1 = up(permute(c1, N, C, M), N);
  d.gk = up(permute(gk, N, C, M), N);
  d.M0im = up(permute(m.M0im, N, C, M), N);
  d.L = up(permute(m.L, N, C, M), N);
  {
    std::vector<double> g(2 * N), s(2 * N);
    std::vector<double> pr = permute(m.gamX_re, N, C, M), pi = permute(m.gamX_im, N, C, M);
    std::vector<double> qr = permute(m.gamXs_re, N, C, M), qi = permute(m.gamXs_im, N, C, M);
    for (int i = 0; i < N; ++i) { g[2 * i] = pr[i]; g[2 * i + 1] = pi[i]; s[2 * i] = qr[i]; s[2 * i + 1] = qi[i]; }
    d.gamX = reinterpret_cast<const double2*>(up(g, 2 * N));
    d.gamXs = reinterpret_cast<const double2*>(up(s, 2 * N));
  }
  {
    std::vector<double> cs(size_t(N) * std::max(K, 1), 0.0), gm(size_t(N) * std::max(K, 1), 0.0);
    for (int j = 0; j < K; ++j) {
      std::vector<double> pc = permute(m.Csq_ref[j], N, C, M);
      std::copy(pc.begin(), pc.end(), cs.begin() + size_t(j) * N);
      std::copy(m.gam_ref[j].begin(), m.gam_ref[j].end(), gm.begin() + size_t(j) * N);
    }
    d.Csq = up(cs, cs.size());
    d.gam = up(gm, gm.size());
  }
  d.dcoef = up(m.dampcoef, N);
  d.dchar = up(m.dampchar, N);
  d.chi = up(m.ChiAdj, N);
  d.depth = up(m.depth, N);
  const size_t ns = size_t(std::max(n, 2));
  d.tt = up(m.ttrace, ns);
  d.ins = up(m.insig, ns);
  d.insc = up(m.sp_c_in.empty() ? std::vector<double>(ns, 0.0) : m.sp_c_in, ns);
  d.skw = up(m.insig_skew, ns);
  d.skwc = up(m.sp_c_skew.empty() ? std::vector<double>(ns, 0.0) : m.sp_c_skew, ns);
  double2* twp = nullptr;
  for (auto& e : tw)
    if (e.first == N) twp = e.second;
  if (!twp) {
    std::vector<double2> t(N);
    for (int q = 0; q < N; ++q) {
      // exp(-2 pi i q / N), argument reduced to the first octant for accuracy
      const double a = 2.0 * M_PI * double(q) / double(N);
      t[q] = make_double2(std::cos(a), -std::sin(a));
    }
    HW_CUDA(cudaMalloc(&twp, sizeof(double2) * N));
    HW_CUDA(cudaMemcpy(twp, t.data(), sizeof(double2) * N, cudaMemcpyHostToDevice));
    tw.emplace_back(N, twp);
  }
  d.tw = twp;
  d.KBC = m.KBC; d.TC = m.TC; d.Tstar = m.Tstar; d.MaxEtaInit = m.MaxEtaInit; d.dt_in = m.dt;
  d.xbstart = m.xbstart; d.xbend = m.xbend; d.xbendL = m.xbendL; d.xbstartR = m.xbstartR;
  d.lenIF = m.lenIF; d.ILL = m.ILL; d.IFF = m.IFF;
  // output stage: gauges (interval index by GSL's bsearch rule)
  d.ngauge = ng;
  d.xg = up(m.x, N);
  d.gpos = up(m.gauge, size_t(std::max(ng, 1)));
  {
    std::vector<int> gi(size_t(std::max(ng, 1)), -1);
    for (int g = 0; g < ng; ++g) {
      const double xq = m.gauge[g];
      if (!(xq >= m.x[0] && xq <= m.x[N - 1])) continue;
      int lo = 0, hi = N - 1;
      while (hi > lo + 1) {
        const int i = (hi + lo) / 2;
        if (m.x[i] > xq) hi = i; else lo = i;
      }
      gi[g] = lo;
    }
    int* p = a.take<int>(gi.size());
    cudaMemcpy(p, gi.data(), sizeof(int) * gi.size(), cudaMemcpyHostToDevice);
    d.gidx = p;
  }
  d.gout = a.take<double>(size_t(std::max(n, 1)) * 2 * std::max(ng, 1));
  d.gtim = a.take<double>(size_t(std::max(n, 1)));
  d.y = a.take<double2>(2 * N);
  d.ynew = a.take<double2>(2 * N);
  for (int i = 0; i < 7; ++i) d.kb[i] = a.take<double2>(2 * N);
  d.zs = a.take<double2>(2 * N);
  for (int i = 0; i < kScratch; ++i) d.sc[i] = a.take<double2>(N);
  // breaking state
  BrkDev bk{};
  bk.cap = cap;
  BrkDev* dbk = a.take<BrkDev>(1);
  bk.cb = a.take<Crest>(cap);
  bk.cbn = a.take<Crest>(cap);
  bk.cbp = a.take<Crest>(cap);
  bk.id_node_end = a.take<int>(cap);
  bk.nodes = a.take<int>(N);
  bk.touched = a.take<int>(N);
  bk.pk = a.take<int>(N);
  bk.B = a.take<double>(N);
  bk.log = a.take<double>(size_t(log_cap));
  bk.log_cap = log_cap;
  HW_CUDA(cudaMemcpy(dbk, &bk, sizeof bk, cudaMemcpyHostToDevice));
  d.bk = dbk;
  if (a.used > a.cap) { err = "internal: arena overflow"; return false; }
  // initial state
  d.t = m.ttrace[0];
  d.h = m.h0;
  h.t0 = d.t;
  h.h0 = d.h;
  d.i_out = 0;
  d.i_stop = 0;
  d.status = kOk;
  d.exact = m.breaking ? 1 : 0;
  d.rhs_budget = 400000;   // RHS evaluations per member and launch
  double* tmp = nullptr;
  HW_CUDA(cudaMalloc(&tmp, sizeof(double) * 4 * N));
  HW_CUDA(cudaMemcpy(tmp, m.y0.data(), sizeof(double) * 4 * N, cudaMemcpyHostToDevice));
  k_to_internal<<<(N + 255) / 256, 256>>>(tmp, d.y, N, h.logC, M);
  HW_CUDA(cudaGetLastError());
  HW_CUDA(cudaDeviceSynchronize());
  cudaFree(tmp);
  return true;
}

bool hw_ctx::init(const std::vector<std::string>& dirs, const hw_opts* o, const int* member_slice) {
  hw_opts opt{};
  if (o) opt = *o;
  device = opt.device;
  HW_CUDA(cudaSetDevice(device));
  int ndev = 0;
  HW_CUDA(cudaGetDeviceCount(&ndev));
  for (cudaError_t e : {hw_attr_256(), hw_attr_512(), hw_attr_1024(), hw_attr_2048()})
    if (e != cudaSuccess) { err = std::string("kernel attributes: ") + cudaGetErrorString(e); return false; }
  hw::SetupOptions so;
  so.eps_abs = opt.eps_abs;
  so.eps_rel = opt.eps_rel;
  so.h0 = opt.h0;
  so.seed = opt.seed;
  so.nref = opt.nref;
  // jonswap decks: every member's influx signal in one device launch; member i
  // draws its phases from seed + i
  std::vector<std::vector<double>> js_sig(dirs.size());
  {
    std::vector<hw_jonswap> specs;
    std::vector<size_t> who;
    for (size_t i = 0; i < dirs.size(); ++i) {
      bool isj = false;
      hw_jonswap sp{};
      if (!hw::jonswap_params(dirs[i], &isj, &sp.T0, &sp.Tend, &sp.dt, &sp.Tp, &sp.Hs, &sp.gamma, &sp.nTramp, err)) {
        err = dirs[i] + ": " + err;
        return false;
      }
      if (!isj) continue;
      sp.seed = opt.seed + (unsigned long long)i;
      specs.push_back(sp);
      who.push_back(i);
    }
    if (!specs.empty()) {
      const int total = hw_jonswap_influx(specs.data(), int(specs.size()), nullptr, 0, device);
      std::vector<double> all(total > 0 ? size_t(total) : 0);
      if (total <= 0 || hw_jonswap_influx(specs.data(), int(specs.size()), all.data(), total, device) != total) {
        err = "jonswap influx synthesis on the device failed";
        return false;
      }
      size_t off = 0;
      for (size_t k = 0; k < specs.size(); ++k) {
        const int nt = int((specs[k].Tend - specs[k].T0) / specs[k].dt + 1);
        js_sig[who[k]].assign(all.begin() + long(off), all.begin() + long(off + size_t(nt)));
        off += size_t(nt);
      }
    }
  }
  mem.resize(dirs.size());
  for (size_t i = 0; i < dirs.size(); ++i) {
    HostMember& h = mem[i];
    so.seed = opt.seed + (unsigned long long)i;
    so.influx_eta = js_sig[i].empty() ? nullptr : &js_sig[i];
    if (!hw::build_member(dirs[i], so, h.m, err)) {
      err = dirs[i] + ": " + err;
      return false;
    }
    const int N = h.m.Nx;
    if (N < 256 || (N & (N - 1)) != 0 || N > 32768) {
      err = dirs[i] + ": the device engine needs a power-of-two grid with 256 <= Nx <= 32768 (Nx=" +
            std::to_string(N) + ")";
      return false;
    }
    if (h.m.breaking && h.m.prop_mode == 2) {
      err = dirs[i] + ": bidirectional breaking windows are not supported on the device";
      return false;
    }
    h.N = N;
    const int slice = (member_slice && member_slice[i] > 0) ? member_slice[i] : (opt.slice > 0 ? opt.slice : 2048);
    int C = opt.cluster > 0 ? opt.cluster : std::max(1, N / slice);
    if ((C & (C - 1)) != 0 || N / C < 256 || N / C > 2048 || C > 16) {
      err = "invalid cluster size " + std::to_string(C) + " for Nx=" + std::to_string(N);
      return false;
    }
    h.C = C;
    h.M = N / C;
    h.logC = 0;
    while ((1 << h.logC) < C) ++h.logC;
    maxN = std::max(maxN, N);
    if (!upload_member(h)) return false;
    if (opt.exact_sequence) h.d.exact = 1;
  }
  HW_CUDA(cudaMalloc(&d_mems, sizeof(DevMember) * mem.size()));
  for (size_t i = 0; i < mem.size(); ++i)
    HW_CUDA(cudaMemcpy(d_mems + i, &mem[i].d, sizeof(DevMember), cudaMemcpyHostToDevice));
  HW_CUDA(cudaMalloc(&d_single, sizeof(int) * mem.size()));
  HW_CUDA(cudaMalloc(&d_stops, sizeof(int) * mem.size()));
  HW_CUDA(cudaMalloc(&d_prev_rhs, sizeof(long long) * mem.size()));
  HW_CUDA(cudaMemset(d_prev_rhs, 0, sizeof(long long) * mem.size()));
  std::vector<int> ids(mem.size());
  for (size_t i = 0; i < mem.size(); ++i) ids[i] = int(i);
  HW_CUDA(cudaMemcpy(d_single, ids.data(), sizeof(int) * ids.size(), cudaMemcpyHostToDevice));
  HW_CUDA(cudaMalloc(&d_ref, sizeof(double) * 4 * maxN));
  HW_CUDA(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
  stream = own_stream;
  HW_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  // group members by (M, C); heavier members first inside each class
  for (size_t i = 0; i < mem.size(); ++i) {
    Class* cls = nullptr;
    for (auto& c : classes)
      if (c.M == mem[i].M && c.C == mem[i].C) cls = &c;
    if (!cls) {
      classes.push_back(Class{mem[i].M, mem[i].C, {}, nullptr, nullptr, nullptr, nullptr, nullptr});
      cls = &classes.back();
    }
    cls->members.push_back(int(i));
  }
  for (auto& c : classes) {
    HW_CUDA(cudaMalloc(&c.d_list, sizeof(int) * c.members.size()));
    HW_CUDA(cudaMemcpy(c.d_list, c.members.data(), sizeof(int) * c.members.size(), cudaMemcpyHostToDevice));
    HW_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    HW_CUDA(cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming));
    HW_CUDA(cudaEventCreate(&c.t_start));
    HW_CUDA(cudaEventCreate(&c.t_stop));
    HW_CUDA(cudaMalloc(&c.d_queue, sizeof(int)));
  }
  // evolve grids: one cluster per member (resident == 0, the default: measured the
  // fastest), or a persistent grid whose clusters pull members from the class's queue --
  // at most `resident` clusters, or (resident < 0) the class's share of the resident
  // clusters by grid points (members x CTAs), a quarter over so that a class that
  // drains its queue early leaves its slots to the waiting clusters of the others
  double total = 0.0;
  for (const auto& c : classes) total += double(c.members.size()) * c.C;
  for (auto& c : classes) {
    const int nm = int(c.members.size());
    if (opt.resident == 0) {
      c.grid = 0;
    } else if (opt.resident > 0) {
      c.grid = std::min(nm, opt.resident);
    } else {
      const int maxc = max_clusters_any(c.M, c.C);
      const double share = double(nm) * c.C / total;
      c.grid = maxc > 0 ? std::min(nm, std::max(1, int(std::ceil(1.25 * maxc * share)))) : 0;
    }
  }
  return true;
}

bool hw_ctx::launch_member(int mi, int mode, double t_rhs) {
  const HostMember& h = mem[size_t(mi)];
  cudaError_t e = launch_any(h.M, mode, d_mems, d_single + mi, 1, h.C, t_rhs, stream);
  if (e != cudaSuccess) { err = std::string("launch: ") + cudaGetErrorString(e); return false; }
  return true;
}

bool hw_ctx::run(int i_stop_all, double t_end, bool by_time, const int* per_member) {
  // stop indices of the members, set on the device descriptors with one copy
  std::vector<int> stops(mem.size());
  for (size_t i = 0; i < mem.size(); ++i) {
    const hw::Member& m = mem[i].m;
    int stop = m.n;
    if (per_member) {
      stop = per_member[i] < 0 ? 0 : std::min(per_member[i], m.n);
    } else if (by_time) {
      stop = 0;
      while (stop < m.n && m.ttrace[size_t(stop)] <= t_end) ++stop;
    } else if (i_stop_all >= 0) {
      stop = std::min(i_stop_all, m.n);
    }
    stops[i] = stop;
  }
  // (from pageable memory: the runtime stages the vector before the call returns)
  HW_CUDA(cudaMemcpyAsync(d_stops, stops.data(), sizeof(int) * stops.size(), cudaMemcpyHostToDevice, stream));
  // a member stopped by the per-launch RHS budget resumes here
  k_resume<<<(unsigned(mem.size()) + 127) / 128, 128, 0, stream>>>(d_mems, int(mem.size()), d_stops);
  HW_CUDA(cudaGetLastError());
  HW_CUDA(cudaEventRecord(fork, stream));
  for (auto& c : classes) {
    HW_CUDA(cudaStreamWaitEvent(c.stream, fork, 0));
    HW_CUDA(cudaEventRecord(c.t_start, c.stream));
    const int nm = int(c.members.size());
    k_order_class<<<1, 256, size_t(nm) * (sizeof(long long) + sizeof(int)), c.stream>>>(d_mems, c.d_list, nm,
                                                                                      d_prev_rhs);
    HW_CUDA(cudaGetLastError());
    if (c.grid > 0) HW_CUDA(cudaMemsetAsync(c.d_queue, 0, sizeof(int), c.stream));
    cudaError_t e = launch_any(c.M, 0, d_mems, c.d_list, int(c.members.size()), c.C, 0.0, c.stream,
                               c.grid > 0 ? c.d_queue : nullptr, c.grid);
    if (e != cudaSuccess) { err = std::string("launch: ") + cudaGetErrorString(e); return false; }
    HW_CUDA(cudaEventRecord(c.t_stop, c.stream));
    HW_CUDA(cudaEventRecord(c.done, c.stream));
    HW_CUDA(cudaStreamWaitEvent(stream, c.done, 0));
  }
  return true;
}

bool hw_ctx::sync_desc() {
  HW_CUDA(cudaStreamSynchronize(stream));
  for (size_t i = 0; i < mem.size(); ++i)
    HW_CUDA(cudaMemcpy(&mem[i].d, d_mems + i, sizeof(DevMember), cudaMemcpyDeviceToHost));
  return true;
}

bool hw_ctx::reset() {
  HW_CUDA(cudaStreamSynchronize(stream));
  for (size_t i = 0; i < mem.size(); ++i) {
    HostMember& h = mem[i];
    HW_CUDA(cudaMemcpy(&h.d, d_mems + i, sizeof(DevMember), cudaMemcpyDeviceToHost));
    h.d.t = h.t0;
    h.d.h = h.h0;
    h.d.i_out = 0;
    h.d.status = kOk;
    h.d.k1_valid = 0;
    h.d.rhs_calls = h.d.accepted = h.d.rejected = 0;
    HW_CUDA(cudaMemcpy(d_ref, h.m.y0.data(), sizeof(double) * 4 * h.N, cudaMemcpyHostToDevice));
    k_to_internal<<<(h.N + 255) / 256, 256, 0, stream>>>(d_ref, h.d.y, h.N, h.logC, h.M);
    HW_CUDA(cudaGetLastError());
    // breaking state
    BrkDev bk;
    HW_CUDA(cudaMemcpy(&bk, h.d.bk, sizeof bk, cudaMemcpyDeviceToHost));
    bk.flag = bk.ITERbdt = bk.ITERbn = bk.n_touched = bk.npk = bk.any_above = 0;
    bk.dirty_cb = bk.dirty_cbn = bk.dirty_cbp = 0;
    bk.log_len = 0;
    HW_CUDA(cudaMemset(bk.cb, 0, sizeof(Crest) * bk.cap));
    HW_CUDA(cudaMemset(bk.cbn, 0, sizeof(Crest) * bk.cap));
    HW_CUDA(cudaMemset(bk.cbp, 0, sizeof(Crest) * bk.cap));
    HW_CUDA(cudaMemset(bk.id_node_end, 0, sizeof(int) * bk.cap));
    HW_CUDA(cudaMemset(bk.B, 0, sizeof(double) * h.N));
    HW_CUDA(cudaMemcpy(h.d.bk, &bk, sizeof bk, cudaMemcpyHostToDevice));
    HW_CUDA(cudaMemcpy(d_mems + i, &h.d, sizeof(DevMember), cudaMemcpyHostToDevice));
  }
  HW_CUDA(cudaStreamSynchronize(stream));
  return true;
}

hw_ctx::~hw_ctx() {
  if (stream) cudaStreamSynchronize(stream);
  for (auto& h : mem) {
    if (h.dev) cudaFree(h.dev);
    if (h.fields) cudaFree(h.fields);
    if (h.kin) hwkin::kin_destroy(h.kin);
  }
  for (auto& e : tw) cudaFree(e.second);
  if (d_stage) cudaFree(d_stage);
  if (d_off) cudaFree(d_off);
  for (auto& c : classes) {
    if (c.d_list) cudaFree(c.d_list);
    if (c.d_queue) cudaFree(c.d_queue);
    if (c.stream) cudaStreamDestroy(c.stream);
    if (c.done) cudaEventDestroy(c.done);
    if (c.t_start) cudaEventDestroy(c.t_start);
    if (c.t_stop) cudaEventDestroy(c.t_stop);
  }
  if (d_mems) cudaFree(d_mems);
  if (d_single) cudaFree(d_single);
  if (d_stops) cudaFree(d_stops);
  if (d_prev_rhs) cudaFree(d_prev_rhs);
  if (d_ref) cudaFree(d_ref);
  if (fork) cudaEventDestroy(fork);
  if (own_stream) cudaStreamDestroy(own_stream);
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
namespace {
bool valid_member(hw_ctx* c, int m) {
  if (!c) return false;
  if (m < 0 || m >= int(c->mem.size())) {
    c->err = "member index out of range";
    return false;
  }
  return true;
}
}  // namespace

extern "C" {

hw_ctx* hw_create(const char* workdir, const hw_opts* opts) {
  if (!workdir) { g_create_err = "workdir is NULL"; return nullptr; }
  return hw_ensemble_create(&workdir, 1, opts);
}

hw_ctx* hw_ensemble_create(const char* const* workdirs, int n, const hw_opts* opts) {
  if (!workdirs || n <= 0) { g_create_err = "no member decks given"; return nullptr; }
  std::unique_ptr<hw_ctx> c(new hw_ctx());
  std::vector<std::string> dirs;
  for (int i = 0; i < n; ++i) dirs.emplace_back(workdirs[i] ? workdirs[i] : "");
  if (!c->init(dirs, opts)) {
    g_create_err = c->err;
    return nullptr;
  }
  return c.release();
}

hw_ctx* hw_ensemble_create_sliced(const char* const* workdirs, int n, const hw_opts* opts,
                                  const int* member_slice) {
  if (!workdirs || n <= 0) { g_create_err = "no member decks given"; return nullptr; }
  std::unique_ptr<hw_ctx> c(new hw_ctx());
  std::vector<std::string> dirs;
  for (int i = 0; i < n; ++i) dirs.emplace_back(workdirs[i] ? workdirs[i] : "");
  if (!c->init(dirs, opts, member_slice)) {
    g_create_err = c->err;
    return nullptr;
  }
  return c.release();
}

void hw_destroy(hw_ctx* ctx) { delete ctx; }

const char* hw_last_error(const hw_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_err.c_str(); }

int hw_members(const hw_ctx* ctx) { return ctx ? int(ctx->mem.size()) : 0; }

int hw_nx(const hw_ctx* ctx, int m) {
  if (!ctx || m < 0 || m >= int(ctx->mem.size())) return -1;
  return ctx->mem[size_t(m)].N;
}

int hw_nt(const hw_ctx* ctx, int m) {
  if (!ctx || m < 0 || m >= int(ctx->mem.size())) return -1;
  return ctx->mem[size_t(m)].m.n;
}

int hw_initial_state(hw_ctx* ctx, int m, double* y) {
  if (!valid_member(ctx, m) || !y) return 1;
  const auto& v = ctx->mem[size_t(m)].m.y0;
  std::memcpy(y, v.data(), sizeof(double) * v.size());
  return 0;
}

int hw_rhs(hw_ctx* ctx, int m, double t, const double* y, double* dydt) {
  if (!valid_member(ctx, m) || !y || !dydt) return 1;
  std::string& err = ctx->err;
  auto body = [&]() -> bool {
    HostMember& h = ctx->mem[size_t(m)];
    const int N = h.N;
    HW_CUDA(cudaMemcpyAsync(ctx->d_ref, y, sizeof(double) * 4 * N, cudaMemcpyHostToDevice, ctx->stream));
    k_to_internal<<<(N + 255) / 256, 256, 0, ctx->stream>>>(ctx->d_ref, h.d.zs, N, h.logC, h.M);
    HW_CUDA(cudaGetLastError());
    if (!ctx->launch_member(m, 2, t)) return false;
    DevMember cur;
    HW_CUDA(cudaMemcpyAsync(&cur, ctx->d_mems + m, sizeof cur, cudaMemcpyDeviceToHost, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    k_to_reference<<<(N + 255) / 256, 256, 0, ctx->stream>>>(cur.kb[6], ctx->d_ref, N, h.logC, h.M);
    HW_CUDA(cudaGetLastError());
    HW_CUDA(cudaMemcpyAsync(dydt, ctx->d_ref, sizeof(double) * 4 * N, cudaMemcpyDeviceToHost, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    return true;
  };
  return body() ? 0 : 1;
}

int hw_rhs_noalloc(hw_ctx* ctx, int m, double t, const double* y_dev, double* dydt_dev, void* cuda_stream) {
  if (!valid_member(ctx, m) || !y_dev || !dydt_dev) return 1;
  // the caller's current device is restored on every return path
  int prev = -1;
  cudaError_t e = cudaGetDevice(&prev);
  if (e != cudaSuccess) {
    ctx->err = std::string("hw_rhs_noalloc: cudaGetDevice: ") + cudaGetErrorString(e);
    return 1;
  }
  if (prev != ctx->device && (e = cudaSetDevice(ctx->device)) != cudaSuccess) {
    ctx->err = std::string("hw_rhs_noalloc: cudaSetDevice: ") + cudaGetErrorString(e);
    return 1;
  }
  const HostMember& h = ctx->mem[size_t(m)];
  const bool ok = hw_noalloc_rhs_launch(ctx->d_mems, m, h.N, h.M, h.C, t, y_dev, dydt_dev,
                                        static_cast<cudaStream_t>(cuda_stream), ctx->device, ctx->err);
  if (prev != ctx->device && (e = cudaSetDevice(prev)) != cudaSuccess) {
    ctx->err = std::string("hw_rhs_noalloc: restoring the caller's device: ") + cudaGetErrorString(e);
    return 1;
  }
  return ok ? 0 : 1;
}

int hw_gsl_rhs(double t, const double* y, double* dydt, void* params) {
  return hw_rhs(static_cast<hw_ctx*>(params), 0, t, y, dydt);
}

int hw_set_state(hw_ctx* ctx, int m, double t, double h, const double* y, int i_out) {
  if (!valid_member(ctx, m)) return 1;
  std::string& err = ctx->err;
  auto body = [&]() -> bool {
    HostMember& hm = ctx->mem[size_t(m)];
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    HW_CUDA(cudaMemcpy(&hm.d, ctx->d_mems + m, sizeof(DevMember), cudaMemcpyDeviceToHost));
    if (y) {
      HW_CUDA(cudaMemcpyAsync(ctx->d_ref, y, sizeof(double) * 4 * hm.N, cudaMemcpyHostToDevice, ctx->stream));
      k_to_internal<<<(hm.N + 255) / 256, 256, 0, ctx->stream>>>(ctx->d_ref, hm.d.y, hm.N, hm.logC, hm.M);
      HW_CUDA(cudaGetLastError());
    }
    hm.d.t = t;
    hm.d.h = h;
    hm.d.i_out = i_out;
    hm.d.k1_valid = 0;
    hm.d.status = kOk;
    HW_CUDA(cudaMemcpyAsync(ctx->d_mems + m, &hm.d, sizeof(DevMember), cudaMemcpyHostToDevice, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    return true;
  };
  return body() ? 0 : 1;
}

int hw_evolve_apply(hw_ctx* ctx, int m, double* t, double t1, double* h, double* y) {
  if (!valid_member(ctx, m) || !t || !h || !y) return 1;
  std::string& err = ctx->err;
  auto body = [&]() -> bool {
    HostMember& hm = ctx->mem[size_t(m)];
    const int N = hm.N;
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    HW_CUDA(cudaMemcpy(&hm.d, ctx->d_mems + m, sizeof(DevMember), cudaMemcpyDeviceToHost));
    HW_CUDA(cudaMemcpyAsync(ctx->d_ref, y, sizeof(double) * 4 * N, cudaMemcpyHostToDevice, ctx->stream));
    k_to_internal<<<(N + 255) / 256, 256, 0, ctx->stream>>>(ctx->d_ref, hm.d.y, N, hm.logC, hm.M);
    HW_CUDA(cudaGetLastError());
    hm.d.t = *t;
    hm.d.h = *h;
    hm.d.t1 = t1;
    hm.d.k1_valid = 0;
    hm.d.status = kOk;
    HW_CUDA(cudaMemcpyAsync(ctx->d_mems + m, &hm.d, sizeof(DevMember), cudaMemcpyHostToDevice, ctx->stream));
    if (!ctx->launch_member(m, 1, 0.0)) return false;
    HW_CUDA(cudaMemcpyAsync(&hm.d, ctx->d_mems + m, sizeof(DevMember), cudaMemcpyDeviceToHost, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    k_to_reference<<<(N + 255) / 256, 256, 0, ctx->stream>>>(hm.d.y, ctx->d_ref, N, hm.logC, hm.M);
    HW_CUDA(cudaGetLastError());
    HW_CUDA(cudaMemcpyAsync(y, ctx->d_ref, sizeof(double) * 4 * N, cudaMemcpyDeviceToHost, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    *t = hm.d.t;
    *h = hm.d.h;
    return true;
  };
  if (!body()) return 1;
  const int st = ctx->mem[size_t(m)].d.status;
  if (st != kOk) {
    ctx->err = "time integration failed (status " + std::to_string(st) + ")";
    return 100 + st;
  }
  return 0;
}

int hw_run(hw_ctx* ctx, int i_stop) {
  if (!ctx) return 1;
  return ctx->run(i_stop, 0.0, false) ? 0 : 1;
}

int hw_run_members(hw_ctx* ctx, const int* i_stop) {
  if (!ctx || !i_stop) return 1;
  return ctx->run(-1, 0.0, false, i_stop) ? 0 : 1;
}

int hw_run_to_time(hw_ctx* ctx, double t_end) {
  if (!ctx) return 1;
  return ctx->run(-1, t_end, true) ? 0 : 1;
}

int hw_get_state(hw_ctx* ctx, int m, double* t, double* h, double* y) {
  if (!valid_member(ctx, m)) return 1;
  std::string& err = ctx->err;
  auto body = [&]() -> bool {
    HostMember& hm = ctx->mem[size_t(m)];
    HW_CUDA(cudaMemcpyAsync(&hm.d, ctx->d_mems + m, sizeof(DevMember), cudaMemcpyDeviceToHost, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    if (t) *t = hm.d.t;
    if (h) *h = hm.d.h;
    if (y) {
      k_to_reference<<<(hm.N + 255) / 256, 256, 0, ctx->stream>>>(hm.d.y, ctx->d_ref, hm.N, hm.logC, hm.M);
      HW_CUDA(cudaGetLastError());
      HW_CUDA(cudaMemcpyAsync(y, ctx->d_ref, sizeof(double) * 4 * hm.N, cudaMemcpyDeviceToHost, ctx->stream));
      HW_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return true;
  };
  return body() ? 0 : 1;
}

int hw_reset(hw_ctx* ctx) { return ctx && ctx->reset() ? 0 : 1; }

int hw_member_stats(hw_ctx* ctx, int m, long long* rhs, long long* acc, long long* rej, int* status) {
  if (!valid_member(ctx, m)) return 1;
  std::string& err = ctx->err;
  auto body = [&]() -> bool {
    HostMember& hm = ctx->mem[size_t(m)];
    HW_CUDA(cudaMemcpyAsync(&hm.d, ctx->d_mems + m, sizeof(DevMember), cudaMemcpyDeviceToHost, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    if (rhs) *rhs = hm.d.rhs_calls;
    if (acc) *acc = hm.d.accepted;
    if (rej) *rej = hm.d.rejected;
    if (status) *status = hm.d.status;
    return true;
  };
  return body() ? 0 : 1;
}

int hw_last_dydt(hw_ctx* ctx, int m, double* dydt) {
  if (!valid_member(ctx, m) || !dydt) return 1;
  std::string& err = ctx->err;
  auto body = [&]() -> bool {
    HostMember& hm = ctx->mem[size_t(m)];
    HW_CUDA(cudaMemcpyAsync(&hm.d, ctx->d_mems + m, sizeof(DevMember), cudaMemcpyDeviceToHost, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    // the last evaluation is kout in the exact sequence, k1 after a reuse in the pure one
    const double2* src = hm.d.k1_valid ? hm.d.kb[0] : hm.d.kb[6];
    k_to_reference<<<(hm.N + 255) / 256, 256, 0, ctx->stream>>>(src, ctx->d_ref, hm.N, hm.logC, hm.M);
    HW_CUDA(cudaGetLastError());
    HW_CUDA(cudaMemcpyAsync(dydt, ctx->d_ref, sizeof(double) * 4 * hm.N, cudaMemcpyDeviceToHost, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    return true;
  };
  return body() ? 0 : 1;
}

namespace {
bool ensure_kin(hw_ctx* ctx, int m) {
  HostMember& hm = ctx->mem[size_t(m)];
  if (hm.kin) return true;
  hm.kin = hwkin::kin_create(hm.m, ctx->err);
  return hm.kin != nullptr;
}
}  // namespace

int hw_kinematics_dims(hw_ctx* ctx, int m, int* nx_out, int* nz_out) {
  if (!valid_member(ctx, m) || !ensure_kin(ctx, m)) return 1;
  hwkin::kin_dims(ctx->mem[size_t(m)].kin, nx_out, nz_out);
  return 0;
}

int hw_kinematics_grid(hw_ctx* ctx, int m, double* x_out, double* z_out) {
  if (!valid_member(ctx, m) || !ensure_kin(ctx, m)) return 1;
  hwkin::kin_grid(ctx->mem[size_t(m)].kin, x_out, z_out);
  return 0;
}

int hw_kinematics(hw_ctx* ctx, int m, double tprev, double* eta_cut, double* P, double* dxphi, double* dzphi,
                  double* dtdxphi, double* dtdzphi) {
  if (!valid_member(ctx, m) || !ensure_kin(ctx, m)) return 1;
  std::string& err = ctx->err;
  auto body = [&]() -> bool {
    HostMember& hm = ctx->mem[size_t(m)];
    HW_CUDA(cudaMemcpyAsync(&hm.d, ctx->d_mems + m, sizeof(DevMember), cudaMemcpyDeviceToHost, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    // the state and the RHS the output stage reads (the global dy: kout in the exact
    // sequence, k1 after a reuse in the pure one), in the reference layout
    const double2* src = hm.d.k1_valid ? hm.d.kb[0] : hm.d.kb[6];
    double* yb = hwkin::kin_state_buffer(hm.kin, 0);
    double* db = hwkin::kin_state_buffer(hm.kin, 1);
    k_to_reference<<<(hm.N + 255) / 256, 256, 0, ctx->stream>>>(hm.d.y, yb, hm.N, hm.logC, hm.M);
    k_to_reference<<<(hm.N + 255) / 256, 256, 0, ctx->stream>>>(src, db, hm.N, hm.logC, hm.M);
    HW_CUDA(cudaGetLastError());
    if (!hwkin::kin_run(hm.kin, yb, db, hm.d.t, tprev, ctx->stream, err)) return false;
    return hwkin::kin_fetch(hm.kin, eta_cut, P, dxphi, dzphi, dtdxphi, dtdzphi, ctx->stream, err);
  };
  return body() ? 0 : 1;
}

int hw_breaking_log(hw_ctx* ctx, int m, double* out, long long cap, long long* len) {
  if (!valid_member(ctx, m)) return -1;
  std::string& err = ctx->err;
  long long recs = 0;
  auto body = [&]() -> bool {
    HostMember& hm = ctx->mem[size_t(m)];
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    BrkDev bk;
    HW_CUDA(cudaMemcpy(&bk, hm.d.bk, sizeof bk, cudaMemcpyDeviceToHost));
    const long long n = std::min(bk.log_len, cap);
    if (len) *len = bk.log_len;
    if (out && n > 0) HW_CUDA(cudaMemcpy(out, bk.log, sizeof(double) * size_t(n), cudaMemcpyDeviceToHost));
    recs = bk.ITERbn;
    return true;
  };
  return body() ? int(recs) : -1;
}

int hw_deck_table(const char* workdir, const hw_opts* opts, const char* name, double* out, int cap) {
  if (!workdir || !name) { g_create_err = "NULL argument"; return -1; }
  hw_opts o{};
  if (opts) o = *opts;
  hw::SetupOptions so;
  so.eps_abs = o.eps_abs; so.eps_rel = o.eps_rel; so.h0 = o.h0; so.seed = o.seed; so.nref = o.nref;
  hw::Member m;
  if (!hw::build_member(workdir, so, m, g_create_err)) return -1;
  const std::string nm(name);
  std::vector<double> v;
  if (nm == "x") v = m.x; else if (nm == "k") v = m.k; else if (nm == "depth") v = m.depth;
  else if (nm == "dampchar") v = m.dampchar; else if (nm == "dampcoef") v = m.dampcoef;
  else if (nm == "aal") v = m.aal; else if (nm == "ChiAdj") v = m.ChiAdj; else if (nm == "Csqr") v = m.Csqr;
  else if (nm == "L") v = m.L; else if (nm == "M0im") v = m.M0im; else if (nm == "insig") v = m.insig;
  else if (nm == "insig_skew") v = m.insig_skew; else if (nm == "ttrace") v = m.ttrace; else if (nm == "y0") v = m.y0;
  else if (nm == "gamX") { v = m.gamX_re; v.insert(v.end(), m.gamX_im.begin(), m.gamX_im.end()); }
  else if (nm == "gamX_skew") { v = m.gamXs_re; v.insert(v.end(), m.gamXs_im.begin(), m.gamXs_im.end()); }
  else if (nm == "CsqK" || nm == "gamK") {
    for (const auto& r : (nm == "CsqK" ? m.Csq_ref : m.gam_ref)) v.insert(v.end(), r.begin(), r.end());
  }
  else if (nm.rfind("gam_", 0) == 0 || nm.rfind("Csq_", 0) == 0) {
    // gam_min / gam_plus / gam_mid and Csq_* in the reference's naming (ref order min, plus, mid)
    const int j = nm.find("min") != std::string::npos ? 0 : nm.find("plus") != std::string::npos ? 1 : 2;
    const auto& src = nm[0] == 'g' ? m.gam_ref : m.Csq_ref;
    if (j < int(src.size())) v = src[size_t(j)];
  } else {
    const double s = nm == "Nx" ? m.Nx : nm == "n" ? m.n : nm == "dx" ? m.dx : nm == "dt" ? m.dt
                   : nm == "nu_peak" ? m.nu_peak : nm == "kp" ? m.kp : nm == "lambda_p" ? m.lambda_p
                   : nm == "Hs_in" ? m.Hs_in : nm == "MaxEtaInit" ? m.MaxEtaInit : nm == "depthinf" ? m.depthinf
                   : nm == "Tstar" ? m.Tstar : nm == "xbstart" ? m.xbstart : nm == "xbend" ? m.xbend
                   : nm == "cutfracwn" ? m.cutfracwn : nm == "Tp_peak" ? m.Tp_peak : std::nan("");
    if (std::isnan(s)) { g_create_err = "unknown table " + nm; return -1; }
    v.assign(1, s);
  }
  const int n = std::min(cap, int(v.size()));
  if (out) std::memcpy(out, v.data(), sizeof(double) * size_t(n));
  return int(v.size());
}

bool hw_ctx::ensure_stage() {
  if (d_stage) return true;
  std::vector<long long> off(mem.size());
  size_t tot = 0;
  for (size_t i = 0; i < mem.size(); ++i) {
    off[i] = (long long)tot;
    tot += size_t(4) * mem[i].N;
  }
  HW_CUDA(cudaMalloc(&d_stage, sizeof(double) * std::max<size_t>(tot, 1)));
  HW_CUDA(cudaMalloc(&d_off, sizeof(long long) * std::max<size_t>(off.size(), 1)));
  HW_CUDA(cudaMemcpy(d_off, off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice));
  stage_doubles = tot;
  return true;
}

// every member's state to the host (concatenated reference layouts): one batched
// layout kernel and one copy, ordered after the work already on the stream
int hw_get_states(hw_ctx* ctx, double* y_all) {
  if (!ctx || !y_all) return 1;
  std::string& err = ctx->err;
  auto body = [&]() -> bool {
    if (!ctx->ensure_stage()) return false;
    const dim3 grid(unsigned((ctx->maxN + 255) / 256), unsigned(ctx->mem.size()));
    k_states_to_reference<<<grid, 256, 0, ctx->stream>>>(ctx->d_mems, ctx->d_stage, ctx->d_off);
    HW_CUDA(cudaGetLastError());
    HW_CUDA(cudaMemcpyAsync(y_all, ctx->d_stage, sizeof(double) * ctx->stage_doubles, cudaMemcpyDeviceToHost,
                            ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    return true;
  };
  return body() ? 0 : 1;
}

// every member's state from the host: one copy and one batched layout kernel on the
// stream (the next run starts after it, with each member's dydt_in recomputed)
int hw_set_states(hw_ctx* ctx, const double* y_all) {
  if (!ctx || !y_all) return 1;
  std::string& err = ctx->err;
  auto body = [&]() -> bool {
    if (!ctx->ensure_stage()) return false;
    HW_CUDA(cudaMemcpyAsync(ctx->d_stage, y_all, sizeof(double) * ctx->stage_doubles, cudaMemcpyHostToDevice,
                            ctx->stream));
    const dim3 grid(unsigned((ctx->maxN + 255) / 256), unsigned(ctx->mem.size()));
    k_states_to_internal<<<grid, 256, 0, ctx->stream>>>(ctx->d_mems, ctx->d_stage, ctx->d_off);
    HW_CUDA(cudaGetLastError());
    for (auto& hm : ctx->mem) hm.d.k1_valid = 0;
    return true;
  };
  return body() ? 0 : 1;
}

int hw_class_timing(hw_ctx* ctx, double* ms, int* members, int* grid_n, int cap) {
  if (!ctx) return -1;
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return -1;
  const int n = int(ctx->classes.size());
  for (int i = 0; i < n && i < cap; ++i) {
    Class& c = ctx->classes[size_t(i)];
    float f = 0.f;
    if (ms) ms[i] = cudaEventElapsedTime(&f, c.t_start, c.t_stop) == cudaSuccess ? double(f) : -1.0;
    if (members) members[i] = int(c.members.size());
    if (grid_n) grid_n[i] = c.M * c.C;
  }
  return n;
}

int hw_set_operator_weights(hw_ctx* ctx, int m, int K, const double* depths, const double* gam) {
  if (!valid_member(ctx, m) || !depths || !gam) return 1;
  HostMember& h = ctx->mem[size_t(m)];
  if (h.m.flat || K != h.d.nref) {
    ctx->err = "operator weights need a varying-depth member created with nref = " + std::to_string(K);
    return 1;
  }
  std::string& err = ctx->err;
  auto body = [&]() -> bool {
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    const int N = h.N;
    for (int j = 0; j < K; ++j) {
      std::vector<double> row = permute(hw::csq_row(h.m.k, depths[j]), N, h.C, h.M);
      HW_CUDA(cudaMemcpy(const_cast<double*>(h.d.Csq) + size_t(j) * N, row.data(), sizeof(double) * N,
                         cudaMemcpyHostToDevice));
      HW_CUDA(cudaMemcpy(const_cast<double*>(h.d.gam) + size_t(j) * N, gam + size_t(j) * N, sizeof(double) * N,
                         cudaMemcpyHostToDevice));
      h.m.Csq_ref[size_t(j)] = hw::csq_row(h.m.k, depths[j]);
      h.m.gam_ref[size_t(j)].assign(gam + size_t(j) * N, gam + size_t(j + 1) * N);
    }
    return true;
  };
  return body() ? 0 : 1;
}

int hw_energy(hw_ctx* ctx, int m, const double* y, double* energy) {
  if (!valid_member(ctx, m) || !energy) return 1;
  const hw::Member& mb = ctx->mem[size_t(m)].m;
  const int N = mb.Nx;
  std::vector<double> own;
  if (!y) {
    own.resize(size_t(4) * N);
    if (hw_get_state(ctx, m, nullptr, nullptr, own.data()) != 0) return 1;
    y = own.data();
  }
  // quadratic Hamiltonian 1/2 int (g eta^2 + u (C^2/g) u) dx in spectral form (Parseval),
  // C^2 at the depth of the influx point
  double s = 0.0;
  for (int k = 0; k < N; ++k) {
    const double e2 = y[k] * y[k] + y[N + k] * y[N + k];
    const double u2 = y[2 * N + k] * y[2 * N + k] + y[3 * N + k] * y[3 * N + k];
    s += hwdev::kG * e2 + mb.Csqr[size_t(k)] / hwdev::kG * u2;
  }
  *energy = 0.5 * s * mb.dx / N;
  return 0;
}

int hw_gauges(hw_ctx* ctx, int member, double* eta, double* dteta, double* tim, int cap) {
  if (!ctx || member < 0 || member >= int(ctx->mem.size())) return -1;
  if (!ctx->sync_desc()) return -1;
  const HostMember& h = ctx->mem[size_t(member)];
  const int ng = h.d.ngauge;
  const int rows = std::min(h.d.i_out, cap);
  if (rows <= 0) return 0;
  if (ng > 0 && (eta || dteta)) {
    std::vector<double> buf(size_t(rows) * 2 * ng);
    if (cudaMemcpy(buf.data(), h.d.gout, sizeof(double) * buf.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
      ctx->err = "gauge read-back failed";
      return -1;
    }
    for (int r = 0; r < rows; ++r)
      for (int g = 0; g < ng; ++g) {
        if (eta) eta[size_t(r) * ng + g] = buf[size_t(r) * 2 * ng + g];
        if (dteta) dteta[size_t(r) * ng + g] = buf[size_t(r) * 2 * ng + ng + g];
      }
  }
  if (tim && cudaMemcpy(tim, h.d.gtim, sizeof(double) * rows, cudaMemcpyDeviceToHost) != cudaSuccess) {
    ctx->err = "gauge read-back failed";
    return -1;
  }
  return rows;
}

int hw_enable_fields(hw_ctx* ctx, int member, int enable) {
  if (!valid_member(ctx, member)) return 1;
  std::string& err = ctx->err;
  auto body = [&]() -> bool {
    HostMember& hm = ctx->mem[size_t(member)];
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    if (enable && !hm.fields) {
      const size_t cnt = size_t(std::max(hm.m.n, 1)) * 3 * size_t(hm.N);
      HW_CUDA(cudaMalloc(&hm.fields, sizeof(double) * cnt));
    }
    double* p = enable ? hm.fields : nullptr;
    HW_CUDA(cudaMemcpy(&ctx->d_mems[member].fields, &p, sizeof(double*), cudaMemcpyHostToDevice));
    hm.d.fields = p;
    return true;
  };
  return body() ? 0 : 1;
}

// The reference's output files of one member from the device-computed samples
// (1d/functions.c:557-760): per partition of NtoutIP = n / npartition samples a
// Constants_NN.dat (print_xt, :784-801) and Hawassi_eta/u/phi_NN.dat (Nx doubles per
// sample); the gauge text files (print_data_gauge, :500-522); breaking.dat.
int hw_write_outputs(hw_ctx* ctx, int member, const char* outdir) {
  if (!valid_member(ctx, member) || !outdir) return -1;
  if (!ctx->sync_desc()) return -1;
  HostMember& hm = ctx->mem[size_t(member)];
  const hw::Member& m = hm.m;
  const int N = hm.N, n = m.n, rows = hm.d.i_out;
  const std::string dir(outdir);
  std::vector<double> tim(size_t(std::max(rows, 1)));
  if (rows > 0 && cudaMemcpy(tim.data(), hm.d.gtim, sizeof(double) * rows, cudaMemcpyDeviceToHost) != cudaSuccess) {
    ctx->err = "output read-back failed";
    return -1;
  }
  if (hm.fields && rows > 0) {
    const int npart = std::max(m.deck.npartition, 1);
    const int ntout = n / npart, ntrest = n - npart * ntout;
    std::vector<double> f(size_t(rows) * 3 * N);
    if (cudaMemcpy(f.data(), hm.fields, sizeof(double) * f.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
      ctx->err = "field read-back failed";
      return -1;
    }
    FILE *fe = nullptr, *fu = nullptr, *fp = nullptr;
    int ip = 0;
    auto closeall = [&]() {
      if (fe) std::fclose(fe);
      if (fu) std::fclose(fu);
      if (fp) std::fclose(fp);
      fe = fu = fp = nullptr;
    };
    for (int i = 0; i < rows; ++i) {
      if (ntout > 0 && i % ntout == 0) {
        ++ip;
        closeall();
        char sfx[32];
        std::snprintf(sfx, sizeof sfx, "%02d.dat", ip);
        // print_xt: the rest partition is recognised by its length (N1 == Ntrest)
        const int n1 = ip <= npart ? ntout : ntrest;
        FILE* fc = std::fopen((dir + "/Constants_" + sfx).c_str(), "wb");
        if (!fc) { ctx->err = "cannot write " + dir; return -1; }
        const double NX = double(N), NT = double(n1);
        std::fwrite(&NX, sizeof(double), 1, fc);
        std::fwrite(m.x.data(), sizeof(double), size_t(N), fc);
        std::fwrite(&NT, sizeof(double), 1, fc);
        const size_t t0 = n1 == ntrest ? size_t(npart) * ntout : size_t(ip - 1) * ntout;
        std::fwrite(m.ttrace.data() + t0, sizeof(double), size_t(n1), fc);
        std::fwrite(m.depth.data(), sizeof(double), size_t(N), fc);
        std::fwrite(m.k.data(), sizeof(double), size_t(N), fc);
        std::fwrite(&m.nu_peak, sizeof(double), 1, fc);
        std::fclose(fc);
        fe = std::fopen((dir + "/Hawassi_eta_" + sfx).c_str(), "wb");
        fu = std::fopen((dir + "/Hawassi_u_" + sfx).c_str(), "wb");
        fp = std::fopen((dir + "/Hawassi_phi_" + sfx).c_str(), "wb");
        if (!fe || !fu || !fp) { closeall(); ctx->err = "cannot write " + dir; return -1; }
      }
      const double* r = f.data() + size_t(i) * 3 * N;
      std::fwrite(r, sizeof(double), size_t(N), fe);
      std::fwrite(r + N, sizeof(double), size_t(N), fu);
      std::fwrite(r + 2 * N, sizeof(double), size_t(N), fp);
    }
    closeall();
  }
  const int ng = hm.d.ngauge;
  if (ng > 0 && rows > 0) {
    std::vector<double> g(size_t(rows) * 2 * ng);
    if (cudaMemcpy(g.data(), hm.d.gout, sizeof(double) * g.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
      ctx->err = "gauge read-back failed";
      return -1;
    }
    FILE* f1 = std::fopen((dir + "/Hawassi_eta_gauge.txt").c_str(), "w");
    FILE* f2 = std::fopen((dir + "/Hawassi_dteta_gauge.txt").c_str(), "w");
    if (!f1 || !f2) {
      if (f1) std::fclose(f1);
      if (f2) std::fclose(f2);
      ctx->err = "cannot write " + dir;
      return -1;
    }
    std::fprintf(f1, "0 ");
    std::fprintf(f2, "0 ");
    for (int j = 0; j < ng; ++j) {
      std::fprintf(f1, "%f ", m.gauge[size_t(j)]);
      std::fprintf(f2, "%f ", m.gauge[size_t(j)]);
    }
    std::fprintf(f1, "\n");
    std::fprintf(f2, "\n");
    for (int i = 0; i < rows; ++i) {
      std::fprintf(f1, "%f ", tim[size_t(i)]);
      std::fprintf(f2, "%f ", tim[size_t(i)]);
      for (int j = 0; j < ng; ++j) {
        std::fprintf(f1, "%f ", g[size_t(i) * 2 * ng + j]);
        std::fprintf(f2, "%f ", g[size_t(i) * 2 * ng + ng + j]);
      }
      std::fprintf(f1, "\n");
      std::fprintf(f2, "\n");
    }
    std::fclose(f1);
    std::fclose(f2);
  }
  if (m.breaking) {
    long long len = 0;
    if (hw_breaking_log(ctx, member, nullptr, 0, &len) < 0) return -1;
    std::vector<double> lg(size_t(std::max(len, 1LL)));
    if (len > 0 && hw_breaking_log(ctx, member, lg.data(), len, &len) < 0) return -1;
    FILE* fb = std::fopen((dir + "/breaking.dat").c_str(), "w");
    if (!fb) { ctx->err = "cannot write " + dir; return -1; }
    for (long long i = 0; i + 1 < len;) {   // records: t, count, nodes (1d/breaking.c:434)
      const int cnt = int(lg[size_t(i + 1)]);
      std::fprintf(fb, "%lf %d ", lg[size_t(i)], cnt);
      for (int q = 0; q < cnt; ++q) std::fprintf(fb, "%d ", int(lg[size_t(i + 2 + q)]));
      std::fprintf(fb, "\n");
      i += 2 + cnt;
    }
    std::fclose(fb);
  }
  return rows;
}

int hw_ngauge(const hw_ctx* ctx, int member) {
  if (!ctx || member < 0 || member >= int(ctx->mem.size())) return -1;
  return int(ctx->mem[size_t(member)].m.gauge.size());
}

int hw_set_stream(hw_ctx* ctx, void* s) {
  if (!ctx) return 1;
  ctx->stream = s ? static_cast<cudaStream_t>(s) : ctx->own_stream;
  return 0;
}

int hw_synchronize(hw_ctx* ctx) {
  if (!ctx) return 1;
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    ctx->err = cudaGetErrorString(e);
    return 1;
  }
  return 0;
}

}  // extern "C"
