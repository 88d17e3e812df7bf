// hw2d_engine.cu -- C ABI of the 2D flat-bottom engine: tables upload, the
// RHS entry points and the device-resident rkf45 loop.
//
// One step attempt is a fixed launch sequence captured once as a CUDA graph:
//   [RHS k1, if needed] [RHS stages 2..6] combine control [RHS k_out, if accepted] finalize
// Every kernel reads the device control block (t, h, h0, done, buffer indices)
// and does nothing once the target time is reached, so the host replays the
// graph in batches and reads the control block back between batches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hawassi_b200.h"
#include "hw2d.cuh"
#include "hw2d_brk.cuh"
#include "hw2d_gen.cuh"
#include "hw2d_hs3.cuh"
#include "hw2d_out.cuh"
#include "hw2d_var.cuh"
#include "hw2d_wall.cuh"
#include "hw_setup.hpp"

using hw2d::Ctl2;
using hw2d::RK2;
using hw2d::Tab2;
using hw2d::Work2;

namespace {

std::string g_err2d;

constexpr int kMinM = 64, kMaxM = 1024;
constexpr long long kMaxAttemptsPerRun = 2000000;

template <int M>
size_t smem_bytes(int slices) { return (size_t)slices * hwdev::padded(M) * sizeof(double2); }

template <int M>
void set_attrs() {
  cudaFuncSetAttribute(hw2d::k2_rowA<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(6));
  cudaFuncSetAttribute(hw2d::k2_colB<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(8));
  cudaFuncSetAttribute(hw2d::k2_rowC<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(8));
  cudaFuncSetAttribute(hw2d::k2_colD<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(10));
  cudaFuncSetAttribute(hw2d::k2_rowE<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(8));
  cudaFuncSetAttribute(hw2d::k2v_rowA<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(8));
  cudaFuncSetAttribute(hw2d::k2v_colB<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(12));
  cudaFuncSetAttribute(hw2d::k2v_rowC<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(12));
  cudaFuncSetAttribute(hw2d::k2v_colD<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(6));
  cudaFuncSetAttribute(hw2d::k2v_rowE<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(6));
  cudaFuncSetAttribute(hw2d::k2v_colF<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(8));
  cudaFuncSetAttribute(hw2d::k2v_rowG<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(8));
  cudaFuncSetAttribute(hw2d::k2b_rowI<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(2));
  cudaFuncSetAttribute(hw2d::k2b_colI<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(2));
  cudaFuncSetAttribute(hw2d::k2b_sbcol<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(2));
  cudaFuncSetAttribute(hw2d::k2b_sbrow<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(2));
  cudaFuncSetAttribute(hw2d::k2w_row1<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(2));
  cudaFuncSetAttribute(hw2d::k2w_col2<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(2));
  cudaFuncSetAttribute(hw2d::k2w_row3<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(2));
  cudaFuncSetAttribute(hw2d::k2w_rowV1<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(4));
  cudaFuncSetAttribute(hw2d::k2w_colV2<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(4));
  cudaFuncSetAttribute(hw2d::k2w_rowV3<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(2));
  cudaFuncSetAttribute(hw2d::k2_colB3<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(10));
  cudaFuncSetAttribute(hw2d::k2_rowC3<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(10));
  cudaFuncSetAttribute(hw2d::k2_colH3<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(6));
  cudaFuncSetAttribute(hw2d::k2_rowI3<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(8));
  cudaFuncSetAttribute(hw2d::k2o_row<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(4));
  cudaFuncSetAttribute(hw2d::k2o_col<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(4));
  cudaFuncSetAttribute(hw2d::k2g_rows<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(4));
  cudaFuncSetAttribute(hw2d::k2g_cols<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<M>(4));
}

// the general path's transform passes over nf consecutive fields (rows: M = nx,
// four rows per CTA; columns: M = ny, four columns per CTA)
template <int M>
void launch_gen(int cols, double2* f, int nf, int nx, int ny, const double2* tw, int sign, cudaStream_t s,
                const Ctl2* ctl, int cond) {
  const int blk = hw2d::kGroups * (M / 8);
  if (!cols)
    hw2d::k2g_rows<M><<<dim3(ny / hw2d::kGroups, nf), blk, smem_bytes<M>(4), s>>>(f, nx, ny, tw, sign, ctl, cond);
  else
    hw2d::k2g_cols<M><<<dim3(nx / 4, nf), blk, smem_bytes<M>(4), s>>>(f, nx, ny, tw, sign, ctl, cond);
}
void gen_pass(int M, int cols, double2* f, int nf, int nx, int ny, const double2* tw, int sign, cudaStream_t s,
              const Ctl2* ctl, int cond) {
  switch (M) {
    case 64: launch_gen<64>(cols, f, nf, nx, ny, tw, sign, s, ctl, cond); break;
    case 128: launch_gen<128>(cols, f, nf, nx, ny, tw, sign, s, ctl, cond); break;
    case 256: launch_gen<256>(cols, f, nf, nx, ny, tw, sign, s, ctl, cond); break;
    case 512: launch_gen<512>(cols, f, nf, nx, ny, tw, sign, s, ctl, cond); break;
    default: launch_gen<1024>(cols, f, nf, nx, ny, tw, sign, s, ctl, cond); break;
  }
}

// the first kernel of a general-path RHS: counts the call when it runs
__global__ void k2g_count(hw2d::Ctl2* ctl, int cond) {
  if (hw2d::rhs_active(ctl, cond)) ctl->rhs += 1;
}

// the output stage's two passes (row M = nx, column M = ny)
template <int M>
void launch_out(int which, int nblocks, cudaStream_t s, const Tab2& tb, const double2* z, double2* P, double* phys,
                float* f32) {
  const int blk = hw2d::kGroups * (M / 8);
  if (which == 0) hw2d::k2o_row<M><<<nblocks, blk, smem_bytes<M>(4), s>>>(tb, z, P);
  else hw2d::k2o_col<M><<<nblocks, blk, smem_bytes<M>(4), s>>>(tb, P, phys, f32);
}
void out_pass(int M, int which, int nb, cudaStream_t s, const Tab2& tb, const double2* z, double2* P, double* phys,
              float* f32) {
  switch (M) {
    case 64: launch_out<64>(which, nb, s, tb, z, P, phys, f32); break;
    case 128: launch_out<128>(which, nb, s, tb, z, P, phys, f32); break;
    case 256: launch_out<256>(which, nb, s, tb, z, P, phys, f32); break;
    case 512: launch_out<512>(which, nb, s, tb, z, P, phys, f32); break;
    default: launch_out<1024>(which, nb, s, tb, z, P, phys, f32); break;
  }
}

// the flat bottom's wall round trip (row M = nx, column M = ny)
template <int M>
void launch_wall(int which, int nblocks, cudaStream_t s, const Tab2& tb, const Work2& w, const Ctl2* ctl, int cond) {
  const int blk = hw2d::kGroups * (M / 8);
  if (which == 0) hw2d::k2w_row1<M><<<nblocks, blk, smem_bytes<M>(2), s>>>(tb, w, ctl, cond);
  else if (which == 1) hw2d::k2w_col2<M><<<nblocks, blk, smem_bytes<M>(2), s>>>(tb, w, ctl, cond);
  else if (which == 2) hw2d::k2w_row3<M><<<nblocks, blk, smem_bytes<M>(2), s>>>(tb, w, ctl, cond);
  else if (which == 3) hw2d::k2w_rowV1<M><<<nblocks, blk, smem_bytes<M>(4), s>>>(tb, w, ctl, cond);
  else if (which == 4) hw2d::k2w_colV2<M><<<nblocks, blk, smem_bytes<M>(4), s>>>(tb, w, ctl, cond);
  else hw2d::k2w_rowV3<M><<<nblocks, blk, smem_bytes<M>(2), s>>>(tb, w, ctl, cond);
}
void wall_pass(int M, int which, int nb, cudaStream_t s, const Tab2& tb, const Work2& w, const Ctl2* ctl, int cond) {
  switch (M) {
    case 64: launch_wall<64>(which, nb, s, tb, w, ctl, cond); break;
    case 128: launch_wall<128>(which, nb, s, tb, w, ctl, cond); break;
    case 256: launch_wall<256>(which, nb, s, tb, w, ctl, cond); break;
    case 512: launch_wall<512>(which, nb, s, tb, w, ctl, cond); break;
    default: launch_wall<1024>(which, nb, s, tb, w, ctl, cond); break;
  }
}

// the breaking kernels of one RHS (row passes: row length M = nx; column passes: M = ny)
template <int M>
void launch_brk_row(int which, int nblocks, cudaStream_t s, const Tab2& tb, const Work2& w, const hw2d::Brk2& b,
                    const RK2& rk, const Ctl2* ctl, int mode, int cond, double2* out) {
  const int blk = hw2d::kGroups * (M / 8);
  if (which == 0) hw2d::k2b_rowI<M><<<nblocks, blk, smem_bytes<M>(2), s>>>(tb, w, b, rk, ctl, mode, cond, out);
  else hw2d::k2b_sbrow<M><<<nblocks, blk, smem_bytes<M>(2), s>>>(tb, b, rk, ctl, mode, cond, out);
}
template <int M>
void launch_brk_col(int which, int nblocks, cudaStream_t s, const Tab2& tb, const Work2& w, const hw2d::Brk2& b,
                    const Ctl2* ctl, int mode, int cond) {
  const int blk = hw2d::kGroups * (M / 8);
  if (which == 0) hw2d::k2b_colI<M><<<nblocks, blk, smem_bytes<M>(2), s>>>(tb, b, ctl, mode, cond);
  else hw2d::k2b_sbcol<M><<<nblocks, blk, smem_bytes<M>(2), s>>>(tb, w, b, ctl, mode, cond);
}
void brk_row(int M, int which, int nb, cudaStream_t s, const Tab2& tb, const Work2& w, const hw2d::Brk2& b,
             const RK2& rk, const Ctl2* ctl, int mode, int cond, double2* out) {
  switch (M) {
    case 64: launch_brk_row<64>(which, nb, s, tb, w, b, rk, ctl, mode, cond, out); break;
    case 128: launch_brk_row<128>(which, nb, s, tb, w, b, rk, ctl, mode, cond, out); break;
    case 256: launch_brk_row<256>(which, nb, s, tb, w, b, rk, ctl, mode, cond, out); break;
    case 512: launch_brk_row<512>(which, nb, s, tb, w, b, rk, ctl, mode, cond, out); break;
    default: launch_brk_row<1024>(which, nb, s, tb, w, b, rk, ctl, mode, cond, out); break;
  }
}
void brk_col(int M, int which, int nb, cudaStream_t s, const Tab2& tb, const Work2& w, const hw2d::Brk2& b,
             const Ctl2* ctl, int mode, int cond) {
  switch (M) {
    case 64: launch_brk_col<64>(which, nb, s, tb, w, b, ctl, mode, cond); break;
    case 128: launch_brk_col<128>(which, nb, s, tb, w, b, ctl, mode, cond); break;
    case 256: launch_brk_col<256>(which, nb, s, tb, w, b, ctl, mode, cond); break;
    case 512: launch_brk_col<512>(which, nb, s, tb, w, b, ctl, mode, cond); break;
    default: launch_brk_col<1024>(which, nb, s, tb, w, b, ctl, mode, cond); break;
  }
}

// the five kernels of one RHS for a row length Mx and a column length My
template <int M>
void launch_row(int which, int nblocks, cudaStream_t s, const Tab2& tb, const Work2& w, const RK2& rk,
                const Ctl2* ctl, Ctl2* ctlw, int mode, int cond, double2* out) {
  const dim3 blk(hw2d::kGroups * (M / 8));
  if (which == 0) hw2d::k2_rowA<M><<<nblocks, blk, smem_bytes<M>(6), s>>>(tb, w, rk, ctl, ctlw, mode, cond);
  else if (which == 2) hw2d::k2_rowC<M><<<nblocks, blk, smem_bytes<M>(8), s>>>(tb, w, ctl, cond);
  else if (which == 10) hw2d::k2v_rowA<M><<<nblocks, blk, smem_bytes<M>(8), s>>>(tb, w, rk, ctl, ctlw, mode, cond);
  else if (which == 12) hw2d::k2v_rowC<M><<<nblocks, blk, smem_bytes<M>(12), s>>>(tb, w, ctl, cond);
  else if (which == 14) hw2d::k2v_rowE<M><<<nblocks, blk, smem_bytes<M>(6), s>>>(tb, w, ctl, cond);
  else if (which == 16) hw2d::k2v_rowG<M><<<nblocks, blk, smem_bytes<M>(8), s>>>(tb, w, ctl, cond);
  else if (which == 20) hw2d::k2_rowC3<M><<<nblocks, blk, smem_bytes<M>(10), s>>>(tb, w, ctl, cond);
  else if (which == 22) hw2d::k2_rowI3<M><<<nblocks, blk, smem_bytes<M>(8), s>>>(tb, w, ctl, cond);
  else hw2d::k2_rowE<M><<<nblocks, blk, smem_bytes<M>(8), s>>>(tb, w, rk, ctl, mode, cond, out);
}
template <int M>
void launch_col(int which, int nblocks, cudaStream_t s, const Tab2& tb, const Work2& w, const Ctl2* ctl, int cond) {
  const dim3 blk(hw2d::kGroups * (M / 8));
  if (which == 1) hw2d::k2_colB<M><<<nblocks, blk, smem_bytes<M>(8), s>>>(tb, w, ctl, cond);
  else if (which == 11) hw2d::k2v_colB<M><<<nblocks, blk, smem_bytes<M>(12), s>>>(tb, w, ctl, cond);
  else if (which == 13) hw2d::k2v_colD<M><<<nblocks, blk, smem_bytes<M>(6), s>>>(tb, w, ctl, cond);
  else if (which == 15) hw2d::k2v_colF<M><<<nblocks, blk, smem_bytes<M>(8), s>>>(tb, w, ctl, cond);
  else if (which == 21) hw2d::k2_colB3<M><<<nblocks, blk, smem_bytes<M>(10), s>>>(tb, w, ctl, cond);
  else if (which == 23) hw2d::k2_colH3<M><<<nblocks, blk, smem_bytes<M>(6), s>>>(tb, w, ctl, cond);
  else hw2d::k2_colD<M><<<nblocks, blk, smem_bytes<M>(10), s>>>(tb, w, ctl, cond);
}

void row_dispatch(int M, int which, int nb, cudaStream_t s, const Tab2& tb, const Work2& w, const RK2& rk,
                  const Ctl2* ctl, Ctl2* ctlw, int mode, int cond, double2* out) {
  switch (M) {
    case 64: launch_row<64>(which, nb, s, tb, w, rk, ctl, ctlw, mode, cond, out); break;
    case 128: launch_row<128>(which, nb, s, tb, w, rk, ctl, ctlw, mode, cond, out); break;
    case 256: launch_row<256>(which, nb, s, tb, w, rk, ctl, ctlw, mode, cond, out); break;
    case 512: launch_row<512>(which, nb, s, tb, w, rk, ctl, ctlw, mode, cond, out); break;
    default: launch_row<1024>(which, nb, s, tb, w, rk, ctl, ctlw, mode, cond, out); break;
  }
}
void col_dispatch(int M, int which, int nb, cudaStream_t s, const Tab2& tb, const Work2& w, const Ctl2* ctl,
                  int cond) {
  switch (M) {
    case 64: launch_col<64>(which, nb, s, tb, w, ctl, cond); break;
    case 128: launch_col<128>(which, nb, s, tb, w, ctl, cond); break;
    case 256: launch_col<256>(which, nb, s, tb, w, ctl, cond); break;
    case 512: launch_col<512>(which, nb, s, tb, w, ctl, cond); break;
    default: launch_col<1024>(which, nb, s, tb, w, ctl, cond); break;
  }
}

void set_all_attrs() {
  static bool done[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || done[dev]) return;
  set_attrs<64>(); set_attrs<128>(); set_attrs<256>(); set_attrs<512>(); set_attrs<1024>();
  cudaFuncSetAttribute(hw2d::k2b_sort, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(hw2d::kBrkPeakCap * sizeof(int)));
  done[dev] = true;
}

std::vector<double2> twiddles(int n) {
  std::vector<double2> t(n);
  for (int q = 0; q < n; ++q) {
    const double a = 2.0 * M_PI * double(q) / double(n);
    t[q] = make_double2(std::cos(a), -std::sin(a));
  }
  return t;
}

bool pow2_in_range(int v) { return v >= kMinM && v <= kMaxM && (v & (v - 1)) == 0; }

}  // namespace

struct hw2d_ctx {
  int device = 0;
  int nx = 0, ny = 0;
  size_t n = 0;
  cudaStream_t own_stream = nullptr, stream = nullptr;
  Tab2 tb{};
  Work2 w{};
  RK2 rk{};
  Ctl2* ctl = nullptr;     // device
  Ctl2* hctl = nullptr;    // pinned host copy
  hw2d::Brk2 brk{};        // kinematic breaking (brk.on = 0: off)
  double* dref = nullptr;  // 6n staging for reference-layout transfers
  double2* dout = nullptr; // 3n direct RHS output
  std::vector<void*> allocs;
  cudaGraphExec_t attempt = nullptr;
  cudaStream_t graph_stream = nullptr;
  double h_first = 0.0;
  // output stage (allocated at first use)
  double2* oP = nullptr;    // 2n packed transforms
  double* ophys = nullptr;  // 3n eta, u, v
  float* of32 = nullptr;    // 3n float copies
  float* hf32 = nullptr;    // pinned host copy of of32
  int* ogpt = nullptr;      // gauge grid points
  double* ogval = nullptr;  // 3 values per gauge
  double* hgval = nullptr;  // pinned host copy of ogval
  int ogcap = 0;
  long long launches = 0;   // kernels issued (graph nodes counted one by one)
  int per_rhs = 5;
  std::string err;

  template <class T>
  T* dalloc(size_t count) {
    void* p = nullptr;
    if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) return nullptr;
    allocs.push_back(p);
    return static_cast<T*>(p);
  }
  template <class T>
  T* upload(const std::vector<T>& v) {
    T* p = dalloc<T>(v.size());
    if (p && cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
    return p;
  }
  // a failed runtime call: record it (with the call's own error) and return 1
  int fail(const char* what, cudaError_t e) {
    err = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    return 1;
  }
  bool check(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      err = std::string(what) + ": " + cudaGetErrorString(e);
      return false;
    }
    return true;
  }
  // ---- the general varying-bottom path (hw2d_gen.cuh) ----
  // pool of complex N-point fields; the numbered slots below
  enum GenSlot {
    gEH = 0, gP = 3, gCU = 6, gCV = 7, gD = 8, gH1 = 11, gM = 13, gEM0U = 16, gEU = 17, gEM0V = 18, gEV = 19,
    gDH2 = 20, gEM0UH = 21, gEM0VH = 22, gLU = 23, gLV = 24, gADJIN = 25, gADJ = 29, gSRC = 33, gHSS = 34,
    // HS3
    gLMU = 43, gLMV = 44, gDIVG = 45, gLELP = 46, gDXU = 47, gDYV = 48, gE2U = 49, gE2V = 50, gPK = 51, gPH = 55,
    gDH3 = 59, gLP = 60, gADJ3IN = 64, gADJ3 = 68, gSlotsHS2 = 43, gSlotsHS3 = 72
  };
  int gen = 0;              // 1: the general path serves this bottom / model
  double2* gpool = nullptr;
  int gcount = 0;           // kernels of the RHS being issued
  double2* G(int i) const { return gpool + (size_t)i * n; }
  void g_fft(double2* f, int nf, int sign, cudaStream_t s, int cond) {
    gen_pass(nx, 0, f, nf, nx, ny, tb.twx, sign, s, ctl, cond);
    gen_pass(ny, 1, f, nf, nx, ny, tb.twy, sign, s, ctl, cond);
    gcount += 2;
  }
  void g_sym(double2* f, int nf, cudaStream_t s, int cond) {
    hw2d::k2g_sym<<<hw2d::kGenBlocks, hw2d::kGenThreads, 0, s>>>(f, nf, nx, ny, ctl, cond);
    ++gcount;
  }
  template <class Op>
  void g_map(const Op& op, cudaStream_t s, int cond) {
    hw2d::k2g_map<Op><<<hw2d::kGenBlocks, hw2d::kGenThreads, 0, s>>>(op, n, nx, ctl, cond);
    ++gcount;
  }
  // HSSgen_2depth / HSSgen_3depth (2d/fun_odesolver.c:500-697): res from phi (the
  // unnormalised physical field, real part used) and its spectrum phihat, with the
  // spectral tables O of the reference depths (min, [mid,] plus)
  // With K reference depths (tb.nk > 0) the same sum runs over the K depths' tables
  // (O = the C^2 or the Omega^2 rows of ck / ok, as omega selects), in the same order.
  int hss_base = gHSS;      // first pool slot of the operator's 3K scratch fields
  void g_hss(const double2* phi, const double2* phihat, const double* omin, const double* omid, const double* oplus,
             double2* res, cudaStream_t s, int cond, bool omega = false) {
    const int K = tb.nk ? tb.nk : (tb.gmid ? 3 : 2);
    const double* O[hw2d::kMaxRef2];
    const double* Gm[hw2d::kMaxRef2];
    if (tb.nk) {
      for (int d = 0; d < K; ++d) {
        O[d] = (omega ? tb.ok : tb.ck) + (size_t)d * n;
        Gm[d] = tb.gk + (size_t)d * n;
      }
    } else {
      O[0] = omin;
      O[1] = tb.gmid ? omid : oplus;
      O[2] = oplus;
      Gm[0] = tb.gmin;
      Gm[1] = tb.gmid ? tb.gmid : tb.gplus;
      Gm[2] = tb.gplus;
    }
    const double N = double(nx) * double(ny);
    double2* L0 = G(hss_base);
    double2* g = G(hss_base + K);
    double2* gl = G(hss_base + 2 * K);
    for (int d = 0; d < K; ++d) g_map(hw2d::OpScaleTable{L0 + d * n, phihat, O[d]}, s, cond);
    g_sym(L0, K, s, cond);
    g_fft(L0, K, +1, s, cond);
    for (int d = 0; d < K; ++d) {
      g_map(hw2d::OpGam{g + d * n, phi, Gm[d], N}, s, cond);
      g_map(hw2d::OpGam{gl + d * n, L0 + d * n, Gm[d], N}, s, cond);
    }
    g_fft(g, 2 * K, -1, s, cond);
    hw2d::OpHssSum sum{};
    sum.res = res;
    for (int d = 0; d < K; ++d) {
      sum.g[d] = g + (size_t)d * n;
      sum.gl[d] = gl + (size_t)d * n;
      sum.o[d] = O[d];
    }
    sum.K = K;
    g_map(sum, s, cond);
  }
  // fun_adjust (2d/fun_odesolver.c:810-884) of nf consecutive fields A into AChi:
  // S(A) in place, AChi = F(ChiAdj F^-1(S(A)) / N)
  void g_adjust(double2* A, double2* AChi, int nf, cudaStream_t s, int cond) {
    const double N = double(nx) * double(ny);
    g_sym(A, nf, s, cond);
    for (int f = 0; f < nf; ++f) g_map(hw2d::OpCopy{AChi + f * n, A + f * n}, s, cond);
    g_fft(AChi, nf, +1, s, cond);
    for (int f = 0; f < nf; ++f) g_map(hw2d::OpChi{AChi + f * n, tb.chi, N}, s, cond);
    g_fft(AChi, nf, -1, s, cond);
  }
  // one RHS of rhs_AB1/AB2/AB3_2DB_uv from the stage input w.z into out
  void gen_rhs(int mode, int cond, cudaStream_t s, double2* out) {
    gcount = 0;
    k2g_count<<<1, 1, 0, s>>>(ctl, cond);
    ++gcount;
    const double N = double(nx) * double(ny), f2 = N * N, f3 = N * N * N, g = hw2d::kGrav;
    const int model = tb.model;
    // AB1: symmetrised spectra, physical fields, HSS of u^ and v^ with Csqr
    for (int f = 0; f < 3; ++f) g_map(hw2d::OpCopy{G(gEH + f), w.z + f * n}, s, cond);
    g_sym(G(gEH), 3, s, cond);
    for (int f = 0; f < 3; ++f) g_map(hw2d::OpCopy{G(gP + f), G(gEH + f)}, s, cond);
    g_fft(G(gP), 3, +1, s, cond);
    g_hss(G(gP + 1), G(gEH + 1), tb.cmin, tb.cmid, tb.cplus, G(gCU), s, cond);
    g_hss(G(gP + 2), G(gEH + 2), tb.cmin, tb.cmid, tb.cplus, G(gCV), s, cond);
    // the damping spectra and the source spectrum go where the breaking kernels read
    // them when they rewrite dt eta^ (w.D, w.src)
    g_map(hw2d::OpDampH1{w.D, w.D + n, w.D + 2 * n, G(gH1), G(gH1 + 1), G(gP), G(gP + 1), G(gP + 2), G(gCU),
                         G(gCV), tb.damp, tb.kx, tb.ky, N, g},
          s, cond);
    g_fft(w.D, 3, -1, s, cond);
    const double2* src = nullptr;
    if (tb.has_src) {
      hw2d::k2g_signal<<<(ny + 127) / 128, 128, 0, s>>>(tb, w, ctl, mode, cond);
      ++gcount;
      g_map(hw2d::OpSource{w.src, tb.gx, tb.sx, w.insig, w.insigs, tb.fac_src}, s, cond);
      gen_pass(ny, 1, w.src, 1, nx, ny, tb.twy, -1, s, ctl, cond);   // its row transform is a set-up table
      ++gcount;
      src = w.src;
    }
    hw2d::OpAssemble as{};
    as.out = out;
    as.rk = rk;
    as.ctl = ctl;
    as.mode = mode;
    as.dph = w.dph;
    as.z = w.z;
    as.src = src;
    as.h1u = G(gH1);
    as.h1v = G(gH1 + 1);
    as.de = w.D;
    as.du = w.D + n;
    as.dv = w.D + 2 * n;
    as.aal = tb.aal;
    as.kx = tb.kx;
    as.ky = tb.ky;
    as.g = g;
    as.model = model;
    as.n = n;
    if (model >= 2) {
      // AB2: M0u, M0v, L phi in physical space; the H2 products
      g_map(hw2d::OpM0{G(gM), G(gM + 1), G(gM + 2), G(gH1), G(gH1 + 1)}, s, cond);
      g_sym(G(gM), 3, s, cond);
      g_fft(G(gM), 3, +1, s, cond);
      g_map(hw2d::OpH2Products{G(gEM0U), G(gEU), G(gEM0V), G(gEV), G(gDH2), G(gEM0UH), G(gEM0VH), w.phys, G(gP),
                               G(gP + 1), G(gP + 2), G(gM), G(gM + 1), G(gM + 2), tb.wallchar, N, f2, n},
            s, cond);
      g_fft(G(gEU), 1, -1, s, cond);
      g_fft(G(gEV), 4, -1, s, cond);   // eta v, deletaH2, (eta M0u)^, (eta M0v)^
      g_map(hw2d::OpScaleRe{G(gEM0U), N}, s, cond);
      g_map(hw2d::OpScaleRe{G(gEM0V), N}, s, cond);
      g_hss(G(gEM0U), G(gEM0UH), tb.omin, tb.omid, tb.oplus, G(gLU), s, cond, true);
      g_hss(G(gEM0V), G(gEM0VH), tb.omin, tb.omid, tb.oplus, G(gLV), s, cond, true);
      // adjust inputs: ikx, iky, delu, delv
      g_map(hw2d::OpDelH2{G(gADJIN), G(gADJIN + 1), G(gADJIN + 2), G(gADJIN + 3), G(gDH2), G(gEU), G(gEV), G(gLU),
                          G(gLV), tb.kx, tb.ky, g},
            s, cond);
      g_adjust(G(gADJIN), G(gADJ), 4, s, cond);
      as.ikx = G(gADJ);
      as.iky = G(gADJ + 1);
      as.au = G(gADJ + 2);
      as.av = G(gADJ + 3);
    }
    if (model == 3) {
      // the cubic terms (fun_termshat_AB3_2DB_uv), L applied as HSS(.; Om2dSq) / g
      g_map(hw2d::OpH3Pre{G(gLMU), G(gLMV), G(gLELP), G(gDIVG), G(gE2U), G(gE2V), G(gDXU), G(gDYV), G(gLU),
                          G(gLV), w.z, G(gP), G(gM), G(gM + 1), tb.kx, tb.ky, tb.wallchar, g, f3, n},
            s, cond);
      g_sym(G(gLMU), 6, s, cond);           // LMu, LMv, divgradphi, LetaLphi, dxu, dyv
      g_fft(G(gLMU), 6, +1, s, cond);
      g_fft(G(gE2U), 2, -1, s, cond);
      hw2d::OpH3Products pr{};
      for (int k = 0; k < 4; ++k) {
        pr.p[k] = G(gPK + k);
        pr.ph[k] = G(gPH + k);
      }
      pr.dh3 = G(gDH3);
      pr.eta = G(gP);
      pr.lmu = G(gLMU);
      pr.lmv = G(gLMV);
      pr.dxu = G(gDXU);
      pr.dyv = G(gDYV);
      pr.lphi = G(gM + 2);
      pr.divg = G(gDIVG);
      pr.lelp = G(gLELP);
      pr.wall = tb.wallchar;
      pr.N = N;
      pr.f3 = f3;
      g_map(pr, s, cond);
      g_fft(G(gPH), 5, -1, s, cond);        // the four products' spectra and deletaH3^
      for (int k = 0; k < 4; ++k) g_map(hw2d::OpScaleRe{G(gPK + k), N}, s, cond);
      for (int k = 0; k < 4; ++k)
        g_hss(G(gPK + k), G(gPH + k), tb.omin, tb.omid, tb.oplus, G(gLP + k), s, cond, true);
      g_map(hw2d::OpDelH3{G(gADJ3IN), G(gADJ3IN + 1), G(gADJ3IN + 2), G(gADJ3IN + 3), G(gDH3), G(gLP), G(gLP + 1),
                          G(gLP + 2), G(gLP + 3), G(gE2U), G(gE2V), tb.kx, tb.ky, g},
            s, cond);
      g_adjust(G(gADJ3IN), G(gADJ3), 4, s, cond);
      as.ikx3 = G(gADJ3);
      as.iky3 = G(gADJ3 + 1);
      as.au3 = G(gADJ3 + 2);
      as.av3 = G(gADJ3 + 3);
    }
    g_map(as, s, cond);
    per_rhs = gcount;
  }

  void rhs_launch(int mode, int cond, cudaStream_t s, double2* out) {
    const int rows = ny / 2, cols = nx / 2;
    if (mode != 0) hw2d::k2_stage<<<hw2d::kCombBlocks, 256, 0, s>>>(rk, w, ctl, mode, cond, 3 * n);
    if (gen) {
      gen_rhs(mode, cond, s, out);
      per_rhs += 1;
      if (brk.on) brk_launch(mode, cond, s, out);
      return;
    }
    if (tb.var) {
      row_dispatch(nx, 10, rows, s, tb, w, rk, ctl, ctl, mode, cond, nullptr);
      col_dispatch(ny, 11, cols, s, tb, w, ctl, cond);
      row_dispatch(nx, 12, rows, s, tb, w, rk, ctl, ctl, mode, cond, nullptr);
      col_dispatch(ny, 13, cols, s, tb, w, ctl, cond);
      row_dispatch(nx, 14, rows, s, tb, w, rk, ctl, ctl, mode, cond, nullptr);
      col_dispatch(ny, 15, cols, s, tb, w, ctl, cond);
      row_dispatch(nx, 16, rows, s, tb, w, rk, ctl, ctl, mode, cond, nullptr);
      if (!tb.chi_one || tb.has_src) col_dispatch(ny, 3, cols, s, tb, w, ctl, cond);
      row_dispatch(nx, 4, rows, s, tb, w, rk, ctl, ctl, mode, cond, out);
      per_rhs = ((!tb.chi_one || tb.has_src) ? 9 : 8) + 1;
      if (brk.on) brk_launch(mode, cond, s, out);
      return;
    }
    if (tb.wallchar) {
      const int base = tb.refl_one ? 3 : 0;
      wall_pass(nx, base + 0, rows, s, tb, w, ctl, cond);
      wall_pass(ny, base + 1, cols, s, tb, w, ctl, cond);
      wall_pass(nx, base + 2, rows, s, tb, w, ctl, cond);
    }
    row_dispatch(nx, 0, rows, s, tb, w, rk, ctl, ctl, mode, cond, nullptr);
    if (tb.model == 3) {   // HS3: B3, C3, H3, I3 in place of B, C
      col_dispatch(ny, 21, cols, s, tb, w, ctl, cond);
      row_dispatch(nx, 20, rows, s, tb, w, rk, ctl, ctl, mode, cond, nullptr);
      col_dispatch(ny, 23, cols, s, tb, w, ctl, cond);
      row_dispatch(nx, 22, rows, s, tb, w, rk, ctl, ctl, mode, cond, nullptr);
    } else {
      col_dispatch(ny, 1, cols, s, tb, w, ctl, cond);
      row_dispatch(nx, 2, rows, s, tb, w, rk, ctl, ctl, mode, cond, nullptr);
    }
    if (!tb.chi_one || tb.has_src) col_dispatch(ny, 3, cols, s, tb, w, ctl, cond);
    row_dispatch(nx, 4, rows, s, tb, w, rk, ctl, ctl, mode, cond, out);
    per_rhs = ((!tb.chi_one || tb.has_src) ? 5 : 4) + 1 + (tb.wallchar ? 3 : 0) + (tb.model == 3 ? 2 : 0);
    if (brk.on) brk_launch(mode, cond, s, out);
  }
  // the breaking kernels after the assembly pass (both bottoms)
  void brk_launch(int mode, int cond, cudaStream_t s, double2* out) {
    const int rows = ny / 2, cols = nx / 2;
    const int gb = (int)std::min<size_t>((n + 255) / 256, 4 * 148);
    brk_row(nx, 0, rows, s, tb, w, brk, rk, ctl, mode, cond, out);
    brk_col(ny, 0, cols, s, tb, w, brk, ctl, mode, cond);
    hw2d::k2b_peaks<<<gb, 256, 0, s>>>(tb, w, brk, ctl, mode, cond);
    hw2d::k2b_sort<<<1, hw2d::kBrkSortThreads, hw2d::kBrkPeakCap * sizeof(int), s>>>(brk, ctl, mode, cond);
    hw2d::k2b_machine<<<1, 32, 0, s>>>(tb, w, brk, ctl, mode, cond);
    hw2d::k2b_flux<<<gb, 256, 0, s>>>(tb, w, brk, ctl, mode, cond);
    brk_col(ny, 1, cols, s, tb, w, brk, ctl, mode, cond);
    brk_row(nx, 1, rows, s, tb, w, brk, rk, ctl, mode, cond, out);
    per_rhs += 8;
  }
  long long kernels_per_attempt() const { return 7LL * per_rhs + 3; }
  void attempt_launch(cudaStream_t s) {
    rhs_launch(1, hw2d::kIfK1, s, nullptr);
    for (int st = 2; st <= 6; ++st) rhs_launch(st, hw2d::kIfStage, s, nullptr);
    if (brk.on) {
      // gsl_odeiv2's order: dydt_out of the candidate state before the step control
      hw2d::k2_combine<<<hw2d::kCombBlocks, hw2d::kCombThreads, 0, s>>>(rk, w, ctl, 3 * n);
      rhs_launch(8, hw2d::kIfStage, s, nullptr);
      hw2d::k2_control<<<1, 256, 0, s>>>(ctl, w, hw2d::kCombBlocks);
      hw2d::k2_finalize<<<1, 1, 0, s>>>(ctl);
      return;
    }
    hw2d::k2_combine<<<hw2d::kCombBlocks, hw2d::kCombThreads, 0, s>>>(rk, w, ctl, 3 * n);
    hw2d::k2_control<<<1, 256, 0, s>>>(ctl, w, hw2d::kCombBlocks);
    rhs_launch(7, hw2d::kIfKout, s, nullptr);
    hw2d::k2_finalize<<<1, 1, 0, s>>>(ctl);
  }
  bool build_graph() {
    if (attempt) return true;
    if (cudaStreamCreateWithFlags(&graph_stream, cudaStreamNonBlocking) != cudaSuccess) {
      err = "stream create failed";
      return false;
    }
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(graph_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      err = "graph capture failed to start";
      return false;
    }
    attempt_launch(graph_stream);
    if (cudaStreamEndCapture(graph_stream, &g) != cudaSuccess || !g) {
      err = "graph capture failed";
      cudaGetLastError();
      return false;
    }
    const cudaError_t e = cudaGraphInstantiate(&attempt, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      err = std::string("graph instantiate: ") + cudaGetErrorString(e);
      return false;
    }
    return true;
  }
  bool read_ctl() {
    if (cudaMemcpyAsync(hctl, ctl, sizeof(Ctl2), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
      return check("control read-back");
    return true;
  }
  // evolve on the device until t1 (or one accepted step when one_step)
  int run(double t1, bool one_step) {
    if (!build_graph()) return 1;
    hw2d::k2_begin<<<1, 1, 0, stream>>>(ctl, t1);
    launches += 1;
    if (!check("begin")) return 1;
    if (!read_ctl()) return 1;
    const long long acc0 = hctl->acc;
    int batch = one_step ? 1 : 2;
    long long launched = 0;
    for (;;) {
      if (hctl->done) break;
      if (launched > kMaxAttemptsPerRun) {
        err = "time integration stopped: attempt budget of one run exceeded (step size collapsed)";
        return 1;
      }
      launched += batch;
      for (int b = 0; b < batch; ++b)
        if (const cudaError_t e = cudaGraphLaunch(attempt, stream); e != cudaSuccess) return fail("graph launch", e);
      launches += batch * kernels_per_attempt();
      if (!read_ctl()) return 1;
      if (hctl->status != hw2d::kOk) break;
      if (one_step && hctl->acc > acc0) {
        // stop here: the next call recomputes its dydt_in like GSL's evolve_apply
        break;
      }
      if (!one_step && batch < 16) batch *= 2;
    }
    if (hctl->status == hw2d::kNonFinite) { err = "non-finite state (the step size collapsed)"; return 1; }
    if (hctl->status == hw2d::kStepFailed) { err = "time integration failed (too many rejected steps)"; return 1; }
    if (hctl->status == hw2d::kBreakCapacity) { err = "breaking: a capacity (peaks, crests or nodes) was exceeded"; return 1; }
    return 0;
  }
  bool ensure_out(int ngauge) {
    if (!oP) {
      oP = dalloc<double2>(2 * n);
      ophys = dalloc<double>(3 * n);
      of32 = dalloc<float>(3 * n);
      if (!oP || !ophys || !of32 || cudaMallocHost(&hf32, 3 * n * sizeof(float)) != cudaSuccess) {
        err = "output buffers: out of memory";
        return false;
      }
    }
    if (ngauge > ogcap) {
      if (hgval) cudaFreeHost(hgval);
      hgval = nullptr;
      ogpt = dalloc<int>(ngauge);
      ogval = dalloc<double>(3 * (size_t)ngauge);
      if (!ogpt || !ogval || cudaMallocHost(&hgval, 3 * (size_t)ngauge * sizeof(double)) != cudaSuccess) {
        err = "gauge buffers: out of memory";
        return false;
      }
      ogcap = ngauge;
    }
    return true;
  }
  // eta, u, v of the current state (hctl must be current) into ophys (and of32)
  void fields_launch(cudaStream_t s, bool keep_f32) {
    out_pass(nx, 0, ny / 2, s, tb, rk.y[hctl->cur], oP, ophys, nullptr);
    out_pass(ny, 1, nx / 2, s, tb, rk.y[hctl->cur], oP, ophys, keep_f32 ? of32 : nullptr);
    launches += 2;
  }
  ~hw2d_ctx() {
    if (hf32) cudaFreeHost(hf32);
    if (hgval) cudaFreeHost(hgval);
    if (attempt) cudaGraphExecDestroy(attempt);
    if (graph_stream) cudaStreamDestroy(graph_stream);
    for (void* p : allocs) cudaFree(p);
    if (hctl) cudaFreeHost(hctl);
    if (own_stream) cudaStreamDestroy(own_stream);
  }
};

extern "C" {

hw2d_ctx* hw2d_create(const hw2d_tables* t, const hw_opts* o) {
  if (!t || !t->kx || !t->ky || !t->c2d || !t->l2d || !t->aal || !t->charac || !t->chiadj) {
    g_err2d = "hw2d_create: missing table";
    return nullptr;
  }
  if (!pow2_in_range(t->nx) || !pow2_in_range(t->ny)) {
    g_err2d = "hw2d_create: nx and ny must be powers of two in [64, 1024]";
    return nullptr;
  }
  if (t->model < 1 || t->model > 3) {
    g_err2d = "hw2d_create: model must be 1 (HS1), 2 (HS2) or 3 (HS3)";
    return nullptr;
  }
  const bool var_tables = t->gam_min && t->gam_plus && t->csq_min && t->csq_plus && t->om2_min && t->om2_plus;
  const bool mid_tables = t->gam_mid && t->csq_mid && t->om2_mid;
  if ((t->gam_mid || t->csq_mid || t->om2_mid) && !(mid_tables && var_tables)) {
    g_err2d = "hw2d_create: three reference depths need all of gam, csq, om2 for the min, mid and plus depths";
    return nullptr;
  }
  const bool kref = t->nrefk != 0;
  if (kref && (t->nrefk < 2 || t->nrefk > hw2d::kMaxRef2 || !t->gam_k || !t->csq_k || !t->om2_k)) {
    g_err2d = "hw2d_create: K reference depths need 2 <= nrefk <= 16 and gam_k, csq_k, om2_k";
    return nullptr;
  }
  if (kref && (var_tables || t->gam_mid)) {
    g_err2d = "hw2d_create: give either the min/plus(/mid) tables or the K-reference tables, not both";
    return nullptr;
  }
  if (t->model == 1 && t->breaking) {
    // rhs_AB1_2DF_uv / rhs_AB1_2DB_uv never call breaking_process: under HS1 a breaking
    // deck is the plain HS1 run, so the tables must say breaking = 0
    g_err2d = "hw2d_create: HS1 runs no breaking process (rhs_AB1_2DF_uv, rhs_AB1_2DB_uv); pass breaking = 0";
    return nullptr;
  }
  (void)var_tables;
  if (t->propagation < 0 || t->propagation > 2) {
    g_err2d = "hw2d_create: propagation must be 0 (Uni+), 1 (Uni-) or 2 (Bi)";
    return nullptr;
  }
  auto* c = new hw2d_ctx();
  c->device = o ? o->device : 0;
  if (cudaSetDevice(c->device) != cudaSuccess) {
    g_err2d = "hw2d_create: cannot select the CUDA device";
    delete c;
    return nullptr;
  }
  set_all_attrs();
  const int nx = t->nx, ny = t->ny;
  const size_t n = (size_t)nx * ny;
  c->nx = nx; c->ny = ny; c->n = n;
  const bool has_src = t->nt >= 2 && t->sig && t->tsig && t->newgam;

  // host tables (reference formulas: C2d^2/grav as pow(C2d, 2)/grav, 7*Cpeak*charac)
  std::vector<double> c2g(n), damp(n);
  bool chi_one = true;
  for (size_t q = 0; q < n; ++q) {
    c2g[q] = std::pow(t->c2d[q], 2) / hw2d::kGrav;
    damp[q] = 7 * t->cpeak * t->charac[q];
    if (t->chiadj[q] != 1.0) chi_one = false;
  }
  Tab2& tb = c->tb;
  tb.nx = nx; tb.ny = ny; tb.n = (int)n; tb.model = t->model; tb.chi_one = chi_one ? 1 : 0;
  tb.has_src = has_src ? 1 : 0;
  tb.fac_src = t->propagation == 2 ? 2.0 : 1.0;
  tb.kx = c->upload(std::vector<double>(t->kx, t->kx + nx));
  tb.ky = c->upload(std::vector<double>(t->ky, t->ky + ny));
  tb.c2g = c->upload(c2g);
  tb.l2d = c->upload(std::vector<double>(t->l2d, t->l2d + n));
  tb.aal = c->upload(std::vector<double>(t->aal, t->aal + n));
  tb.damp = c->upload(damp);
  tb.chi = c->upload(std::vector<double>(t->chiadj, t->chiadj + n));
  tb.twx = c->upload(twiddles(nx));
  tb.twy = c->upload(twiddles(ny));
  if (has_src) {
    // row transforms of the area kernels (the source's row pass is done once here)
    const double sk = t->propagation == 0 ? -1.0 : (t->propagation == 1 ? 1.0 : 0.0);
    std::vector<double2> gx(n), sx(n);
    std::vector<double> re(nx), im(nx);
    for (int i = 0; i < ny; ++i) {
      for (int j = 0; j < nx; ++j) { re[j] = t->newgam[(size_t)i * nx + j]; im[j] = 0.0; }
      hw::host_dft(re, im, -1);
      for (int j = 0; j < nx; ++j) gx[(size_t)i * nx + j] = make_double2(re[j], im[j]);
      for (int j = 0; j < nx; ++j) {
        re[j] = t->skewgam ? sk * t->skewgam[(size_t)i * nx + j] : 0.0;
        im[j] = 0.0;
      }
      hw::host_dft(re, im, -1);
      for (int j = 0; j < nx; ++j) sx[(size_t)i * nx + j] = make_double2(re[j], im[j]);
    }
    tb.gx = c->upload(gx);
    tb.sx = c->upload(sx);
    const int nt = t->nt;
    tb.nt = nt;
    std::vector<double> ts(t->tsig, t->tsig + nt);
    std::vector<double> sig((size_t)ny * nt), sigc((size_t)ny * nt), sigs((size_t)ny * nt, 0.0),
        sigsc((size_t)ny * nt, 0.0);
    for (int i = 0; i < ny; ++i) {
      std::vector<double> a(t->sig + (size_t)i * nt, t->sig + (size_t)(i + 1) * nt);
      std::vector<double> ca = hw::natural_spline_c(ts, a);
      std::copy(a.begin(), a.end(), sig.begin() + (size_t)i * nt);
      std::copy(ca.begin(), ca.end(), sigc.begin() + (size_t)i * nt);
      if (t->sigskew) {
        std::vector<double> b(t->sigskew + (size_t)i * nt, t->sigskew + (size_t)(i + 1) * nt);
        std::vector<double> cb = hw::natural_spline_c(ts, b);
        std::copy(b.begin(), b.end(), sigs.begin() + (size_t)i * nt);
        std::copy(cb.begin(), cb.end(), sigsc.begin() + (size_t)i * nt);
      }
    }
    tb.tsig = c->upload(ts);
    tb.sig = c->upload(sig);
    tb.sigc = c->upload(sigc);
    tb.sigs = c->upload(sigs);
    tb.sigsc = c->upload(sigsc);
    c->h_first = (ts[nt - 1] - ts[0]) / (nt - 1) / 5.0;   // h = dt/5 (2d/fun_odesolver.c:2580)
  } else {
    c->h_first = 1e-3;
  }
  if (o && o->h0 > 0) c->h_first = o->h0;
  const bool var = kref || (t->gam_min && t->gam_plus && t->csq_min && t->csq_plus && t->om2_min && t->om2_plus);
  tb.var = var ? 1 : 0;
  if (kref) {   // K reference depths: the general path with the K-depth sum
    const size_t kn = (size_t)t->nrefk * n;
    tb.nk = t->nrefk;
    tb.gk = c->upload(std::vector<double>(t->gam_k, t->gam_k + kn));
    tb.ck = c->upload(std::vector<double>(t->csq_k, t->csq_k + kn));
    tb.ok = c->upload(std::vector<double>(t->om2_k, t->om2_k + kn));
    c->gen = 1;
  } else if (var) {
    tb.gmin = c->upload(std::vector<double>(t->gam_min, t->gam_min + n));
    tb.gplus = c->upload(std::vector<double>(t->gam_plus, t->gam_plus + n));
    tb.cmin = c->upload(std::vector<double>(t->csq_min, t->csq_min + n));
    tb.cplus = c->upload(std::vector<double>(t->csq_plus, t->csq_plus + n));
    tb.omin = c->upload(std::vector<double>(t->om2_min, t->om2_min + n));
    tb.oplus = c->upload(std::vector<double>(t->om2_plus, t->om2_plus + n));
    if (t->gam_mid) {   // three reference depths: the general path
      tb.gmid = c->upload(std::vector<double>(t->gam_mid, t->gam_mid + n));
      tb.cmid = c->upload(std::vector<double>(t->csq_mid, t->csq_mid + n));
      tb.omid = c->upload(std::vector<double>(t->om2_mid, t->om2_mid + n));
    }
    // the fused passes serve two reference depths under HS1 / HS2; three depths and
    // HS3 on this bottom take the general path
    c->gen = (t->gam_mid || t->model == 3) ? 1 : 0;
  }
  if (t->wallchar) {
    tb.wallchar = c->upload(std::vector<double>(t->wallchar, t->wallchar + n));
    if (!var) tb.c2d = c->upload(std::vector<double>(t->c2d, t->c2d + n));
    if (!var && t->refl_coef == 1) {
      // fun_delphiH1hat's refl_coef == 1 branch needs fun_gradient(wallchar)
      // (2d/functions.c:392-460, called at :741): periodic forward and backward
      // differences, the forward ones clipped to <= 0, the backward ones to >= 0
      if (!(t->dx > 0) || !(t->dy > 0)) {
        g_err2d = "hw2d_create: walls with refl_coef 1 need dx and dy";
        delete c;
        return nullptr;
      }
      std::vector<double> gx(n), gy(n);
      const double* f = t->wallchar;
      for (int i = 0; i < ny; ++i)
        for (int j = 0; j < nx; ++j) {
          const size_t q = (size_t)i * nx + j;
          double Fx = (j < nx - 1) ? (f[q + 1] - f[q]) / t->dx : (f[(size_t)i * nx] - f[q]) / t->dx;
          double Fy = (i < ny - 1) ? (f[q + nx] - f[q]) / t->dy : (f[j] - f[q]) / t->dy;
          double Bx = (j > 0) ? (f[q] - f[q - 1]) / t->dx : (f[q] - f[(size_t)i * nx + nx - 1]) / t->dx;
          double By = (i > 0) ? (f[q] - f[q - nx]) / t->dy : (f[q] - f[(size_t)(ny - 1) * nx + j]) / t->dy;
          if (Fx > 0) Fx = 0;
          if (Fy > 0) Fy = 0;
          if (Bx < 0) Bx = 0;
          if (By < 0) By = 0;
          gx[q] = Fx + Bx;
          gy[q] = Fy + By;
        }
      tb.refl_one = 1;
      tb.gwx = c->upload(gx);
      tb.gwy = c->upload(gy);
    }
  }

  hw2d::Brk2& bk = c->brk;
  if (t->breaking) {
    if (!t->bathy || !t->brchar || !t->x || !t->y || !(t->dx > 0) || !(t->dy > 0) || !(t->dt_out > 0) ||
        !(t->rsearch > 0)) {
      g_err2d = "hw2d_create: breaking tables missing or invalid";
      delete c;
      return nullptr;
    }
    bk.on = 1;
    bk.bathy = c->upload(std::vector<double>(t->bathy, t->bathy + n));
    bk.pbchar = c->upload(std::vector<double>(t->brchar, t->brchar + n));
    bk.x = c->upload(std::vector<double>(t->x, t->x + nx));
    bk.y = c->upload(std::vector<double>(t->y, t->y + ny));
    bk.dx = t->dx; bk.dy = t->dy; bk.thr = t->max_eta_init; bk.tstar = t->tstar; bk.rsearch = t->rsearch;
    bk.kbc = t->kbc; bk.tc = t->tc; bk.delb = t->delb; bk.cur_u = t->cur_u; bk.t0 = t->t0; bk.dt_out = t->dt_out;
    bk.B = c->dalloc<double>(n);
    bk.flux = c->dalloc<double>(n);
    bk.P = c->dalloc<double2>(n);
    bk.dh = c->dalloc<double2>(n);
    bk.sb = c->dalloc<double2>(2 * n);
    bk.peaks = c->dalloc<int>(hw2d::kBrkPeakCap);
    bk.CB = c->dalloc<hw2d::Crest2>(hw2d::kBrkCrestCap);
    bk.CBNew = c->dalloc<hw2d::Crest2>(hw2d::kBrkCrestCap);
    bk.CBPrev = c->dalloc<hw2d::Crest2>(hw2d::kBrkCrestCap);
    bk.cap_nodes = (int)std::max<size_t>(4096, n / 4);
    bk.bn[0] = c->dalloc<int2>(bk.cap_nodes);
    bk.bn[1] = c->dalloc<int2>(bk.cap_nodes);
    bk.bnp = c->dalloc<int2>(bk.cap_nodes);
    bk.cap_rec = 1 << 18;
    bk.cap_log = (long long)std::max<size_t>(1 << 16, 4 * n);
    bk.log_t = c->dalloc<double>(bk.cap_rec);
    bk.log_cnt = c->dalloc<int>(bk.cap_rec);
    bk.log_nodes = c->dalloc<int2>((size_t)bk.cap_log);
    bk.st = c->dalloc<hw2d::BrkSt>(1);
    const bool bok = bk.bathy && bk.pbchar && bk.x && bk.y && bk.B && bk.flux && bk.P && bk.dh && bk.sb && bk.peaks &&
                     bk.CB && bk.CBNew && bk.CBPrev && bk.bn[0] && bk.bn[1] && bk.bnp && bk.log_t && bk.log_cnt &&
                     bk.log_nodes && bk.st;
    if (!bok) {
      g_err2d = "hw2d_create: device allocation failed (breaking)";
      delete c;
      return nullptr;
    }
    hw2d::BrkSt s0{};
    s0.sb_zero = 1;   // Sb_xhat, Sb_yhat start at zero
    cudaMemcpy(bk.st, &s0, sizeof s0, cudaMemcpyHostToDevice);
    cudaMemset(bk.B, 0, n * sizeof(double));
    cudaMemset(bk.sb, 0, 2 * n * sizeof(double2));
  }

  Work2& w = c->w;
  w.dph = bk.on ? c->dalloc<double2>(n) : nullptr;
  w.z = c->dalloc<double2>(3 * n);
  w.R = c->dalloc<double2>(4 * n);
  w.Q = c->dalloc<double2>((var ? 6 : (t->model == 3 ? 5 : 4)) * n);
  if (t->model == 3) {
    w.p3 = c->dalloc<double>(2 * n);
    w.T3 = c->dalloc<double2>(6 * n);
  }
  if (!var && bk.on) w.phys = c->dalloc<double>(3 * n);   // eta, u, v for the breaking kernels
  if (!var && t->wallchar) {   // the flat bottom's wall round trip
    w.WP = c->dalloc<double2>((tb.refl_one ? 2 : 1) * n);
    w.H1 = c->dalloc<double2>(n);
  }
  if (var) {
    w.phys = c->dalloc<double>(3 * n);
    w.pe = c->dalloc<double>(2 * n);
    w.H1 = c->dalloc<double2>(2 * n);
    w.EU = c->dalloc<double2>(3 * n);
  }
  if (c->gen) {
    int slots = t->model == 3 ? hw2d_ctx::gSlotsHS3 : hw2d_ctx::gSlotsHS2;
    if (kref && t->nrefk > 3) {   // the operator's 3K scratch fields after the model's own
      c->hss_base = slots;
      slots += 3 * t->nrefk;
    }
    c->gpool = c->dalloc<double2>((size_t)slots * n);
  }
  w.D = c->dalloc<double2>(3 * n);
  w.W = chi_one ? nullptr : c->dalloc<double2>(4 * n);
  w.V = c->dalloc<double2>(4 * n);
  w.src = has_src ? c->dalloc<double2>(n) : nullptr;
  w.insig = c->dalloc<double>(ny);
  w.insigs = c->dalloc<double>(ny);
  w.part = c->dalloc<double>(hw2d::kCombBlocks);
  RK2& rk = c->rk;
  for (int i = 0; i < 2; ++i) rk.y[i] = c->dalloc<double2>(3 * n);
  for (int i = 0; i < 2; ++i) rk.kk[i] = c->dalloc<double2>(3 * n);
  for (int i = 0; i < 5; ++i) rk.ks[i] = c->dalloc<double2>(3 * n);
  c->dref = c->dalloc<double>(6 * n);
  c->dout = c->dalloc<double2>(3 * n);
  c->ctl = c->dalloc<Ctl2>(1);
  bool ok = tb.kx && tb.ky && tb.c2g && tb.l2d && tb.aal && tb.damp && tb.chi && tb.twx && tb.twy && w.z && w.R &&
            w.Q && w.D && w.V && w.insig && w.insigs && w.part && c->dref && c->dout && c->ctl &&
            (chi_one || w.W) && (!has_src || (tb.gx && tb.sx && tb.sig && w.src)) && (!bk.on || (w.dph && w.phys)) &&
            (var || !t->wallchar || (w.WP && w.H1 && tb.c2d && (!tb.refl_one || (tb.gwx && tb.gwy)))) &&
            (!var || ((kref ? (tb.gk && tb.ck && tb.ok) : (tb.gmin && tb.gplus && tb.cmin && tb.cplus && tb.omin &&
                                                             tb.oplus)) &&
                      w.phys && w.pe && w.H1 && w.EU)) &&
            (!t->wallchar || tb.wallchar) && (t->model != 3 || (w.p3 && w.T3)) &&
            (!c->gen || (c->gpool && (!t->gam_mid || (tb.gmid && tb.cmid && tb.omid))));
  for (int i = 0; i < 2; ++i) ok = ok && rk.y[i] && rk.kk[i];
  for (int i = 0; i < 5; ++i) ok = ok && rk.ks[i];
  if (!ok || cudaMallocHost(&c->hctl, sizeof(Ctl2)) != cudaSuccess) {
    g_err2d = "hw2d_create: device allocation failed";
    delete c;
    return nullptr;
  }
  cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  c->stream = c->own_stream;
  Ctl2 h{};
  h.eps_abs = (o && o->eps_abs > 0) ? o->eps_abs : 1e-3;
  h.eps_rel = (o && o->eps_rel > 0) ? o->eps_rel : 1e-2;
  h.h = c->h_first;
  h.need_k1 = 1;
  h.done = 1;
  h.brk = bk.on;
  cudaMemcpy(c->ctl, &h, sizeof h, cudaMemcpyHostToDevice);
  cudaMemset(rk.y[0], 0, 3 * n * sizeof(double2));
  if (!c->check("hw2d_create")) {
    g_err2d = c->err;
    delete c;
    return nullptr;
  }
  return c;
}

void hw2d_destroy(hw2d_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  delete c;
}

const char* hw2d_last_error(const hw2d_ctx* c) { return c ? c->err.c_str() : g_err2d.c_str(); }
int hw2d_nx(const hw2d_ctx* c) { return c ? c->nx : 0; }
int hw2d_ny(const hw2d_ctx* c) { return c ? c->ny : 0; }

int hw2d_rhs(hw2d_ctx* c, double t, const double* y, double* dydt) {
  if (!c || !y || !dydt) return 1;
  cudaSetDevice(c->device);
  const size_t n = c->n;
  cudaMemcpyAsync(c->dref, y, 6 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream);
  hw2d::k2_to_internal<<<592, 256, 0, c->stream>>>(c->dref, c->w.z, n);
  cudaMemcpyAsync(&c->ctl->t_direct, &t, sizeof(double), cudaMemcpyHostToDevice, c->stream);
  c->rhs_launch(0, hw2d::kAlways, c->stream, c->dout);
  hw2d::k2_to_reference<<<592, 256, 0, c->stream>>>(c->dout, c->dref, n);
  c->launches += c->per_rhs + 2;
  cudaMemcpyAsync(dydt, c->dref, 6 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (const cudaError_t e = cudaStreamSynchronize(c->stream); e != cudaSuccess) return c->fail("hw2d_rhs", e);
  if (!c->check("hw2d_rhs")) return 1;
  if (c->brk.on) {
    hw2d::BrkSt st{};
    if (const cudaError_t e = cudaMemcpy(&st, c->brk.st, sizeof st, cudaMemcpyDeviceToHost); e != cudaSuccess)
      return c->fail("hw2d_rhs", e);
    if (st.err & (hw2d::kBrkErrPeaks | hw2d::kBrkErrCrests | hw2d::kBrkErrNodes)) {
      c->err = "breaking: a capacity (peaks, crests or nodes) was exceeded";
      return 1;
    }
  }
  return 0;
}

int hw2d_gsl_rhs(double t, const double* y, double* dydt, void* params) {
  return hw2d_rhs(static_cast<hw2d_ctx*>(params), t, y, dydt);
}

int hw2d_set_state(hw2d_ctx* c, double t, double h, const double* y) {
  if (!c || !y) return 1;
  cudaSetDevice(c->device);
  if (!c->read_ctl()) return 1;
  Ctl2 s = *c->hctl;
  s.t = t;
  s.h = h > 0 ? h : c->h_first;
  s.cur = 0;
  s.need_k1 = 1;
  s.need_kout = 0;
  s.done = 1;
  s.status = hw2d::kOk;
  *c->hctl = s;
  cudaMemcpyAsync(c->dref, y, 6 * c->n * sizeof(double), cudaMemcpyHostToDevice, c->stream);
  hw2d::k2_to_internal<<<592, 256, 0, c->stream>>>(c->dref, c->rk.y[0], c->n);
  c->launches += 1;
  cudaMemcpyAsync(c->ctl, c->hctl, sizeof(Ctl2), cudaMemcpyHostToDevice, c->stream);
  if (const cudaError_t e = cudaStreamSynchronize(c->stream); e != cudaSuccess) return c->fail("hw2d_set_state", e);
  return c->check("hw2d_set_state") ? 0 : 1;
}

int hw2d_get_state(hw2d_ctx* c, double* t, double* h, double* y) {
  if (!c) return 1;
  cudaSetDevice(c->device);
  if (!c->read_ctl()) return 1;
  if (t) *t = c->hctl->t;
  if (h) *h = c->hctl->h;
  if (y) {
    hw2d::k2_to_reference<<<592, 256, 0, c->stream>>>(c->rk.y[c->hctl->cur], c->dref, c->n);
    c->launches += 1;
    cudaMemcpyAsync(y, c->dref, 6 * c->n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (const cudaError_t e = cudaStreamSynchronize(c->stream); e != cudaSuccess) return c->fail("hw2d_get_state", e);
  }
  return c->check("hw2d_get_state") ? 0 : 1;
}

int hw2d_run_to_time(hw2d_ctx* c, double t1) {
  if (!c) return 1;
  cudaSetDevice(c->device);
  return c->run(t1, false);
}

int hw2d_evolve_apply(hw2d_ctx* c, double* t, double t1, double* h, double* y) {
  if (!c || !t || !h || !y) return 1;
  if (hw2d_set_state(c, *t, *h, y)) return 1;
  // gsl_odeiv2_evolve_apply rejects a step whose direction disagrees with t1 - t
  const double dt = t1 - *t;
  if ((dt < 0.0 && *h > 0.0) || (dt > 0.0 && *h < 0.0)) {
    c->err = "step direction does not match t1 - t";
    return 1;
  }
  if (c->run(t1, true)) return 1;
  return hw2d_get_state(c, t, h, y);
}

int hw2d_stats(const hw2d_ctx* cc, long long* r, long long* a, long long* j) {
  auto* c = const_cast<hw2d_ctx*>(cc);
  if (!c || !c->read_ctl()) return 1;
  if (r) *r = c->hctl->rhs;
  if (a) *a = c->hctl->acc;
  if (j) *j = c->hctl->rej;
  return 0;
}

long long hw2d_launches(const hw2d_ctx* c) { return c ? c->launches : 0; }

int hw2d_breaking_fields(hw2d_ctx* c, double* B, double* sbx, double* sby, int* flagbr, int* ncrest) {
  if (!c || !c->brk.on) return -1;
  cudaSetDevice(c->device);
  if (const cudaError_t e = cudaStreamSynchronize(c->stream); e != cudaSuccess)
    return c->fail("hw2d_breaking_fields", e);
  const size_t n = c->n;
  struct Copy { void* dst; const void* src; size_t bytes; };
  hw2d::BrkSt st{};
  const Copy copies[4] = {{B, c->brk.B, n * sizeof(double)}, {sbx, c->brk.sb, n * sizeof(double2)},
                          {sby, c->brk.sb + n, n * sizeof(double2)}, {&st, c->brk.st, sizeof st}};
  for (const Copy& k : copies)
    if (k.dst)
      if (const cudaError_t e = cudaMemcpy(k.dst, k.src, k.bytes, cudaMemcpyDeviceToHost); e != cudaSuccess)
        return c->fail("hw2d_breaking_fields", e);
  if (flagbr) *flagbr = st.flagbr;
  if (ncrest) *ncrest = st.flagbr == 2 ? st.ncbprev : 0;
  return 0;
}

long long hw2d_breaking_log_nodes(hw2d_ctx* c) {
  if (!c || !c->brk.on) return -1;
  cudaSetDevice(c->device);
  hw2d::BrkSt st{};
  if (cudaStreamSynchronize(c->stream) != cudaSuccess ||
      cudaMemcpy(&st, c->brk.st, sizeof st, cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  return st.nlog;
}

int hw2d_breaking_log(hw2d_ctx* c, double* times, int* counts, int* nodes, int cap_rec, long long cap_nodes) {
  if (!c || !c->brk.on) return -1;
  cudaSetDevice(c->device);
  hw2d::BrkSt st{};
  if (cudaStreamSynchronize(c->stream) != cudaSuccess ||
      cudaMemcpy(&st, c->brk.st, sizeof st, cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  const int nr = std::min(st.nrec, std::max(cap_rec, 0));
  const long long nn = std::min(st.nlog, std::max(cap_nodes, 0LL));
  if (times && nr > 0 && cudaMemcpy(times, c->brk.log_t, nr * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  if (counts && nr > 0 && cudaMemcpy(counts, c->brk.log_cnt, nr * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  if (nodes && nn > 0 && cudaMemcpy(nodes, c->brk.log_nodes, nn * sizeof(int2), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  if (st.err & hw2d::kBrkErrLog) return -2;
  return st.nrec;
}

int hw2d_fields(hw2d_ctx* c, double* eta, double* u, double* v) {
  if (!c) return 1;
  cudaSetDevice(c->device);
  if (!c->ensure_out(0) || !c->read_ctl()) return 1;
  c->fields_launch(c->stream, false);
  if (!c->check("hw2d_fields")) return 1;
  double* dst[3] = {eta, u, v};
  for (int f = 0; f < 3; ++f)
    if (dst[f])
      if (const cudaError_t e = cudaMemcpyAsync(dst[f], c->ophys + f * c->n, c->n * sizeof(double),
                                                cudaMemcpyDeviceToHost, c->stream);
          e != cudaSuccess)
        return c->fail("hw2d_fields", e);
  if (const cudaError_t e = cudaStreamSynchronize(c->stream); e != cudaSuccess) return c->fail("hw2d_fields", e);
  return 0;
}

namespace {

// the file set of ode_solver_uv's output loop; every file is closed on the way out
struct OutFiles {
  FILE* part[3] = {nullptr, nullptr, nullptr};   // Hawassi_eta/u/v_NN.dat
  FILE* gauge[3] = {nullptr, nullptr, nullptr};  // Hawassi_eta/u/v_gauge.dat
  void close_part() {
    for (FILE*& f : part)
      if (f) { fclose(f); f = nullptr; }
  }
  ~OutFiles() {
    close_part();
    for (FILE*& f : gauge)
      if (f) { fclose(f); f = nullptr; }
  }
};

// print_xt (2d/fun_odesolver.c:2532-2563)
bool write_constant(const std::string& path, const hw2d_outputs* o, int nx, int ny, int ntpart) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return false;
  std::vector<double> th(ntpart);
  for (int j = 0; j < ntpart; ++j) th[j] = (0 + j) * o->dt;
  const double NX = nx, NT = ntpart, NY = ny;
  const size_t n = (size_t)nx * ny;
  bool ok = fwrite(&NX, sizeof(double), 1, f) == 1 && fwrite(o->x, sizeof(double), nx, f) == (size_t)nx &&
            fwrite(&NY, sizeof(double), 1, f) == 1 && fwrite(o->y, sizeof(double), ny, f) == (size_t)ny &&
            fwrite(&NT, sizeof(double), 1, f) == 1 &&
            fwrite(th.data(), sizeof(double), ntpart, f) == (size_t)ntpart &&
            fwrite(&o->hs, sizeof(double), 1, f) == 1 && fwrite(&o->kp, sizeof(double), 1, f) == 1 &&
            fwrite(&o->wp, sizeof(double), 1, f) == 1 && fwrite(o->kx, sizeof(double), nx, f) == (size_t)nx &&
            fwrite(o->ky, sizeof(double), ny, f) == (size_t)ny && fwrite(o->bathy, sizeof(double), n, f) == n &&
            fwrite(o->cfsa, sizeof(double), n, f) == n;
  if (ok && o->chiadjphi) ok = fwrite(o->chiadjphi, sizeof(double), n, f) == n;
  return fclose(f) == 0 && ok;
}

}  // namespace

int hw2d_run_outputs(hw2d_ctx* c, const hw2d_outputs* o) {
  if (!c || !o) return -1;
  cudaSetDevice(c->device);
  auto fail = [&](const std::string& m) {
    c->err = m;
    return -1;
  };
  if (!o->outdir || o->nt < 1 || !o->tout) return fail("outputs: outdir, nt and tout are required");
  if (o->npartition < 1 || o->nt / o->npartition < 1) return fail("outputs: npartition must be in [1, nt]");
  if (!o->x || !o->y || !o->kx || !o->ky || !o->bathy || !o->cfsa)
    return fail("outputs: x, y, kx, ky, bathy and cfsa are required (Constant_01.dat)");
  if (o->ngauge < 0 || (o->ngauge > 0 && (!o->xgauge || !o->ygauge || !(o->dx > 0) || !(o->dy > 0))))
    return fail("outputs: gauges need xgauge, ygauge, dx and dy");
  const int nx = c->nx, ny = c->ny, ng = o->ngauge;
  const size_t n = c->n;
  const int ntpart = o->nt / o->npartition;
  // index_gauge (2d/functions.c:774-781): the nearest grid point
  std::vector<int> gx(ng), gy(ng), gpt(ng);
  for (int j = 0; j < ng; ++j) {
    const double fx = std::round((o->xgauge[j] - o->x[0]) / o->dx), fy = std::round((o->ygauge[j] - o->y[0]) / o->dy);
    if (!(fx >= 0 && fx < nx && fy >= 0 && fy < ny)) return fail("Gauges are outside of the domain!");
    gx[j] = (int)fx;
    gy[j] = (int)fy;
    gpt[j] = gy[j] * nx + gx[j];
  }
  if (!c->ensure_out(ng)) return -1;
  if (ng > 0)
    if (const cudaError_t e = cudaMemcpy(c->ogpt, gpt.data(), ng * sizeof(int), cudaMemcpyHostToDevice);
        e != cudaSuccess)
      return -c->fail("gauge upload", e);
  const std::string pre(o->outdir);
  OutFiles files;
  static const char* kField[3] = {"eta", "u", "v"};
  if (ng > 0)
    for (int f = 0; f < 3; ++f) {
      files.gauge[f] = fopen((pre + "Hawassi_" + kField[f] + "_gauge.dat").c_str(), "wb");
      if (!files.gauge[f]) return fail("cannot open " + pre + "Hawassi_" + kField[f] + "_gauge.dat");
    }
  int ipart = 1;
  char name[64];
  for (int i = 0; i < o->nt; ++i) {
    if (c->run(o->tout[i], false)) return -1;
    const double t = c->hctl->t;
    const bool first = (i % ntpart) == 0;
    const bool uv = o->uv_every_sample || first;
    c->fields_launch(c->stream, true);
    if (ng > 0) {
      hw2d::k2o_gauge<<<(ng + 127) / 128, 128, 0, c->stream>>>(c->ophys, c->ogpt, ng, n, c->ogval);
      c->launches += 1;
      cudaMemcpyAsync(c->hgval, c->ogval, 3 * (size_t)ng * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    }
    cudaMemcpyAsync(c->hf32, c->of32, (uv ? 3 : 1) * n * sizeof(float), cudaMemcpyDeviceToHost, c->stream);
    if (const cudaError_t e = cudaStreamSynchronize(c->stream); e != cudaSuccess) return -c->fail("output stage", e);
    if (!c->check("output stage")) return -1;
    if (first) {
      // the reference opens the next partition's files without closing the last ones
      files.close_part();
      for (int f = 0; f < 3; ++f) {
        snprintf(name, sizeof name, "Hawassi_%s_%02d.dat", kField[f], ipart);
        files.part[f] = fopen((pre + name).c_str(), "wb");
        if (!files.part[f]) return fail("cannot open " + pre + name);
      }
      if (i == 0) {
        snprintf(name, sizeof name, "Constant_%02d.dat", ipart);
        if (!write_constant(pre + name, o, nx, ny, ntpart)) return fail("cannot write " + pre + name);
      }
      ++ipart;
    }
    bool ok = fwrite(c->hf32, sizeof(float), n, files.part[0]) == n;
    if (uv)
      ok = ok && fwrite(c->hf32 + n, sizeof(float), n, files.part[1]) == n &&
           fwrite(c->hf32 + 2 * n, sizeof(float), n, files.part[2]) == n;
    for (FILE* f : files.part) ok = ok && fflush(f) == 0;
    if (ng > 0) {
      // print_data_gauges_uv (2d/fun_odesolver.c:427-476)
      for (int f = 0; f < 3; ++f) {
        FILE* g = files.gauge[f];
        if (i == 0) {
          fprintf(g, "0 ");
          for (int j = 0; j < ng; ++j) fprintf(g, "%f ", o->x[gx[j]]);
          fprintf(g, "\n");
          fprintf(g, "0 ");
          for (int j = 0; j < ng; ++j) fprintf(g, "%f ", o->y[gy[j]]);
          fprintf(g, "\n");
        }
        fprintf(g, "%f ", t);
        for (int j = 0; j < ng; ++j) fprintf(g, "%f ", c->hgval[3 * j + f]);
        fprintf(g, "\n");
        ok = ok && fflush(g) == 0;
      }
    }
    if (!ok) return fail("output files: write failed");
    if (std::isnan(c->hf32[n - 1])) {
      snprintf(name, sizeof name, "Time stepping failed at t=%fs.", t);
      return fail(name);
    }
  }
  if (c->brk.on) {
    // breaking.dat (2d/breaking.c:707-718): "t" then " x y " per break node, one line a record
    const int nrec = hw2d_breaking_log(c, nullptr, nullptr, nullptr, 0, 0);
    if (nrec < 0) return fail(nrec == -2 ? "breaking log overflowed" : "breaking log read failed");
    const long long nn = hw2d_breaking_log_nodes(c);
    std::vector<double> tr(nrec);
    std::vector<int> cnt(nrec), nodes(2 * (size_t)std::max(nn, 0LL));
    if (hw2d_breaking_log(c, tr.data(), cnt.data(), nodes.data(), nrec, nn) != nrec)
      return fail("breaking log read failed");
    FILE* f = fopen((pre + "breaking.dat").c_str(), "w");
    if (!f) return fail("cannot open " + pre + "breaking.dat");
    size_t k = 0;
    for (int r = 0; r < nrec; ++r) {
      fprintf(f, "%lf ", tr[r]);
      for (int j = 0; j < cnt[r] && k < (size_t)nn; ++j, ++k) fprintf(f, " %d %d ", nodes[2 * k], nodes[2 * k + 1]);
      fprintf(f, "\n");
    }
    if (fclose(f) != 0) return fail("cannot write " + pre + "breaking.dat");
  }
  return o->nt;
}

int hw2d_set_stream(hw2d_ctx* c, void* s) {
  if (!c) return 1;
  c->stream = s ? static_cast<cudaStream_t>(s) : c->own_stream;
  return 0;
}

int hw2d_synchronize(hw2d_ctx* c) {
  if (!c) return 1;
  return cudaStreamSynchronize(c->stream) == cudaSuccess ? 0 : 1;
}

}  // extern "C"
