// hw_noalloc.cu -- one RHS evaluation that allocates no device memory.
//
// Its scratch (the stage input, the RHS output and the twelve intermediate
// fields of the RHS) lives in the file-scope array g_rhs_scratch below instead
// of per-context cudaMalloc'd buffers.  Every GPU that loads this library holds
// the array (1 MiB) until the process exits.  Host code cannot pass the array's
// name to a kernel: the name is a host-side stand-in, not a device address.  The
// device address is fetched once per device with cudaGetSymbolAddress (with that
// device current) on the first call and reused.
//
// Everything else the RHS reads or writes stays in the context: the tables, the
// member's breaking state (crest records, B, the breaking.dat log), which a
// breaking deck's RHS advances exactly as hw_rhs does, and the member's RHS
// counter.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "hw_kernels.cuh"

namespace {

using namespace hwdev;

constexpr int kNoAllocMaxNx = 4096;   // largest grid the static scratch covers
constexpr int kSlots = 16;            // 2N stage input + 2N output + 12 N fields, in N double2 units
static __device__ __align__(256) double2 g_rhs_scratch[size_t(kSlots) * kNoAllocMaxNx];

constexpr int kMaxDevices = 128;

// per-device set-up done by the first call on that device (the scratch array's
// device address and the kernels' attributes), under a lock so that two host
// threads making their first call on one device at once do it once
struct DeviceScratch {
  bool ready = false;
  double2* ptr = nullptr;
};
DeviceScratch g_scratch_addr[kMaxDevices];
std::mutex g_setup_lock;

template <int M>
__global__ void __launch_bounds__(M / kPts, (4096 / M)) k_rhs_noalloc(DevMember* mems, int mi, double t,
                                                                      const double* __restrict__ y_ref,
                                                                      double* __restrict__ dy_ref,
                                                                      double2* scratch) {
  extern __shared__ double2 smem_buf[];
  __shared__ DevMember sd;
  __shared__ double red[48];
  cg::cluster_group cl = cg::this_cluster();
  const int rank = int(cl.block_rank());
  if (threadIdx.x == 0) {
    sd = mems[mi];
    const int N = sd.N;
    sd.zs = scratch;
    sd.kb[6] = scratch + 2 * N;
    for (int i = 0; i < kScratch; ++i) sd.sc[i] = scratch + size_t(4 + i) * N;
  }
  __syncthreads();
  Ctx<M> X = make_ctx<M>(sd, smem_buf, red, rank);
  const int N = sd.N;
  // reference layout -> this CTA's spectral slice of the stage input
  HW_FOREACH(X) {
    const int kk = X.c + (idx << sd.logC);
    sd.zs[p] = make_double2(y_ref[kk], y_ref[N + kk]);
    sd.zs[N + p] = make_double2(y_ref[2 * N + kk], y_ref[3 * N + kk]);
  }
  rhs_eval<M>(X, t, sd.kb[6]);
  HW_FOREACH(X) {
    const int kk = X.c + (idx << sd.logC);
    const double2 e = sd.kb[6][p], u = sd.kb[6][N + p];
    dy_ref[kk] = e.x;
    dy_ref[N + kk] = e.y;
    dy_ref[2 * N + kk] = u.x;
    dy_ref[3 * N + kk] = u.y;
  }
  member_sync(int(cl.num_blocks()));
  if (rank == 0 && threadIdx.x == 0) mems[mi].rhs_calls += 1;
}

template <int M>
cudaError_t set_noalloc_attrs() {
  const int bytes = int(slice_smem_bytes(M));
  cudaError_t e = cudaFuncSetAttribute(k_rhs_noalloc<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_rhs_noalloc<M>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

template <int M>
cudaError_t launch_noalloc(DevMember* mems, int mi, int C, double t, const double* y, double* dy,
                           double2* scratch, cudaStream_t s) {
  const int bytes = int(slice_smem_bytes(M));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(C));
  cfg.blockDim = dim3(M / kPts);
  cfg.dynamicSmemBytes = size_t(bytes);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = unsigned(C);
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_rhs_noalloc<M>, mems, mi, t, y, dy, scratch);
}

}  // namespace

int hw_noalloc_max_nx() { return kNoAllocMaxNx; }

// Launch the no-allocation RHS for member mi (grid N, slice M, cluster C) on stream s,
// with the member's device (dev) current.  The first call on a device looks up the
// scratch array's device address and sets the kernels' attributes, once, under a lock.
bool hw_noalloc_rhs_launch(DevMember* mems, int mi, int N, int M, int C, double t, const double* y,
                           double* dy, cudaStream_t s, int dev, std::string& err) {
  if (N > kNoAllocMaxNx) {
    err = "hw_rhs_noalloc: Nx=" + std::to_string(N) + " exceeds the " + std::to_string(kNoAllocMaxNx) +
          "-point limit of its static scratch";
    return false;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    err = "hw_rhs_noalloc: device ordinal " + std::to_string(dev) + " out of range";
    return false;
  }
  cudaError_t e = cudaSuccess;
  DeviceScratch& ds = g_scratch_addr[dev];
  {
    std::lock_guard<std::mutex> lk(g_setup_lock);
    if (!ds.ready) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_rhs_scratch);
      if (e != cudaSuccess) {
        err = std::string("hw_rhs_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e);
        return false;
      }
      if ((e = set_noalloc_attrs<256>()) != cudaSuccess || (e = set_noalloc_attrs<512>()) != cudaSuccess ||
          (e = set_noalloc_attrs<1024>()) != cudaSuccess || (e = set_noalloc_attrs<2048>()) != cudaSuccess) {
        err = std::string("hw_rhs_noalloc: cudaFuncSetAttribute: ") + cudaGetErrorString(e);
        return false;
      }
      ds.ptr = static_cast<double2*>(p);
      ds.ready = true;
    }
  }
  switch (M) {
    case 256: e = launch_noalloc<256>(mems, mi, C, t, y, dy, ds.ptr, s); break;
    case 512: e = launch_noalloc<512>(mems, mi, C, t, y, dy, ds.ptr, s); break;
    case 1024: e = launch_noalloc<1024>(mems, mi, C, t, y, dy, ds.ptr, s); break;
    case 2048: e = launch_noalloc<2048>(mems, mi, C, t, y, dy, ds.ptr, s); break;
    default: e = cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) {
    err = std::string("hw_rhs_noalloc: launch: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}
