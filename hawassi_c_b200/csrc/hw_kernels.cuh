// hw_kernels.cuh -- the persistent evolve kernel and the single-RHS kernel of one
// slice size M (instantiated once per M in hw_inst_<M>.cu).
#pragma once

#include "hw_breaking.cuh"
#include "hw_rhs_fast.cuh"
#include "hw_kernels.h"
#include "hw_stepper.cuh"
#include "hw_output.cuh"

// resident CTAs per SM the register allocation is sized for (slice M, M / 8 threads)
#ifndef HW_EVOLVE_MIN_BLOCKS
#define HW_EVOLVE_MIN_BLOCKS(M) (4096 / (M))
#endif

namespace hwdev {

// One member's work of a launch: mode 0 advances it through its output samples up to
// its stop index (clipping steps at each sample like the reference), mode 1 takes one
// evolve_apply to sd.t1.  The member's descriptor is in shared memory (sd).
template <int M>
__device__ __forceinline__ void evolve_member(DevMember* mems, int mi, int mode, DevMember& sd, double* red,
                                              double2* smem_buf, int C, int rank) {
  if (threadIdx.x == 0) sd = mems[mi];
  // a cluster barrier, not only the CTA's: the RHS's first phase writes into the
  // partner CTA's shared memory, which must be running
  member_sync(C);
  Ctx<M> X = make_ctx<M>(sd, smem_buf, red, rank);
  Bufs B;
  B.y = sd.y;
  B.yn = sd.ynew;
  for (int i = 0; i < 7; ++i) B.k[i] = sd.kb[i];
  StepState S{sd.t, sd.h, sd.status, sd.k1_valid, 0, 0, 0};
  int iout = sd.i_out;
  if (S.status == kOk) {
    if (mode == 1) {
      evolve_apply<M>(X, B, S, sd.t1);
    } else {
      while (iout < sd.i_stop && S.status == kOk) {
        const double ti = sd.tt[iout];
        while (S.t < ti && S.status == kOk) {
          evolve_apply<M>(X, B, S, ti);
          if (S.rhs >= sd.rhs_budget && S.status == kOk) S.status = kBudget;   // bounded launch
        }
        if (S.status == kOk) {
          if (sd.ngauge > 0 || sd.fields) output_stage<M>(X, B, S, iout);
          ++iout;
        }
      }
    }
  }
  member_sync(C);
  if (rank == 0 && threadIdx.x == 0) {
    DevMember& g = mems[mi];
    g.t = S.t;
    g.h = S.h;
    g.status = S.status;
    g.k1_valid = S.k1_valid;
    g.i_out = iout;
    g.rhs_calls += S.rhs;
    g.accepted += S.acc;
    g.rejected += S.rej;
    g.y = B.y;
    g.ynew = B.yn;
    for (int i = 0; i < 7; ++i) g.kb[i] = B.k[i];
  }
}

// The evolve kernel, persistent over a work queue: a grid of resident clusters (one
// cluster of C CTAs per member at a time) whose leaders take the next entry of the
// class's member list (ordered longest-first) from the queue counter until the list
// is used up, so no cluster waits for a member another cluster is running and the
// number of members in flight -- and their stage vectors in L2 -- is the grid's.
// With queue == nullptr cluster b runs entry b of the list (one cluster per member).
template <int M>
__global__ void __launch_bounds__(M / kPts, HW_EVOLVE_MIN_BLOCKS(M))
    k_evolve(DevMember* mems, const int* list, int mode, int* queue, int nlist) {
  extern __shared__ double2 smem_buf[];
  __shared__ DevMember sd;
  __shared__ double red[48];
  __shared__ int s_next;
  cg::cluster_group cl = cg::this_cluster();
  const int C = int(cl.num_blocks());
  const int rank = int(cl.block_rank());
  if (!queue) {
    evolve_member<M>(mems, list[blockIdx.x / C], mode, sd, red, smem_buf, C, rank);
    return;
  }
  for (;;) {
    if (rank == 0 && threadIdx.x == 0) s_next = atomicAdd(queue, 1);
    member_sync(C);
    // every CTA reads the leader's entry before the leader can take the next one: the
    // member's work below passes through cluster barriers first
    const int w = C > 1 ? *cl.map_shared_rank(&s_next, 0) : s_next;
    if (w >= nlist) break;
    evolve_member<M>(mems, list[w], mode, sd, red, smem_buf, C, rank);
  }
  // no CTA leaves while a peer may still read its shared memory
  member_sync(C);
}

// single RHS evaluation of member mi: kout = f(t, zs)
template <int M>
__global__ void __launch_bounds__(M / kPts, (4096 / M)) k_rhs(DevMember* mems, const int* list, double t) {
  extern __shared__ double2 smem_buf[];
  __shared__ DevMember sd;
  __shared__ double red[48];
  cg::cluster_group cl = cg::this_cluster();
  const int C = int(cl.num_blocks());
  const int rank = int(cl.block_rank());
  const int mi = list[blockIdx.x / C];
  if (threadIdx.x == 0) sd = mems[mi];
  __syncthreads();
  Ctx<M> X = make_ctx<M>(sd, smem_buf, red, rank);
  rhs_eval<M>(X, t, sd.kb[6]);
  member_sync(C);
  if (rank == 0 && threadIdx.x == 0) mems[mi].rhs_calls += 1;
}


template <int M>
cudaError_t set_attrs() {
  const int bytes = int(slice_smem_bytes(M));
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_evolve<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_rhs<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_evolve<M>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_rhs<M>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

// resident clusters of C CTAs of the evolve kernel (the persistent grid's size limit)
template <int M>
int max_clusters(int C) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(C));
  cfg.blockDim = dim3(M / kPts);
  cfg.dynamicSmemBytes = slice_smem_bytes(M);
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = unsigned(C);
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_evolve<M>, &cfg) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return n;
}

// mode 0/1: evolve (nmem list entries; with a queue, ngrid resident clusters pull them);
// mode 2: one RHS of each listed member
template <int M>
cudaError_t launch(int mode, DevMember* mems, const int* list, int nmem, int C, double t, cudaStream_t s,
                   int* queue, int ngrid) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned((queue && mode != 2 ? ngrid : nmem) * C));
  cfg.blockDim = dim3(M / kPts);
  cfg.dynamicSmemBytes = slice_smem_bytes(M);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = unsigned(C);
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (mode == 2) return cudaLaunchKernelEx(&cfg, k_rhs<M>, mems, list, t);
  return cudaLaunchKernelEx(&cfg, k_evolve<M>, mems, list, mode, queue, nmem);
}

}  // namespace hwdev

#define HW_INSTANTIATE(MM)                                                                          \
  cudaError_t hw_attr_##MM() { return hwdev::set_attrs<MM>(); }                                    \
  cudaError_t hw_launch_##MM(int mode, hwdev::DevMember* mems, const int* list, int nmem, int C,  \
                             double t, cudaStream_t s, int* queue, int ngrid) {                     \
    return hwdev::launch<MM>(mode, mems, list, nmem, C, t, s, queue, ngrid);                        \
  }                                                                                                 \
  int hw_max_clusters_##MM(int C) { return hwdev::max_clusters<MM>(C); }
