// hw_kernels.h -- host-callable launchers of the per-slice-size kernels.
#pragma once

#include <cuda_runtime.h>

#include "hw_device.cuh"

#define HW_DECLARE(MM)                                                                             \
  cudaError_t hw_attr_##MM();                                                                      \
  cudaError_t hw_launch_##MM(int mode, hwdev::DevMember* mems, const int* list, int nmem, int C, \
                             double t, cudaStream_t s, int* queue, int ngrid);                    \
  int hw_max_clusters_##MM(int C);
HW_DECLARE(256)
HW_DECLARE(512)
HW_DECLARE(1024)
HW_DECLARE(2048)
#undef HW_DECLARE
