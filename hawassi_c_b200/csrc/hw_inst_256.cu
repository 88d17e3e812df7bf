// hw_inst_256.cu -- kernels for 256-point slices.
#include "hw_kernels.cuh"

HW_INSTANTIATE(256)
