// hw_inst_1024.cu -- kernels for 1024-point slices.
#include "hw_kernels.cuh"

HW_INSTANTIATE(1024)
