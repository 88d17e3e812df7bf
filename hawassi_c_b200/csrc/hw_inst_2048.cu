// hw_inst_2048.cu -- kernels for 2048-point slices.
#include "hw_kernels.cuh"

HW_INSTANTIATE(2048)
