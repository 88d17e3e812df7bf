// hw_inst_512.cu -- kernels for 512-point slices.
#include "hw_kernels.cuh"

HW_INSTANTIATE(512)
