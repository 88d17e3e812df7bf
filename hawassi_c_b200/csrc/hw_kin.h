// hw_kin.h -- kinematics of the 1D model (kinematic_modul, 1d/kinematic_modul.c)
// on the device: velocity-potential derivatives, pressure and accelerations under
// the surface on the overlay window [xinterv1, xinterv2] x zoutIP of a member
// whose deck has "kinematic yes".  Host interface used by the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "hw_setup.hpp"

namespace hwkin {

struct Kin;

// Static tables of read_kinematics (1d/functions.c:3555-3669) and of the
// interpolation kinematic_modul builds (sinhcosh2IP over 101 total depths).
// Returns nullptr with err set on unsupported input (runup, nsurf < 2, ...).
Kin* kin_create(const hw::Member& m, std::string& err);
void kin_destroy(Kin* k);
// device buffers (4 Nx doubles) for the state (which = 0) and its RHS (which = 1)
// in the reference layout, filled by the caller before kin_run
double* kin_state_buffer(Kin* k, int which);
void kin_dims(const Kin* k, int* nx_out, int* nz_out);
void kin_grid(const Kin* k, double* x_out, double* z_out);
// One evaluation at time t from the state y and its RHS dy, both in the
// reference layout on the device; results stay on the device until kin_fetch.
bool kin_run(Kin* k, const double* d_y, const double* d_dy, double t, double tprev, cudaStream_t s,
             std::string& err);
// Copy the last evaluation to host arrays ([nx_out][nz_out], x-major; eta_cut [nx_out]).
bool kin_fetch(Kin* k, double* eta_cut, double* P, double* dxphi, double* dzphi, double* dtdxphi, double* dtdzphi,
               cudaStream_t s, std::string& err);

}  // namespace hwkin
