// isotropic.cuh -- the reference's isotropic-turbulence initial field on the
// device (generate_full_turbulence + init_isotropic_turbulence,
// isotropic_ini.cpp:16-193).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "common.cuh"

namespace ns3d {

// Writes rho = 1, the velocity field and p = Rgas (T = 1) into the interior
// cells of the FP64 primitive arrays Wp (device table of five pointers, layout
// L); other cells keep their values.  Allocates its own scratch (three complex
// fields), works on stream st and synchronises it.  Returns 0 or an NS3D_ERR_*
// status with a message in err.
int isotropic_fill(double *const *Wp, const Layout &L, double Rgas, cudaStream_t st, std::string &err);

}  // namespace ns3d
