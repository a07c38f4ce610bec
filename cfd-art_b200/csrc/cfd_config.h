// Configuration checks and material constants shared by the library's
// translation units (defined in cfd_api.cu).
#pragma once

#include "../../include/cfdgpu.h"
#include "cfd_physics.cuh"

namespace cfd {

// The checks cfd_create applies to a configuration: CFD_OK, or a failure
// code with its message left for cfd_last_error.
int validate_config(const cfd_config* c);

// FP64 material constants of a configuration (gamma - 1 and gamma * pinf
// formed once, as the reference forms them inline).
Eos make_eos(const cfd_config& c);

}  // namespace cfd
