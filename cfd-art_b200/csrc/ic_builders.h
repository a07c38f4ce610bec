// Shape programs of the named test cases and the seeded recipes (built on the
// host in host/ic.cpp, evaluated there and by the device builder).
#pragma once

#include <stdint.h>

#include <vector>

#include "../../include/cfdgpu.h"
#include "ic_program.h"

namespace cfdic {

// CFD_OK, or CFD_ERR_INVALID (unknown case, or recipe for the other model).
int case_program(const cfd_config* cfg, const char* test_case, uint64_t seed,
                 std::vector<Op>& ops, Eos& q);
int recipe_program(const cfd_config* cfg, int recipe, uint64_t seed, int nbubbles,
                   std::vector<Op>& ops, Eos& q);

}  // namespace cfdic
