// Two-level (patch + dense interface) solve of the skeleton system.
#pragma once

#include <algorithm>
#include <cstddef>

#include "device.hpp"

namespace stx {

// Doubles of scratch twolevel_solve needs (interface RHS and solution).
size_t twolevel_workspace_doubles(const DevModal& S, int nz);

// In place on the skeleton vectors R[k][0..nglobal) of every solved plane:
// on entry the condensed right-hand sides, on exit the skeleton solution.
cudaError_t twolevel_solve(const DevModal& S, double* R, int rstride, double* work, int nz, cudaStream_t st);

int twolevel_launches(const DevModal& S);

}  // namespace stx
