// Device setup of the two-level skeleton matrices (see l2setup.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "host/mesh.hpp"
#include "host/patch.hpp"

namespace stx {

// Form, on the device, every mode's packed S_II^-1 (per patch family, at
// fam_off[m * nfamily + f]), G (at g_off[...]) and interface inverse (at
// if_off[m]) into d_pack (FP64, zeroed by the caller), from the element Schur
// complements hbb [nmodes][mesh families][next][next] and the pinned
// interface id of each mode (-1: none).  Synchronises `st`; throws when a
// system is not positive definite.  Temporaries stay within budget_bytes
// (modes are processed in chunks).
void l2_device_setup_guarded(const Mesh& M, const Numbering& N, const Patching& P, const std::vector<double>& hbb,
                             int nmodes, const std::vector<int>& pin, const std::vector<long long>& fam_off,
                             const std::vector<long long>& g_off, const std::vector<long long>& if_off,
                             double* d_pack, cudaStream_t st, size_t budget_bytes = size_t(2) << 30);

}  // namespace stx
