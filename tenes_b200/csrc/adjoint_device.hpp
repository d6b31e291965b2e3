// Device instantiation of the CTMRG energy adjoint (adjoint.hpp) on the
// library's device tensors and sm_100a kernels.
#pragma once

#include <functional>
#include <vector>

#include "adjoint.hpp"
#include "dtensor.hpp"

namespace tg {

// Thin SVD of a row-major m x n matrix (A is consumed): U (m x k), s (k), VT (k x n).
using SvdFn = std::function<void(DT<double>& A, int64_t m, int64_t n, DT<double>& U, DT<double>& s,
                                 DT<double>& VT)>;

// E and, when grads != nullptr, dE/dTn per site (see adjoint.hpp), on stream st.
double energy_grad_device(cudaStream_t st, const Lattice& lat, const std::vector<DT<double>>& Tn,
                          const std::vector<ad::WindowTerm>& terms, const ad::Options& o, const SvdFn& svd,
                          std::vector<DT<double>>* grads);

}  // namespace tg
