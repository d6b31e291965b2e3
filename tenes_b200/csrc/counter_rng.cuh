// Counter-based random numbers shared by the kernels that draw them: the
// rSVD Gaussian test matrices and the CholeskyQR perturbation.  The CPU
// oracle's counter_normal (oracle/tenes_oracle.py) computes the same numbers.
#pragma once

#include <cstdint>

namespace tg {

// splitmix64 finaliser on a Weyl sequence -> uniform in (0, 1)
__device__ __forceinline__ double counter_uniform(uint64_t idx, uint64_t key) {
  uint64_t z = idx * 0x9E3779B97F4A7C15ull + key;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z = z ^ (z >> 31);
  return (static_cast<double>(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

// standard normal number n of stream `key` (Box-Muller on counters 2n, 2n+1)
__device__ __forceinline__ double counter_gauss(uint64_t n, uint64_t key) {
  const double u1 = counter_uniform(2 * n, key);
  const double u2 = counter_uniform(2 * n + 1, key);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

// uniform number of mean 0 and variance 1 (on (-sqrt 3, sqrt 3)) from
// counter idx of stream `key`: the CholeskyQR perturbation, whose only
// purpose is to make rank-deficient panels full rank
__device__ __forceinline__ double counter_unit_uniform(uint64_t idx, uint64_t key) {
  return (2.0 * counter_uniform(idx, key) - 1.0) * 1.7320508075688772;
}

// keys of the CholeskyQR perturbation stream `stream` (real, imaginary parts),
// disjoint from the rSVD test matrices' keys
inline uint64_t noise_key_re(uint64_t stream) { return 0xD1B54A32D192ED03ull + (2 * stream) * 0xBF58476D1CE4E5B9ull; }
inline uint64_t noise_key_im(uint64_t stream) {
  return 0xD1B54A32D192ED03ull + (2 * stream + 1) * 0xBF58476D1CE4E5B9ull;
}

}  // namespace tg
