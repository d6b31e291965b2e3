// Shared types and error handling of libtenes_gpu.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "tenes_gpu.h"

namespace tg {

// complex128 is stored as interleaved (re, im) doubles: double2 on device.
using cplx = double2;

template <typename T>
struct is_cplx {
  static constexpr bool value = false;
};
template <>
struct is_cplx<cplx> {
  static constexpr bool value = true;
};

// Error carried across the C ABI as a tg_status (never thrown past it).
struct Error : std::runtime_error {
  tg_status code;
  Error(tg_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(tg_status c, const std::string& m) { throw Error(c, m); }

inline void check_cuda(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess) {
    fail(TG_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e) + " at " + file + ":" +
                        std::to_string(line));
  }
}

#define TG_CUDA(x) ::tg::check_cuda((x), #x, __FILE__, __LINE__)
#define TG_CHECK_LAUNCH() ::tg::check_cuda(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

// Number of kernels launched by this library (host-side counter).
void count_launch(uint64_t n = 1);
uint64_t launch_count();

using Shape = std::vector<int64_t>;

inline int64_t numel(const Shape& s) {
  int64_t n = 1;
  for (auto d : s) n *= d;
  return n;
}

}  // namespace tg
