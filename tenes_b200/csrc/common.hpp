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

// Message returned by tg_last_error() on this thread.
void set_last_error(const std::string& m);

[[noreturn]] inline void fail(tg_status c, const std::string& m) { throw Error(c, m); }

inline void check_cuda(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess) {
    fail(TG_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e) + " at " + file + ":" +
                        std::to_string(line));
  }
}

#define TG_CUDA(x) ::tg::check_cuda((x), #x, __FILE__, __LINE__)
#define TG_CHECK_LAUNCH() ::tg::check_cuda(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

// Raise the dynamic shared-memory limit of `kernel` on the current device to
// at least `bytes`.  cudaFuncSetAttribute acts on the current device's
// context only, so what has been set is remembered per (kernel, device),
// under a lock shared by all host threads.
void ensure_dynamic_smem(const void* kernel, size_t bytes);

// Current device ordinal, checked against the per-device tables (64 devices).
int current_device();
constexpr int kMaxDevices = 64;

// Number of kernels launched by this library (host-side counter).  Kernels
// recorded into a CUDA graph are taken back off with uncount_launch and
// counted again at every launch of the graph.
void count_launch(uint64_t n = 1);
void uncount_launch(uint64_t n);
uint64_t launch_count();

// Optional per-launch CUDA-event profiling, grouped by kernel family.  When
// enabled, every launch of the family is bracketed by two events on its
// stream; the totals (launches, device ms, algorithmic flops / bytes) are
// read back by tg_profile_query.
enum ProfKind {
  PK_GEMM = 0,       // FP64 DMMA strided batched matrix product
  PK_PERMUTE = 1,    // leg permutation
  PK_NORMALIZE = 2,  // max-abs normalisation
  PK_SPECTRUM = 3,   // batched Jacobi corner spectra
  PK_SOLVER = 4,     // dense factorisations: cuSOLVER, CholeskyQR, Jacobi SVD of the rSVD core
  PK_OTHER = 5,      // small helpers
  PK_GEMM_TC = 6,    // 3xTF32 tcgen05 product, split / pack pre-pass included (flops: 2 M N K)
  PK_COUNT = 7
};
void profile_enable(bool on);
bool profile_enabled();
void profile_reset();
void profile_query(int kind, uint64_t* launches, double* ms, double* flops, double* bytes);

struct ProfScope {
  int kind;
  cudaStream_t st;
  double flops, bytes;
  cudaEvent_t e0 = nullptr;
  ProfScope(int k, cudaStream_t s, double f, double b);
  ~ProfScope();
};

using Shape = std::vector<int64_t>;

inline int64_t numel(const Shape& s) {
  int64_t n = 1;
  for (auto d : s) n *= d;
  return n;
}

}  // namespace tg
