// Allocation-free corner spectra.
//
// tg_corner_spectra_noalloc computes the same L2-normalised singular values as
// tg_corner_spectrum (the batched one-sided Jacobi kernel of kernels.cu), but
// for matrices the caller already holds in device memory, and without any
// device allocation: the one piece of scratch memory the kernel needs, the
// device-side table of matrix pointers, is the file-scope array below.
//
// It is meant for callers that cannot call cudaMalloc at the point where they
// need the spectra: code running inside a host-side memory budget that
// forbids new device allocations, callers that own every byte of device
// memory through their own pool, or a convergence check issued between other
// work where an allocation could synchronise the device.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "common.hpp"
#include "kernels.cuh"
#include "tenes_gpu.h"

namespace tg {
namespace {

constexpr int kNoallocMaxMatrices = 1024;

// Device-side pointer table (8 KiB).  Every GPU that loads the library holds
// it until the process exits.  All calls share it and it keeps the last
// call's contents, so calls whose work overlaps on the GPU race on it.
static __device__ __align__(256) const void* g_noalloc_ptrs[kNoallocMaxMatrices];

std::mutex g_mu;
void* g_symbol_addr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_ptrs on the current device, looked up once per
// device (the host-side name is only a stand-in, not a device address).
const void** scratch_address() {
  const int dev = current_device();
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_symbol_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_ptrs);
    if (e != cudaSuccess || p == nullptr)
      fail(TG_E_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_ptrs): ") + cudaGetErrorString(e));
    g_symbol_addr[dev] = p;
  }
  return static_cast<const void**>(g_symbol_addr[dev]);
}

}  // namespace
}  // namespace tg

extern "C" tg_status tg_corner_spectra_noalloc(const void* const* device_mats, int count, int n, int is_complex,
                                               double* device_out, void* stream) {
  try {
    if (!device_mats || !device_out) tg::fail(TG_E_INPUT, "null pointer argument");
    if (count < 1 || count > tg::kNoallocMaxMatrices)
      tg::fail(TG_E_INPUT, "count must be in 1.." + std::to_string(tg::kNoallocMaxMatrices) +
                               " (size of the static pointer table); got " + std::to_string(count));
    const int nmax = is_complex ? 112 : 160;
    if (n < 1 || n > nmax)
      tg::fail(TG_E_INPUT, "n must be in 1.." + std::to_string(nmax) + "; got " + std::to_string(n));
    for (int i = 0; i < count; ++i)
      if (!device_mats[i]) tg::fail(TG_E_INPUT, "null matrix pointer at index " + std::to_string(i));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const void** table = tg::scratch_address();
    // The copy is staged through this stack array, which is pageable: a
    // host-to-device cudaMemcpyAsync from pageable memory has read its source
    // when it returns, so the caller may reuse device_mats at once, even when
    // that array is page-locked (from page-locked memory the copy would read
    // it later, in stream order).
    const void* staged[tg::kNoallocMaxMatrices];
    for (int i = 0; i < count; ++i) staged[i] = device_mats[i];
    TG_CUDA(cudaMemcpyAsync(table, staged, sizeof(void*) * count, cudaMemcpyHostToDevice, st));
    if (is_complex) {
      tg::batched_spectrum<tg::cplx>(reinterpret_cast<const tg::cplx* const*>(table), count, n, device_out,
                                     nullptr, st);
    } else {
      tg::batched_spectrum<double>(reinterpret_cast<const double* const*>(table), count, n, device_out, nullptr,
                                   st);
    }
    return TG_OK;
  } catch (const tg::Error& e) {
    tg::set_last_error(e.what());
    return e.code;
  } catch (...) {
    tg::set_last_error("unknown error");
    return TG_E_RUNTIME;
  }
}
