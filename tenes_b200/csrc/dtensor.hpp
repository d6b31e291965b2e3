// Device-resident dense tensors and the tensordot / transpose primitives the
// CTMRG driver is written in.  A tensordot is mapped onto one strided DMMA
// matrix product; an operand is permuted first only when its free and
// contracted legs are not already two contiguous groups (the same leg algebra
// as mptensor::tensordot, which the reference calls everywhere).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <numeric>
#include <vector>

#include "common.hpp"
#include "kernels.cuh"

namespace tg {

// Stream-ordered allocation from the device's default memory pool (kept
// cached: the pool's release threshold is raised at context creation).
struct DevMem {
  void* p = nullptr;
  cudaStream_t st = nullptr;
  DevMem(size_t bytes, cudaStream_t s) : st(s) {
    if (bytes) TG_CUDA(cudaMallocAsync(&p, bytes, st));
  }
  ~DevMem() {
    if (p) cudaFreeAsync(p, st);
  }
  DevMem(const DevMem&) = delete;
  DevMem& operator=(const DevMem&) = delete;
};

template <typename T>
struct DT {
  T* p = nullptr;
  Shape sh;
  std::shared_ptr<DevMem> mem;

  DT() = default;
  DT(const Shape& s, cudaStream_t st) : sh(s) {
    mem = std::make_shared<DevMem>(sizeof(T) * static_cast<size_t>(numel(s)), st);
    p = static_cast<T*>(mem->p);
  }
  int64_t size() const { return numel(sh); }
  int rank() const { return static_cast<int>(sh.size()); }
  int64_t dim(int i) const { return sh[static_cast<size_t>(i)]; }
  bool empty() const { return p == nullptr; }
};

template <typename T>
DT<T> zeros(const Shape& s, cudaStream_t st) {
  DT<T> t(s, st);
  TG_CUDA(cudaMemsetAsync(t.p, 0, sizeof(T) * static_cast<size_t>(t.size()), st));
  return t;
}

template <typename T>
DT<T> clone(const DT<T>& a, cudaStream_t st) {
  DT<T> t(a.sh, st);
  TG_CUDA(cudaMemcpyAsync(t.p, a.p, sizeof(T) * static_cast<size_t>(a.size()),
                          cudaMemcpyDeviceToDevice, st));
  return t;
}

inline bool is_identity(const std::vector<int>& p) {
  for (size_t i = 0; i < p.size(); ++i)
    if (p[i] != static_cast<int>(i)) return false;
  return true;
}

// out.shape[i] = a.shape[perm[i]]
template <typename T>
DT<T> transpose(const DT<T>& a, const std::vector<int>& perm, cudaStream_t st, bool conj = false) {
  if (static_cast<int>(perm.size()) != a.rank()) fail(TG_E_INPUT, "transpose: rank mismatch");
  Shape s(perm.size());
  for (size_t i = 0; i < perm.size(); ++i) s[i] = a.sh[static_cast<size_t>(perm[i])];
  DT<T> out(s, st);
  if (is_identity(perm) && !conj) {
    TG_CUDA(cudaMemcpyAsync(out.p, a.p, sizeof(T) * static_cast<size_t>(a.size()),
                            cudaMemcpyDeviceToDevice, st));
  } else {
    permute<T>(a.p, out.p, a.sh, perm, conj, st);
  }
  return out;
}

template <typename T>
DT<T> reshape(const DT<T>& a, const Shape& s) {
  if (numel(s) != a.size()) fail(TG_E_INPUT, "reshape: size mismatch");
  DT<T> t = a;
  t.sh = s;
  return t;
}

// A tensordot reduced to one matrix product: the operands as used (the
// inputs themselves, or permuted copies where no strided matrix view
// exists), the allocated result and the product's descriptor.
template <typename T>
struct TdPlan {
  DT<T> A, B, C;
  GemmDesc g{};
};

template <typename T>
TdPlan<T> plan_tensordot(const DT<T>& A, const DT<T>& B, const std::vector<int>& axA,
                         const std::vector<int>& axB, cudaStream_t st, bool conjA = false,
                         bool conjB = false, int prec = 0) {
  if (axA.size() != axB.size()) fail(TG_E_INPUT, "tensordot: axes length mismatch");
  std::vector<int> freeA, freeB;
  for (int i = 0; i < A.rank(); ++i)
    if (std::find(axA.begin(), axA.end(), i) == axA.end()) freeA.push_back(i);
  for (int i = 0; i < B.rank(); ++i)
    if (std::find(axB.begin(), axB.end(), i) == axB.end()) freeB.push_back(i);
  int64_t M = 1, N = 1, K = 1;
  Shape out;
  for (int i : freeA) {
    M *= A.dim(i);
    out.push_back(A.dim(i));
  }
  for (int i : freeB) {
    N *= B.dim(i);
    out.push_back(B.dim(i));
  }
  for (size_t i = 0; i < axA.size(); ++i) {
    if (A.dim(axA[i]) != B.dim(axB[i])) fail(TG_E_INPUT, "tensordot: contracted dims differ");
    K *= A.dim(axA[i]);
  }
  TdPlan<T> pl;
  GemmDesc& g = pl.g;
  g.M = M;
  g.N = N;
  g.K = K;
  g.batch = 1;
  g.conjA = conjA;
  g.conjB = conjB;
  g.accumulate = false;
  g.prec = prec;
  // A as (M, K) or (K, M)
  pl.A = A;
  std::vector<int> pa(freeA);
  pa.insert(pa.end(), axA.begin(), axA.end());
  std::vector<int> pa2(axA);
  pa2.insert(pa2.end(), freeA.begin(), freeA.end());
  if (is_identity(pa)) {
    g.sAm = K;
    g.sAk = 1;
  } else if (is_identity(pa2)) {
    g.sAm = 1;
    g.sAk = M;
  } else {
    pl.A = transpose(A, pa, st);
    g.sAm = K;
    g.sAk = 1;
  }
  pl.B = B;
  std::vector<int> pb(axB);
  pb.insert(pb.end(), freeB.begin(), freeB.end());
  std::vector<int> pb2(freeB);
  pb2.insert(pb2.end(), axB.begin(), axB.end());
  if (is_identity(pb)) {
    g.sBk = N;
    g.sBn = 1;
  } else if (is_identity(pb2)) {
    g.sBk = 1;
    g.sBn = K;
  } else {
    pl.B = transpose(B, pb, st);
    g.sBk = N;
    g.sBn = 1;
  }
  g.sCm = N;
  g.sCn = 1;
  pl.C = DT<T>(out, st);
  if (K == 0) TG_CUDA(cudaMemsetAsync(pl.C.p, 0, sizeof(T) * static_cast<size_t>(pl.C.size()), st));
  return pl;
}

// tensordot(A, B, axA, axB): result legs = free legs of A (in order) then
// free legs of B (in order).  conjA / conjB conjugate the operands.
template <typename T>
DT<T> tensordot(const DT<T>& A, const DT<T>& B, const std::vector<int>& axA,
                const std::vector<int>& axB, cudaStream_t st, bool conjA = false,
                bool conjB = false, int prec = 0) {
  TdPlan<T> pl = plan_tensordot(A, B, axA, axB, st, conjA, conjB, prec);
  if (pl.g.K > 0) gemm<T>(pl.A.p, pl.B.p, pl.C.p, pl.g, st);
  return std::move(pl.C);
}

// Independent tensordots as one grouped product launch (FP64; see
// gemm_group): plan them all -- the permuted copies of their operands --
// then contract every one in one persistent launch.
template <typename T>
std::vector<DT<T>> tensordot_group(const std::vector<TdPlan<T>>& plans, cudaStream_t st) {
  std::vector<GroupItem> items;
  for (const TdPlan<T>& pl : plans) {
    if (pl.g.K == 0 || pl.g.M == 0 || pl.g.N == 0) continue;
    if (pl.g.prec != 0) fail(TG_E_RUNTIME, "tensordot_group: FP64 products only");
    GroupItem it;
    it.A = pl.A.p;
    it.B = pl.B.p;
    it.C = pl.C.p;
    it.M = pl.g.M;
    it.N = pl.g.N;
    it.K = pl.g.K;
    it.sAm = pl.g.sAm;
    it.sAk = pl.g.sAk;
    it.sBk = pl.g.sBk;
    it.sBn = pl.g.sBn;
    it.sCm = pl.g.sCm;
    it.sCn = pl.g.sCn;
    it.conjA = pl.g.conjA;
    it.conjB = pl.g.conjB;
    items.push_back(it);
  }
  if (!items.empty()) gemm_group<T>(items.data(), static_cast<int>(items.size()), st);
  std::vector<DT<T>> out;
  out.reserve(plans.size());
  for (const TdPlan<T>& pl : plans) out.push_back(pl.C);
  return out;
}

}  // namespace tg
