// Hand-written sm_100a kernels of the CTMRG path: FP64 tensor-core (DMMA)
// strided batched matrix product, leg permutation, max-abs normalisation,
// projector truncation helpers and a batched one-sided Jacobi spectrum.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <numeric>
#include <vector>
#include <cmath>
#include <string>

#include "counter_rng.cuh"
#include "kernels.cuh"

namespace tg {

static std::atomic<uint64_t> g_launches{0};
void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void uncount_launch(uint64_t n) { g_launches.fetch_sub(n, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

int current_device() {
  int dev = 0;
  TG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) fail(TG_E_INPUT, "device ordinal out of range: " + std::to_string(dev));
  return dev;
}

void ensure_dynamic_smem(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> raised;
  const int dev = current_device();
  std::lock_guard<std::mutex> g(mu);
  size_t& cur = raised[{kernel, dev}];
  if (bytes > cur) {
    TG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    cur = bytes;
  }
}

namespace {
struct ProfRec {
  int kind;
  cudaEvent_t a, b;
  double flops, bytes;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRec> g_prof;
struct ProfTot {
  uint64_t n = 0;
  double ms = 0, flops = 0, bytes = 0;
};
ProfTot g_tot[PK_COUNT];

void prof_drain() {
  for (auto& r : g_prof) {
    float ms = 0.f;
    cudaEventSynchronize(r.b);
    cudaEventElapsedTime(&ms, r.a, r.b);
    auto& t = g_tot[r.kind];
    t.n += 1;
    t.ms += ms;
    t.flops += r.flops;
    t.bytes += r.bytes;
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  g_prof.clear();
}
}  // namespace

void profile_enable(bool on) {
  std::lock_guard<std::mutex> g(g_prof_mu);
  g_prof_on = on;
}
bool profile_enabled() { return g_prof_on; }
void profile_reset() {
  std::lock_guard<std::mutex> g(g_prof_mu);
  prof_drain();
  for (auto& t : g_tot) t = ProfTot{};
}
void profile_query(int kind, uint64_t* launches, double* ms, double* flops, double* bytes) {
  std::lock_guard<std::mutex> g(g_prof_mu);
  prof_drain();
  if (kind < 0 || kind >= PK_COUNT) fail(TG_E_INPUT, "profile kind out of range");
  const auto& t = g_tot[kind];
  if (launches) *launches = t.n;
  if (ms) *ms = t.ms;
  if (flops) *flops = t.flops;
  if (bytes) *bytes = t.bytes;
}

ProfScope::ProfScope(int k, cudaStream_t s, double f, double b) : kind(k), st(s), flops(f), bytes(b) {
  if (g_prof_on) {
    TG_CUDA(cudaEventCreate(&e0));
    TG_CUDA(cudaEventRecord(e0, st));
  }
}
ProfScope::~ProfScope() {
  if (!e0) return;
  cudaEvent_t e1;
  if (cudaEventCreate(&e1) != cudaSuccess) return;
  cudaEventRecord(e1, st);
  std::lock_guard<std::mutex> g(g_prof_mu);
  g_prof.push_back(ProfRec{kind, e0, e1, flops, bytes});
  if (g_prof.size() > 4096) prof_drain();
}

namespace {

__device__ __forceinline__ double re_of(double x) { return x; }
__device__ __forceinline__ double re_of(cplx x) { return x.x; }
__device__ __forceinline__ double im_of(double) { return 0.0; }
__device__ __forceinline__ double im_of(cplx x) { return x.y; }
__device__ __forceinline__ double abs_of(double x) { return fabs(x); }
__device__ __forceinline__ double abs_of(cplx x) { return hypot(x.x, x.y); }
__device__ __forceinline__ double conj_of(double x) { return x; }
__device__ __forceinline__ cplx conj_of(cplx x) { return make_double2(x.x, -x.y); }
__device__ __forceinline__ double mul_real(double x, double a) { return x * a; }
__device__ __forceinline__ cplx mul_real(cplx x, double a) { return make_double2(x.x * a, x.y * a); }
template <typename T>
__device__ __forceinline__ T zero_of();
template <>
__device__ __forceinline__ double zero_of<double>() { return 0.0; }
template <>
__device__ __forceinline__ cplx zero_of<cplx>() { return make_double2(0.0, 0.0); }
template <typename T>
__device__ __forceinline__ T one_of();
template <>
__device__ __forceinline__ double one_of<double>() { return 1.0; }
template <>
__device__ __forceinline__ cplx one_of<cplx>() { return make_double2(1.0, 0.0); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

int num_blocks(int64_t n, int threads, int64_t cap = 148 * 32) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  return static_cast<int>(std::min<int64_t>(b, cap));
}

// ---------------------------------------------------------------------------
// GEMM: 64 x 64 x 16 CTA tile, 4 warps of 32 x 32, register-staged double
// buffering of the global loads, DMMA m8n8k4 on the FP64 tensor pipe.
// Complex operands are split into real / imaginary planes in shared memory
// and multiplied with four real DMMAs per complex MAC.
// ---------------------------------------------------------------------------
constexpr int GBM = 64, GBN = 64, GBK = 16, GPAD = 4;
constexpr int GLD = GBM + GPAD;  // row length of the k-major smem tiles

template <typename T>
struct GemmParams {
  const T* A;
  const T* B;
  T* C;
  GemmDesc d;
};

template <typename T, bool CPLX>
__global__ void __launch_bounds__(128) gemm_kernel(GemmParams<T> p) {
  constexpr int NP = CPLX ? 2 : 1;  // planes
  extern __shared__ double smem[];
  // layout: As[stage][plane][GBK][GLD], Bs[stage][plane][GBK][GLD]
  double* As = smem;
  double* Bs = smem + 2 * NP * GBK * GLD;
  const GemmDesc& d = p.d;
  const int64_t bz = blockIdx.z;
  const T* A = p.A + bz * d.bA;
  const T* B = p.B + bz * d.bB;
  T* C = p.C + bz * d.bC;
  const int64_t m0 = static_cast<int64_t>(blockIdx.y) * GBM;
  const int64_t n0 = static_cast<int64_t>(blockIdx.x) * GBN;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int wm = (warp & 1) * 32;
  const int wn = (warp >> 1) * 32;
  const bool a_kc = (d.sAk == 1);  // A contiguous along k
  const bool b_nc = (d.sBn == 1);  // B contiguous along n
  // split-K launches: the last chunk may be shorter
  const int64_t Kz = (d.klast > 0 && blockIdx.z == gridDim.z - 1) ? d.klast : d.K;

  T ra[8], rb[8];
  auto load_tiles = [&](int64_t k0) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int idx = tid + i * 128;
      int mm, kk;
      if (a_kc) {
        kk = idx % GBK;
        mm = idx / GBK;
      } else {
        mm = idx % GBM;
        kk = idx / GBM;
      }
      const int64_t gm = m0 + mm, gk = k0 + kk;
      ra[i] = (gm < d.M && gk < Kz) ? A[gm * d.sAm + gk * d.sAk] : zero_of<T>();
      int nn, kb;
      if (b_nc) {
        nn = idx % GBN;
        kb = idx / GBN;
      } else {
        kb = idx % GBK;
        nn = idx / GBK;
      }
      const int64_t gn = n0 + nn, gkb = k0 + kb;
      rb[i] = (gn < d.N && gkb < Kz) ? B[gkb * d.sBk + gn * d.sBn] : zero_of<T>();
    }
  };
  auto store_tiles = [&](int stage) {
    double* as = As + stage * NP * GBK * GLD;
    double* bs = Bs + stage * NP * GBK * GLD;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int idx = tid + i * 128;
      int mm, kk;
      if (a_kc) {
        kk = idx % GBK;
        mm = idx / GBK;
      } else {
        mm = idx % GBM;
        kk = idx / GBM;
      }
      as[kk * GLD + mm] = re_of(ra[i]);
      if constexpr (CPLX) as[GBK * GLD + kk * GLD + mm] = d.conjA ? -im_of(ra[i]) : im_of(ra[i]);
      int nn, kb;
      if (b_nc) {
        nn = idx % GBN;
        kb = idx / GBN;
      } else {
        kb = idx % GBK;
        nn = idx / GBK;
      }
      bs[kb * GLD + nn] = re_of(rb[i]);
      if constexpr (CPLX) bs[GBK * GLD + kb * GLD + nn] = d.conjB ? -im_of(rb[i]) : im_of(rb[i]);
    }
  };

  double acc_r[4][4][2];
  double acc_i[CPLX ? 4 : 1][CPLX ? 4 : 1][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc_r[i][j][0] = acc_r[i][j][1] = 0.0;
  if constexpr (CPLX) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc_i[i][j][0] = acc_i[i][j][1] = 0.0;
  }

  const int64_t nk = (Kz + GBK - 1) / GBK;
  load_tiles(0);
  store_tiles(0);
  __syncthreads();
  for (int64_t kt = 0; kt < nk; ++kt) {
    const int stage = static_cast<int>(kt & 1);
    if (kt + 1 < nk) load_tiles((kt + 1) * GBK);
    const double* as = As + stage * NP * GBK * GLD;
    const double* bs = Bs + stage * NP * GBK * GLD;
#pragma unroll
    for (int k4 = 0; k4 < GBK; k4 += 4) {
      const int kr = k4 + (lane & 3);
      double a_r[4], b_r[4], a_i[CPLX ? 4 : 1], b_i[CPLX ? 4 : 1];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a_r[i] = as[kr * GLD + wm + i * 8 + (lane >> 2)];
        b_r[i] = bs[kr * GLD + wn + i * 8 + (lane >> 2)];
        if constexpr (CPLX) {
          a_i[i] = as[GBK * GLD + kr * GLD + wm + i * 8 + (lane >> 2)];
          b_i[i] = bs[GBK * GLD + kr * GLD + wn + i * 8 + (lane >> 2)];
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          dmma(acc_r[i][j][0], acc_r[i][j][1], a_r[i], b_r[j]);
          if constexpr (CPLX) {
            dmma(acc_r[i][j][0], acc_r[i][j][1], -a_i[i], b_i[j]);
            dmma(acc_i[i][j][0], acc_i[i][j][1], a_r[i], b_i[j]);
            dmma(acc_i[i][j][0], acc_i[i][j][1], a_i[i], b_r[j]);
          }
        }
    }
    if (kt + 1 < nk) {
      store_tiles(stage ^ 1);
    }
    __syncthreads();
  }

  // epilogue
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int64_t gm = m0 + wm + i * 8 + (lane >> 2);
        const int64_t gn = n0 + wn + j * 8 + 2 * (lane & 3) + h;
        if (gm < d.M && gn < d.N) {
          T* c = C + gm * d.sCm + gn * d.sCn;
          if constexpr (CPLX) {
            cplx v = make_double2(acc_r[i][j][h], acc_i[i][j][h]);
            if (d.accumulate) {
              v.x += c->x;
              v.y += c->y;
            }
            *c = v;
          } else {
            double v = acc_r[i][j][h];
            if (d.accumulate) v += *c;
            *c = v;
          }
        }
      }
}

// ---------------------------------------------------------------------------
// Narrow FP64 GEMM (real operands, 64 < N <= 96): one column tile of 8 NF columns
// covers the whole of N, so N pads to the next multiple of 8 instead of 64
// -- the rSVD panels (N = k = chi + 10, 82 at chi = 72) waste 7% of the
// DMMAs instead of 36%.  CTA tile 64 x 8NF x 16, 4 warps of 16 rows x 8NF
// (2 x NF m8n8k4 fragments each).  The tiles move global -> shared with
// 8-byte cp.async (zero-filled outside the matrix) through a 3-stage ring,
// one barrier per k tile, so no registers hold staged elements.
// ---------------------------------------------------------------------------
constexpr int NSTAGE = 3;

__device__ __forceinline__ void cp_async8_zfill(double* dst, const double* src, bool valid) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const int n = valid ? 8 : 0;  // src-size 0: the 8 destination bytes are zero-filled
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int NF>
__global__ void __launch_bounds__(128) gemm_narrow_kernel(GemmParams<double> p) {
  constexpr int BN = 8 * NF;
  constexpr int LDB = BN + 4;  // LDB = 4 or 12 mod 16: conflict-free fragment reads
  constexpr int ASZ = GBK * GLD, BSZ = GBK * LDB;
  extern __shared__ double smem[];
  double* As = smem;                 // [NSTAGE][GBK][GLD]
  double* Bs = smem + NSTAGE * ASZ;  // [NSTAGE][GBK][LDB]
  const GemmDesc& d = p.d;
  const int64_t bz = blockIdx.z;
  const double* A = p.A + bz * d.bA;
  const double* B = p.B + bz * d.bB;
  double* C = p.C + bz * d.bC;
  const int64_t m0 = static_cast<int64_t>(blockIdx.y) * GBM;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int wm = (tid >> 5) * 16;
  const bool a_kc = (d.sAk == 1);
  const bool b_nc = (d.sBn == 1);
  const int64_t Kz = (d.klast > 0 && blockIdx.z == gridDim.z - 1) ? d.klast : d.K;
  const int64_t nk = (Kz + GBK - 1) / GBK;

  auto issue = [&](int64_t kt) {
    if (kt < nk) {
      const int64_t k0 = kt * GBK;
      double* as = As + (kt % NSTAGE) * ASZ;
      double* bs = Bs + (kt % NSTAGE) * BSZ;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int idx = tid + i * 128;
        const int mm = a_kc ? idx / GBK : idx % GBM;
        const int kk = a_kc ? idx % GBK : idx / GBM;
        const int64_t gm = m0 + mm, gk = k0 + kk;
        const bool ok = gm < d.M && gk < Kz;
        cp_async8_zfill(as + kk * GLD + mm, ok ? A + gm * d.sAm + gk * d.sAk : A, ok);
      }
#pragma unroll
      for (int i = 0; i < NF; ++i) {
        const int idx = tid + i * 128;
        const int nn = b_nc ? idx % BN : idx / GBK;
        const int kb = b_nc ? idx / BN : idx % GBK;
        const int64_t gk = k0 + kb;
        const bool ok = nn < d.N && gk < Kz;
        cp_async8_zfill(bs + kb * LDB + nn, ok ? B + gk * d.sBk + nn * d.sBn : B, ok);
      }
    }
    cp_async_commit();  // an empty group past the last tile keeps the group count uniform
  };

  double acc[2][NF][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < NF; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
  for (int s0 = 0; s0 < NSTAGE - 1; ++s0) issue(s0);
  for (int64_t kt = 0; kt < nk; ++kt) {
    cp_async_wait<NSTAGE - 2>();  // this thread's copies of tile kt have landed
    __syncthreads();              // ... everyone's; and tile kt-1's stage is free again
    issue(kt + NSTAGE - 1);
    const double* as = As + (kt % NSTAGE) * ASZ;
    const double* bs = Bs + (kt % NSTAGE) * BSZ;
#pragma unroll
    for (int k4 = 0; k4 < GBK; k4 += 4) {
      const int kr = k4 + (lane & 3);
      double a[2], b[NF];
#pragma unroll
      for (int i = 0; i < 2; ++i) a[i] = as[kr * GLD + wm + i * 8 + (lane >> 2)];
#pragma unroll
      for (int j = 0; j < NF; ++j) b[j] = bs[kr * LDB + j * 8 + (lane >> 2)];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < NF; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
  }
  cp_async_wait<0>();

#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < NF; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int64_t gm = m0 + wm + i * 8 + (lane >> 2);
        const int64_t gn = j * 8 + 2 * (lane & 3) + h;
        if (gm < d.M && gn < d.N) {
          double* c = C + gm * d.sCm + gn * d.sCn;
          double v = acc[i][j][h];
          if (d.accumulate) v += *c;
          *c = v;
        }
      }
}

// ---------------------------------------------------------------------------
// Grouped persistent product (gemm_group in kernels.cuh).  The problem table
// travels as a __grid_constant__ kernel parameter (no copy, no memcpy node in
// a captured graph); tile t of the group belongs to the problem whose tile0
// is the last one <= t.  CTA tile (16 WFM) x (16 WFN) x 16, 4 warps of
// (8 WFM) x (8 WFN), operands staged global -> shared by cp.async through a
// 3-stage ring (zero-filled outside the matrix).  Complex operands stay
// interleaved in shared memory; each fragment load forms re, im and re + im.
// ---------------------------------------------------------------------------
struct GroupTab {
  struct P {
    const void* A;
    const void* B;
    void* C;
    void* part;  // split-K: nsplit partial products (M x N, row-major) instead of C
    int64_t M, N, K, sAm, sAk, sBk, sBn, sCm, sCn;
    int64_t kchunk;  // K of one split chunk (a multiple of 16)
    int tn, tiles;   // column tiles, output tiles
    int tile0;       // first work item (tile x chunk) of the problem
    int nsplit;
    int conjA, conjB;
  } p[kGroupMax];
  int count, total;
};
// the partial sums of the split problems of a group, added in chunk order
struct GroupRed {
  struct R {
    const void* part;
    void* C;
    int64_t M, N, sCm, sCn, elem0;
    int nsplit;
  } r[kGroupMax];
  int count;
  int64_t total;
};

__device__ __forceinline__ void cp_async16_zfill(void* dst, const void* src, bool valid) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src, bool valid) {
  if constexpr (is_cplx<T>::value) cp_async16_zfill(dst, src, valid);
  else cp_async8_zfill(dst, src, valid);
}

template <typename T, int WFM, int WFN>
__global__ void __launch_bounds__(128) gemm_group_kernel(const __grid_constant__ GroupTab tab) {
  constexpr bool CPLX = is_cplx<T>::value;
  constexpr int BM = 16 * WFM, BN = 16 * WFN;
  // row pitches: fragment reads conflict-free (8-byte: 4 mod 16; 16-byte: 2 mod 8)
  constexpr int LDA = BM + (CPLX ? 2 : 4), LDB = BN + (CPLX ? 2 : 4);
  constexpr int ASZ = GBK * LDA, BSZ = GBK * LDB;
  extern __shared__ __align__(16) double smem_g[];
  T* As = reinterpret_cast<T*>(smem_g);  // [NSTAGE][GBK][LDA]
  T* Bs = As + NSTAGE * ASZ;             // [NSTAGE][GBK][LDB]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp & 1) * (8 * WFM), wn = (warp >> 1) * (8 * WFN);
  constexpr int NACC = CPLX ? 3 : 1;

  for (int t = blockIdx.x; t < tab.total; t += gridDim.x) {
    int pi = 0;
    while (pi + 1 < tab.count && t >= tab.p[pi + 1].tile0) ++pi;
    const GroupTab::P& P = tab.p[pi];
    const int lt = (t - P.tile0) % P.tiles, z = (t - P.tile0) / P.tiles;  // tile, K chunk
    const int64_t m0 = static_cast<int64_t>(lt / P.tn) * BM, n0 = static_cast<int64_t>(lt % P.tn) * BN;
    const int64_t M = P.M, N = P.N;
    const int64_t kb0 = z * P.kchunk;
    const int64_t K = std::min(P.K - kb0, P.kchunk);  // this chunk's K
    const T* A = static_cast<const T*>(P.A) + kb0 * P.sAk;
    const T* B = static_cast<const T*>(P.B) + kb0 * P.sBk;
    const bool split = P.nsplit > 1;
    T* C = split ? static_cast<T*>(P.part) + z * M * N : static_cast<T*>(P.C);
    const int64_t sCm = split ? N : P.sCm, sCn = split ? 1 : P.sCn;
    const bool a_kc = P.sAk == 1, b_nc = P.sBn == 1;
    const int64_t nk = (K + GBK - 1) / GBK;

    auto issue = [&](int64_t kt) {
      if (kt < nk) {
        const int64_t k0 = kt * GBK;
        T* as = As + (kt % NSTAGE) * ASZ;
        T* bs = Bs + (kt % NSTAGE) * BSZ;
#pragma unroll
        for (int i = 0; i < BM / 8; ++i) {
          const int idx = tid + i * 128;
          const int mm = a_kc ? idx / GBK : idx % BM;
          const int kk = a_kc ? idx % GBK : idx / BM;
          const int64_t gm = m0 + mm, gk = k0 + kk;
          const bool ok = gm < M && gk < K;
          cp_async_elem<T>(as + kk * LDA + mm, ok ? A + gm * P.sAm + gk * P.sAk : A, ok);
        }
#pragma unroll
        for (int i = 0; i < BN / 8; ++i) {
          const int idx = tid + i * 128;
          const int nn = b_nc ? idx % BN : idx / GBK;
          const int kb = b_nc ? idx / BN : idx % GBK;
          const int64_t gn = n0 + nn, gk = k0 + kb;
          const bool ok = gn < N && gk < K;
          cp_async_elem<T>(bs + kb * LDB + nn, ok ? B + gk * P.sBk + gn * P.sBn : B, ok);
        }
      }
      cp_async_commit();
    };

    double acc[NACC][WFM][WFN][2];
#pragma unroll
    for (int c = 0; c < NACC; ++c)
#pragma unroll
      for (int i = 0; i < WFM; ++i)
#pragma unroll
        for (int j = 0; j < WFN; ++j) acc[c][i][j][0] = acc[c][i][j][1] = 0.0;
    const double sa = P.conjA ? -1.0 : 1.0, sb = P.conjB ? -1.0 : 1.0;

#pragma unroll
    for (int s0 = 0; s0 < NSTAGE - 1; ++s0) issue(s0);
    for (int64_t kt = 0; kt < nk; ++kt) {
      cp_async_wait<NSTAGE - 2>();
      __syncthreads();
      issue(kt + NSTAGE - 1);
      const T* as = As + (kt % NSTAGE) * ASZ;
      const T* bs = Bs + (kt % NSTAGE) * BSZ;
#pragma unroll
      for (int k4 = 0; k4 < GBK; k4 += 4) {
        const int kr = k4 + (lane & 3);
        if constexpr (CPLX) {
          double ar[WFM], ai[WFM], br[WFN], bi[WFN];
#pragma unroll
          for (int i = 0; i < WFM; ++i) {
            const cplx v = as[kr * LDA + wm + i * 8 + (lane >> 2)];
            ar[i] = v.x;
            ai[i] = sa * v.y;
          }
#pragma unroll
          for (int j = 0; j < WFN; ++j) {
            const cplx v = bs[kr * LDB + wn + j * 8 + (lane >> 2)];
            br[j] = v.x;
            bi[j] = sb * v.y;
          }
#pragma unroll
          for (int i = 0; i < WFM; ++i)
#pragma unroll
            for (int j = 0; j < WFN; ++j) {
              dmma(acc[0][i][j][0], acc[0][i][j][1], ar[i], br[j]);
              dmma(acc[1][i][j][0], acc[1][i][j][1], ai[i], bi[j]);
              dmma(acc[2][i][j][0], acc[2][i][j][1], ar[i] + ai[i], br[j] + bi[j]);
            }
        } else {
          double a[WFM], b[WFN];
#pragma unroll
          for (int i = 0; i < WFM; ++i) a[i] = as[kr * LDA + wm + i * 8 + (lane >> 2)];
#pragma unroll
          for (int j = 0; j < WFN; ++j) b[j] = bs[kr * LDB + wn + j * 8 + (lane >> 2)];
#pragma unroll
          for (int i = 0; i < WFM; ++i)
#pragma unroll
            for (int j = 0; j < WFN; ++j) dmma(acc[0][i][j][0], acc[0][i][j][1], a[i], b[j]);
        }
      }
    }
    cp_async_wait<0>();

#pragma unroll
    for (int i = 0; i < WFM; ++i)
#pragma unroll
      for (int j = 0; j < WFN; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int64_t gm = m0 + wm + i * 8 + (lane >> 2);
          const int64_t gn = n0 + wn + j * 8 + 2 * (lane & 3) + h;
          if (gm < M && gn < N) {
            T* c = C + gm * sCm + gn * sCn;
            if constexpr (CPLX) {
              const double p1 = acc[0][i][j][h], p2 = acc[1][i][j][h], p3 = acc[2][i][j][h];
              *c = make_double2(p1 - p2, p3 - p1 - p2);
            } else {
              *c = acc[0][i][j][h];
            }
          }
        }
    __syncthreads();  // the next tile's first copies reuse the stages
  }
}

template <typename T>
__global__ void group_reduce_kernel(const __grid_constant__ GroupRed red) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < red.total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int ri = 0;
    while (ri + 1 < red.count && i >= red.r[ri + 1].elem0) ++ri;
    const GroupRed::R& R = red.r[ri];
    const int64_t e = i - R.elem0, len = R.M * R.N;
    const T* part = static_cast<const T*>(R.part);
    double re = 0.0, im = 0.0;
    for (int z = 0; z < R.nsplit; ++z) {
      const T v = part[z * len + e];
      re += re_of(v);
      im += im_of(v);
    }
    const int64_t m = e / R.N, n = e - m * R.N;
    T* c = static_cast<T*>(R.C) + m * R.sCm + n * R.sCn;
    if constexpr (is_cplx<T>::value) *c = make_double2(re, im);
    else *c = re;
  }
}

// ---------------------------------------------------------------------------
// Mixed precision: 3xTF32 product on the 5th-generation tensor cores
// (tcgen05.mma kind::tf32, accumulator in tensor memory).
//
// Each FP64 operand element a is split as a = hi + lo, hi = tf32(a),
// lo = tf32(a - hi) (residual taken in FP64), and a*b ~ hi*hi + hi*lo + lo*hi:
// three MMAs into one FP32 accumulator.  The split-K chunks of the launcher
// are summed in FP64, so FP32 accumulation runs over one chunk only.
//
// CTA: 256 threads, tile 128 (M, the TMEM lanes) x BN (N, TMEM columns), K
// staged 16 at a time through three shared-memory stages.  Each thread keeps
// two stages of its FP64 half-row of A (and half-column of B) in flight in
// registers, splits them with integer ALU work and stores hi / lo in the
// K-major no-swizzle canonical layout: 8-row x 16-byte core matrices,
// K-adjacent core matrices 128 B apart (LBO), 8-row groups 512 B apart (SBO).
// One thread issues the MMAs of a stage (two K=8 steps x three products) and
// commits them to the stage's mbarrier, which gates the reuse of that stage.
// The epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM lanes
// 32 (w % 4) and one half of the columns).  Every mbarrier wait is bounded
// (2 s of %globaltimer); a timeout sets g_tc_fault, skips the rest of the
// work and still releases the tensor memory.
// ---------------------------------------------------------------------------
__device__ int g_tc_fault = 0;

namespace tc {
constexpr int BM = 128, BK = 16, STAGES = 3, THREADS = 256;
constexpr uint32_t LBO = 128, SBO = (BK / 4) * 128;  // bytes

// x = hi + lo + O(2^-23 |x|), hi and lo TF32 values given as FP32 bits:
// one FP64 -> FP32 conversion, then round-to-nearest to 10 mantissa bits on
// the FP32 pattern; the residual xf - hi is exact in FP32.
__device__ __forceinline__ void split_tf32(double x, uint32_t& hi, uint32_t& lo) {
  const float xf = __double2float_rn(x);
  const uint32_t hb = (__float_as_uint(xf) + 0x1000u) & 0xFFFFE000u;
  const float l = xf - __uint_as_float(hb);
  hi = hb;
  lo = (__float_as_uint(l) + 0x1000u) & 0xFFFFE000u;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// byte offset of element (r, k) of an R x BK K-major canonical tile
__device__ __forceinline__ uint32_t tile_off(int r, int k) {
  return static_cast<uint32_t>((r >> 3) * SBO + (k >> 2) * LBO + (r & 7) * 16 + (k & 3) * 4);
}
__device__ __forceinline__ uint64_t desc(uint32_t addr) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFF) | (static_cast<uint64_t>((LBO >> 4) & 0x3FFF) << 16) |
         (static_cast<uint64_t>((SBO >> 4) & 0x3FFF) << 32) | (1ull << 46);  // version 1, no swizzle
}
// kind::tf32, F32 accumulator, A and B K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(n >> 3) << 17) | ((BM >> 4) << 24);
}
__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const uint64_t t0 = now_ns();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (now_ns() - t0 > 2000000000ull) return false;
  }
}
__device__ __forceinline__ void mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem), "l"(a), "l"(b), "r"(id), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
}  // namespace tc

template <int BN>
__global__ void __launch_bounds__(tc::THREADS) gemm_tc_tf32x3_kernel(GemmParams<double> p) {
  using namespace tc;
  constexpr int TILE_A = BM * BK * 4, TILE_B = BN * BK * 4;     // bytes of one hi or lo tile
  constexpr int STAGE = 2 * TILE_A + 2 * TILE_B;                // A hi, A lo, B hi, B lo
  constexpr int TCOLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
  extern __shared__ __align__(1024) uint8_t tc_smem[];
  __shared__ __align__(8) uint64_t mbar[STAGES];
  __shared__ uint32_t tmem_slot;
  const GemmDesc& d = p.d;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t bz = blockIdx.z;
  const double* A = p.A + bz * d.bA;
  const double* B = p.B + bz * d.bB;
  double* C = p.C + bz * d.bC;
  const int64_t m0 = static_cast<int64_t>(blockIdx.y) * BM, n0 = static_cast<int64_t>(blockIdx.x) * BN;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar[s])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t sbase = smem_addr(tc_smem);

  const int64_t nk = (d.K + BK - 1) / BK;
  // Each thread moves two pieces of four K-consecutive values per operand and
  // stage.  When the operand's rows are contiguous in memory (stride 1 along
  // M or N) piece p is row t & 127 at k = 8 (t >> 7) + 4p, so a warp reads
  // consecutive rows; when K is contiguous piece p is row (t >> 2) + 64p at
  // k = 4 (t & 3), so four threads read one row's 16 consecutive values.
  constexpr int KH = BK / 2;
  struct Pieces {
    int row[2], k[2];
    bool ok[2];
    const double* base[2];
    int64_t sk;
  };
  auto pieces = [&](const double* X, int64_t row0, int64_t nrows_valid, int nrows_tile, int64_t s_row,
                    int64_t s_k) {
    Pieces P;
    const bool rows_contig = (s_row == 1 && s_k != 1);
    for (int q = 0; q < 2; ++q) {
      P.row[q] = rows_contig ? (tid & (BM - 1)) : (tid >> 2) + 64 * q;
      P.k[q] = rows_contig ? (tid >> 7) * KH + 4 * q : 4 * (tid & 3);
      P.ok[q] = P.row[q] < nrows_tile && row0 + P.row[q] < nrows_valid;
      P.base[q] = X + (row0 + P.row[q]) * s_row;
    }
    P.sk = s_k;
    return P;
  };
  const Pieces PA = pieces(A, m0, d.M, BM, d.sAm, d.sAk);
  const Pieces PB = pieces(B, n0, d.N, BN, d.sBn, d.sBk);
  double ra0[KH], rb0[KH], ra1[KH], rb1[KH];
  auto load = [&](int64_t kt, double (&va)[KH], double (&vb)[KH]) {
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int64_t ka = kt * BK + PA.k[q] + j, kb = kt * BK + PB.k[q] + j;
        va[4 * q + j] = (PA.ok[q] && ka < d.K) ? PA.base[q][ka * PA.sk] : 0.0;
        vb[4 * q + j] = (PB.ok[q] && kb < d.K) ? PB.base[q][kb * PB.sk] : 0.0;
      }
  };
  auto split_store = [&](uint8_t* hi, uint8_t* lo, const double (&v)[KH], const Pieces& P, int nrows_tile) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      if (P.row[q] >= nrows_tile) continue;
      uint32_t h[4], l[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) split_tf32(v[4 * q + e], h[e], l[e]);
      const uint32_t o = tile_off(P.row[q], P.k[q]);
      *reinterpret_cast<uint4*>(hi + o) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(lo + o) = make_uint4(l[0], l[1], l[2], l[3]);
    }
  };
  bool ok = true;
  int64_t issued = 0;  // stages whose MMAs have been issued (the same in every thread)
  // one pipeline step: stage kt from registers (va, vb) into shared memory,
  // refill (va, vb) with stage kt + 2, hand stage kt to the tensor cores
  auto step = [&](int64_t kt, double (&va)[KH], double (&vb)[KH]) {
    const int s = static_cast<int>(kt % STAGES);
    uint8_t* st = tc_smem + s * STAGE;
    if (kt >= STAGES) ok = mbar_wait(smem_addr(&mbar[s]), static_cast<uint32_t>((kt / STAGES - 1) & 1));
    split_store(st, st + TILE_A, va, PA, BM);
    split_store(st + 2 * TILE_A, st + 2 * TILE_A + TILE_B, vb, PB, BN);
    if (kt + 2 < nk) load(kt + 2, va, vb);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    ok = __syncthreads_and(ok);
    if (!ok) return;
    issued = kt + 1;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a_hi = sbase + s * STAGE, a_lo = a_hi + TILE_A, b_hi = a_hi + 2 * TILE_A, b_lo = b_hi + TILE_B;
#pragma unroll
      for (int kk = 0; kk < BK / 8; ++kk) {
        const uint32_t off = kk * 2 * LBO;
        mma(tmem, desc(a_hi + off), desc(b_hi + off), idesc(BN), (kt > 0 || kk > 0) ? 1u : 0u);
        mma(tmem, desc(a_hi + off), desc(b_lo + off), idesc(BN), 1u);
        mma(tmem, desc(a_lo + off), desc(b_hi + off), idesc(BN), 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(&mbar[s]))
                   : "memory");
    }
  };
  load(0, ra0, rb0);
  if (nk > 1) load(1, ra1, rb1);
  for (int64_t kt = 0; kt < nk && ok; kt += 2) {
    step(kt, ra0, rb0);
    if (kt + 1 < nk && ok) step(kt + 1, ra1, rb1);
  }
  if (issued > 0) {  // the last commit covers every MMA issued before it; also waited for on failure
    const int s = static_cast<int>((issued - 1) % STAGES);
    ok = mbar_wait(smem_addr(&mbar[s]), static_cast<uint32_t>(((issued - 1) / STAGES) & 1)) && ok;
  }
  ok = __syncthreads_and(ok);
  if (ok) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // warp w reads TMEM lanes 32 (w % 4) ...; warps 0-3 take the first half of the columns, 4-7 the second
    const int quarter = warp & 3, half = warp >> 2;
    const int64_t m = m0 + quarter * 32 + lane;
#pragma unroll
    for (int cc = 0; cc < BN / 2; cc += 16) {
      const int c0 = half * (BN / 2) + cc;
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(tmem + (static_cast<uint32_t>(quarter * 32) << 16) + static_cast<uint32_t>(c0)));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m < d.M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int64_t n = n0 + c0 + j;
          if (n < d.N) {
            double* c = C + m * d.sCm + n * d.sCn;
            const double r = static_cast<double>(__uint_as_float(v[j]));
            *c = d.accumulate ? *c + r : r;
          }
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(&g_tc_fault, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS));
}

// ---------------------------------------------------------------------------
// 3xTF32 with TMA-fed operands.
//
// split_pack_kernel: an FP64 matrix view X(r, k) = X[r*s_r + k*s_k] becomes
// two FP32 arrays hi, lo of shape [rows_pad][kpad] (K contiguous, zero
// padding), x = hi + lo + O(2^-23 |x|).  32 x 32 tiles through shared memory
// keep both the read (along whichever stride is 1) and the write coalesced.
//
// gemm_tma_kernel: 128 threads.  Lane 0 of warp 0 streams the hi / lo tiles
// of A (128 rows x 32 K) and B (BN rows x 32 K) with cp.async.bulk.tensor
// into a three-stage ring (128-byte swizzle), each stage completing a "full"
// mbarrier by its transaction bytes; lane 0 of warp 1 issues, per stage,
// four K=8 steps x three tcgen05.mma (hi*hi, hi*lo, lo*hi) into the TMEM
// accumulator and commits them to the stage's "empty" mbarrier, which the
// producer waits on before refilling the slot; the last commit arrives on
// "done", after which all four warps move the accumulator out through
// tcgen05.ld (warp w: TMEM lanes 32w..32w+31) as FP64.  blockIdx.z selects
// a K chunk; with more than one chunk the CTA writes an FP64 partial tile.
// Waits are bounded (2 s); a timeout sets g_tc_fault and the CTA still
// releases its tensor memory after a bounded wait for its own MMAs.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) split_pack_kernel(const double* __restrict__ X, int64_t rows, int64_t K,
                                                         int64_t s_r, int64_t s_k, int64_t kpad,
                                                         float* __restrict__ hi, float* __restrict__ lo) {
  __shared__ double t[32][33];
  const int64_t k0 = static_cast<int64_t>(blockIdx.x) * 32, r0 = static_cast<int64_t>(blockIdx.y) * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const bool k_contig = (s_k == 1);
  for (int i = ty; i < 32; i += 8) {
    // element (r0 + a, k0 + b) with the thread index on the contiguous axis
    const int a = k_contig ? i : tx, b = k_contig ? tx : i;
    const int64_t r = r0 + a, k = k0 + b;
    t[a][b] = (r < rows && k < K) ? X[r * s_r + k * s_k] : 0.0;
  }
  __syncthreads();
  for (int i = ty; i < 32; i += 8) {
    uint32_t h, l;
    tc::split_tf32(t[i][tx], h, l);
    const int64_t o = (r0 + i) * kpad + k0 + tx;
    hi[o] = __uint_as_float(h);
    lo[o] = __uint_as_float(l);
  }
}

namespace tma {
constexpr int BM = 128, BK = 32, STAGES = 3, THREADS = 128;
constexpr uint32_t A_TILE = BM * BK * 4;  // 16 KB, one hi or lo tile
__device__ __forceinline__ bool wait(uint32_t bar, uint32_t parity) {
  const uint64_t t0 = tc::now_ns();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (tc::now_ns() - t0 > 2000000000ull) return false;
  }
}
// K-major operand tile with 128-byte swizzle: rows of 128 B, 8-row atoms
// 1024 B apart (SBO); the leading offset is unused for this layout (1)
__device__ __forceinline__ uint64_t desc_sw128(uint32_t addr) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFF) | (1ull << 16) | (static_cast<uint64_t>(1024 >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
}
__device__ __forceinline__ void load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      :
      : "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}
}  // namespace tma

struct TmaGemm {
  int64_t M, N;
  int ktiles_per_chunk, ktiles;  // K tiles of 32 per CTA chunk, in total
  double* C;                     // output (nchunks == 1) or partials [chunk][M][N]
  int64_t sCm, sCn;
  int nchunks;
  bool accumulate;
};

template <int BN>
__global__ void __launch_bounds__(tma::THREADS) gemm_tma_kernel(const __grid_constant__ CUtensorMap mAh,
                                                                const __grid_constant__ CUtensorMap mAl,
                                                                const __grid_constant__ CUtensorMap mBh,
                                                                const __grid_constant__ CUtensorMap mBl, TmaGemm g) {
  using namespace tma;
  constexpr uint32_t B_TILE = BN * BK * 4;
  constexpr uint32_t STAGE = 2 * A_TILE + 2 * B_TILE;
  constexpr uint32_t TX = STAGE;  // bytes each stage's four loads deliver
  constexpr int TCOLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : 128);
  extern __shared__ __align__(1024) uint8_t tma_smem[];
  __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], done;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN, chunk = blockIdx.z;
  const int kt0 = chunk * g.ktiles_per_chunk;
  const int nk = min(g.ktiles_per_chunk, g.ktiles - kt0);
  // 1024-byte aligned ring (the 128-byte swizzle repeats every 8 rows of 128 B)
  const uint32_t raw = tc::smem_addr(tma_smem);
  const uint32_t ring = (raw + 1023u) & ~1023u;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_addr(&tmem_slot)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 32) {
    for (int s = 0; s < STAGES; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc::smem_addr(&full[s])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc::smem_addr(&empty[s])));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc::smem_addr(&done)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;

  bool ok = true;
  int issued = 0;  // stages handed to the tensor cores (MMA thread only)
  if (tid == 0) {
    // producer
    for (int i = 0; i < nk && ok; ++i) {
      const int s = i % STAGES;
      if (i >= STAGES) ok = wait(tc::smem_addr(&empty[s]), static_cast<uint32_t>((i / STAGES - 1) & 1));
      if (!ok) break;
      const uint32_t st = ring + s * STAGE, bar = tc::smem_addr(&full[s]);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(TX) : "memory");
      const int x = (kt0 + i) * BK;
      load_2d(st, &mAh, bar, x, m0);
      load_2d(st + A_TILE, &mAl, bar, x, m0);
      load_2d(st + 2 * A_TILE, &mBh, bar, x, n0);
      load_2d(st + 2 * A_TILE + B_TILE, &mBl, bar, x, n0);
    }
  } else if (tid == 32) {
    // MMA issuer
    constexpr uint32_t id = tc::idesc(BN);
    for (int i = 0; i < nk && ok; ++i) {
      const int s = i % STAGES;
      ok = wait(tc::smem_addr(&full[s]), static_cast<uint32_t>((i / STAGES) & 1));
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a_hi = ring + s * STAGE, a_lo = a_hi + A_TILE, b_hi = a_hi + 2 * A_TILE, b_lo = b_hi + B_TILE;
#pragma unroll
      for (int kk = 0; kk < BK / 8; ++kk) {
        const uint32_t off = kk * 32;  // 8 TF32 values of a 128-byte swizzled row
        tc::mma(tmem, desc_sw128(a_hi + off), desc_sw128(b_hi + off), id, (i > 0 || kk > 0) ? 1u : 0u);
        tc::mma(tmem, desc_sw128(a_hi + off), desc_sw128(b_lo + off), id, 1u);
        tc::mma(tmem, desc_sw128(a_lo + off), desc_sw128(b_hi + off), id, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       tc::smem_addr(&empty[s]))
                   : "memory");
      issued = i + 1;
    }
    // "done" follows every issued MMA (also after a failure, so that the
    // other warps stop waiting)
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     tc::smem_addr(&done))
                 : "memory");
  }
  __syncwarp();
  const bool mma_done = wait(tc::smem_addr(&done), 0u);
  ok = __syncthreads_and(ok && mma_done && (nk > 0));
  if (ok) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int64_t m = m0 + warp * 32 + lane;
    double* out = g.nchunks > 1 ? g.C + static_cast<int64_t>(chunk) * g.M * g.N : g.C;
    const int64_t sm_ = g.nchunks > 1 ? g.N : g.sCm, sn_ = g.nchunks > 1 ? 1 : g.sCn;
    const bool acc = g.nchunks == 1 && g.accumulate;
    // C contiguous along n: each 32 x 16 block goes through a per-warp
    // staging tile in the (now idle) ring so that a warp's stores cover two
    // rows of 16 consecutive columns; contiguous along m (or neither), each
    // lane stores its own row, which is then the coalesced direction
    const bool by_rows = sn_ == 1 && sm_ != 1;
    double* stg = reinterpret_cast<double*>(tma_smem + (ring - raw)) + warp * 32 * 17;
#pragma unroll
    for (int c0 = 0; c0 < BN; c0 += 16) {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0)));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (by_rows) {
#pragma unroll
        for (int j = 0; j < 16; ++j) stg[lane * 17 + j] = static_cast<double>(__uint_as_float(v[j]));
        __syncwarp();
        const int col = lane & 15;
        const int64_t n = n0 + c0 + col;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int r = 2 * i + (lane >> 4);
          const int64_t mr = m0 + warp * 32 + r;
          if (mr < g.M && n < g.N) {
            double* c = out + mr * sm_ + n;
            const double x = stg[r * 17 + col];
            *c = acc ? *c + x : x;
          }
        }
        __syncwarp();
      } else if (m < g.M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int64_t n = n0 + c0 + j;
          if (n < g.N) {
            double* c = out + m * sm_ + n * sn_;
            const double r = static_cast<double>(__uint_as_float(v[j]));
            *c = acc ? *c + r : r;
          }
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(&g_tc_fault, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS));
  (void)issued;
}

// C[m*sCm + n*sCn] (+)= sum_p parts[p][m*N + n]  (split-K epilogue)
template <typename T>
__global__ void splitk_reduce_kernel(const T* __restrict__ parts, int nparts, int64_t M, int64_t N, T* C,
                                     int64_t sCm, int64_t sCn, bool accumulate) {
  const int64_t len = M * N;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < len;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    // partials summed in order p = 0, 1, ...; up to 16 of them are loaded
    // together first so that their loads are in flight at once
    double re = 0.0, im = 0.0;
    for (int p0 = 0; p0 < nparts; p0 += 16) {
      T v[16];
#pragma unroll
      for (int q = 0; q < 16; ++q)
        if (p0 + q < nparts) v[q] = parts[(p0 + q) * len + i];
#pragma unroll
      for (int q = 0; q < 16; ++q)
        if (p0 + q < nparts) {
          re += re_of(v[q]);
          im += im_of(v[q]);
        }
    }
    const int64_t m = i / N, n = i - m * N;
    T* c = C + m * sCm + n * sCn;
    if constexpr (is_cplx<T>::value) {
      if (accumulate) {
        re += c->x;
        im += c->y;
      }
      *c = make_double2(re, im);
    } else {
      if (accumulate) re += *c;
      *c = re;
    }
  }
}

// ---------------------------------------------------------------------------
// Permutation: one thread per output element, output-coalesced.
// ---------------------------------------------------------------------------
constexpr int kMaxRank = 16;  // N x M window boundaries reach rank 2 + 2 M + 4

struct PermParams {
  int rank;
  int64_t total;
  int64_t out_dims[kMaxRank];
  int64_t src_stride[kMaxRank];  // stride in `in` of output axis i
  bool conj;
};

template <typename T>
__global__ void permute_kernel(const T* __restrict__ in, T* __restrict__ out, PermParams p) {
  for (int64_t lin = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; lin < p.total;
       lin += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t rem = lin, off = 0;
    for (int i = p.rank - 1; i >= 0; --i) {
      const int64_t q = rem / p.out_dims[i];
      off += (rem - q * p.out_dims[i]) * p.src_stride[i];
      rem = q;
    }
    T v = in[off];
    out[lin] = p.conj ? conj_of(v) : v;
  }
}

// The same gather with 32-bit index arithmetic (total < 2^31), for
// permutations that keep the innermost axis innermost: consecutive threads
// read consecutive elements within each contiguous run.
struct PermParams32 {
  int rank;
  uint32_t total;
  uint32_t out_dims[kMaxRank];
  uint32_t src_stride[kMaxRank];
  bool conj;
};

// Permutations that keep the innermost axis: one thread copies a whole run
// of `run` contiguous elements (16-byte copies when aligned), the run's
// source offset decoded with multiplicative inverses instead of divisions
// (Granlund & Montgomery, PLDI 1994: q = (t + ((n - t) >> 1)) >> (l - 1),
// t = umulhi(m, n), l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1).
struct PermRunParams {
  int nouter;  // output axes outside the run, outermost first
  uint32_t run, nruns;
  uint32_t nchunks, cmagic, cshift;  // chunks of kRunChunk elements per run, and their inverse
  uint32_t dims[kMaxRank], magic[kMaxRank], shift[kMaxRank], src_stride[kMaxRank];
  bool conj, vec;
};
constexpr uint32_t kRunChunk = 8;  // elements one thread copies

__device__ __forceinline__ uint32_t div_magic(uint32_t n, uint32_t m, uint32_t l) {
  if (l == 0) return n;  // d == 1
  const uint32_t t = __umulhi(m, n);
  return (t + ((n - t) >> 1)) >> (l - 1);
}

// Permutations whose new innermost axis a sits directly before the old one
// b (extent nb < 16) in the input: every (na x nb) block is contiguous in
// the input and becomes nb runs of na contiguous elements in the output.
// Consecutive threads take consecutive groups of kBlkVec elements of a
// block (coalesced reads, several loads in flight per thread; the writes
// fill whole runs); the other axes index the blocks.
constexpr uint32_t kBlkVec = 4;  // consecutive block elements one thread moves (loads issued together)
struct PermBlockParams {
  int nbatch;
  uint32_t na, nb, blk, out_b, nblocks;
  uint32_t nq, q_magic, q_shift, nb_magic, nb_shift;  // nq = ceil(blk / kBlkVec) groups per block
  uint32_t bdims[kMaxRank], bmagic[kMaxRank], bshift[kMaxRank], bin[kMaxRank], bout[kMaxRank];
  bool conj;
};

template <typename T>
__global__ void permute_blocks_kernel(const T* __restrict__ in, T* __restrict__ out, PermBlockParams p) {
  const uint64_t items = static_cast<uint64_t>(p.nblocks) * p.nq;
  for (uint64_t it = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; it < items;
       it += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t u = div_magic(static_cast<uint32_t>(it), p.q_magic, p.q_shift);
    const uint32_t j0 = (static_cast<uint32_t>(it) - u * p.nq) * kBlkVec;
    uint32_t rem = u, ibase = 0, obase = 0;
    for (int i = p.nbatch - 1; i >= 0; --i) {
      const uint32_t q = div_magic(rem, p.bmagic[i], p.bshift[i]);
      const uint32_t idx = rem - q * p.bdims[i];
      ibase += idx * p.bin[i];
      obase += idx * p.bout[i];
      rem = q;
    }
    T v[kBlkVec];
#pragma unroll
    for (uint32_t e = 0; e < kBlkVec; ++e) v[e] = j0 + e < p.blk ? in[ibase + j0 + e] : zero_of<T>();
#pragma unroll
    for (uint32_t e = 0; e < kBlkVec; ++e) {
      const uint32_t j = j0 + e;
      if (j < p.blk) {
        const uint32_t ia = div_magic(j, p.nb_magic, p.nb_shift), ib = j - ia * p.nb;
        out[obase + ib * p.out_b + ia] = p.conj ? conj_of(v[e]) : v[e];
      }
    }
  }
}

template <typename T>
__global__ void permute_runs_kernel(const T* __restrict__ in, T* __restrict__ out, PermRunParams p) {
  const uint64_t items = static_cast<uint64_t>(p.nruns) * p.nchunks;
  for (uint64_t it = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; it < items;
       it += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    // item = (run u, chunk c): consecutive threads take consecutive chunks of a run
    const uint32_t u = div_magic(static_cast<uint32_t>(it), p.cmagic, p.cshift);
    const uint32_t c0 = (static_cast<uint32_t>(it) - u * p.nchunks) * kRunChunk;
    const uint32_t len = min(kRunChunk, p.run - c0);
    uint32_t rem = u, off = c0;
    for (int i = p.nouter - 1; i > 0; --i) {
      const uint32_t q = div_magic(rem, p.magic[i], p.shift[i]);
      off += (rem - q * p.dims[i]) * p.src_stride[i];
      rem = q;
    }
    off += rem * p.src_stride[0];
    const T* src = in + off;
    T* dst = out + static_cast<size_t>(u) * p.run + c0;
    if constexpr (!is_cplx<T>::value) {
      if (p.vec) {  // pairs of doubles (the run and the chunk are even)
        const double2* s2 = reinterpret_cast<const double2*>(src);
        double2* d2 = reinterpret_cast<double2*>(dst);
        for (uint32_t j = 0; j < len / 2; ++j) d2[j] = s2[j];
        continue;
      }
    }
    for (uint32_t j = 0; j < len; ++j) dst[j] = p.conj ? conj_of(src[j]) : src[j];
  }
}

template <typename T>
__global__ void permute32_kernel(const T* __restrict__ in, T* __restrict__ out, PermParams32 p) {
  for (uint32_t lin = blockIdx.x * blockDim.x + threadIdx.x; lin < p.total; lin += gridDim.x * blockDim.x) {
    uint32_t rem = lin, off = 0;
    for (int i = p.rank - 1; i > 0; --i) {
      const uint32_t q = rem / p.out_dims[i];
      off += (rem - q * p.out_dims[i]) * p.src_stride[i];
      rem = q;
    }
    off += rem * p.src_stride[0];
    const T v = in[off];
    out[lin] = p.conj ? conj_of(v) : v;
  }
}

// Permutations that move the innermost axis: batched 32 x 32 tile
// transposes through shared memory between input axis b (innermost in the
// input) and input axis a (innermost in the output), so that reads and
// writes are both coalesced.  The other axes index the batch of tiles.
struct TransParams {
  int nbatch_dims;
  uint32_t na, nb;                      // extents of axes a and b
  uint32_t in_a, out_b;                 // input stride of a, output stride of b
  uint32_t tiles_a, tiles_b, ntiles;    // tiles per batch entry, in total
  uint32_t bdims[kMaxRank];             // extents of the batch axes
  uint32_t bin[kMaxRank], bout[kMaxRank];  // their input / output strides
  bool conj;
};

template <typename T>
__global__ void __launch_bounds__(256) transpose_tiles_kernel(const T* __restrict__ in, T* __restrict__ out,
                                                              TransParams p) {
  __shared__ T tile[32][33];
  for (uint32_t t = blockIdx.x; t < p.ntiles; t += gridDim.x) {
    uint32_t rem = t / (p.tiles_a * p.tiles_b);
    const uint32_t tt = t - rem * (p.tiles_a * p.tiles_b);
    const uint32_t ta = tt / p.tiles_b, tb = tt - ta * p.tiles_b;
    uint32_t ibase = 0, obase = 0;
    for (int i = p.nbatch_dims - 1; i >= 0; --i) {
      const uint32_t q = rem / p.bdims[i];
      const uint32_t idx = rem - q * p.bdims[i];
      ibase += idx * p.bin[i];
      obase += idx * p.bout[i];
      rem = q;
    }
    const uint32_t a0 = ta * 32, b0 = tb * 32;
    const uint32_t tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
    for (uint32_t r = ty; r < 32; r += 8) {  // read rows of a, coalesced along b
      const uint32_t a = a0 + r, b = b0 + tx;
      if (a < p.na && b < p.nb) tile[r][tx] = in[ibase + a * p.in_a + b];
    }
    __syncthreads();
    for (uint32_t r = ty; r < 32; r += 8) {  // write rows of b, coalesced along a
      const uint32_t b = b0 + r, a = a0 + tx;
      if (a < p.na && b < p.nb) {
        const T v = tile[tx][r];
        out[obase + b * p.out_b + a] = p.conj ? conj_of(v) : v;
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// max |x| then x /= max
// ---------------------------------------------------------------------------
template <typename T>
__global__ void maxabs_kernel(const T* __restrict__ x, int64_t n, unsigned long long* out) {
  double m = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    m = fmax(m, abs_of(x[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double wmax[32];
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = (threadIdx.x < (blockDim.x >> 5)) ? wmax[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    // non-negative doubles order like their bit patterns
    if (threadIdx.x == 0) atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(m)));
  }
}

template <typename T>
__global__ void divide_kernel(const T* x, T* out, int64_t n, const unsigned long long* mx) {
  const double m = __longlong_as_double(static_cast<long long>(*mx));
  const double inv = 1.0 / m;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = mul_real(x[i], inv);
}

template <typename T>
__global__ void axpy_kernel(T* __restrict__ y, const T* __restrict__ x, double a, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if constexpr (is_cplx<T>::value) {
      y[i] = make_double2(y[i].x + a * x[i].x, y[i].y + a * x[i].y);
    } else {
      y[i] += a * x[i];
    }
  }
}

template <typename T>
__global__ void scale_kernel(T* __restrict__ x, int64_t n, double a) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    x[i] = mul_real(x[i], a);
}

template <typename T>
__global__ void scale_leg_kernel(T* __restrict__ x, int64_t outer, int64_t dim, int64_t inner,
                                 const double* __restrict__ v) {
  const int64_t n = outer * dim * inner;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t k = (i / inner) % dim;
    x[i] = mul_real(x[i], v[k]);
  }
}

template <typename T>
__global__ void fit_chi_kernel(const T* __restrict__ in, int64_t d1, int64_t d2, int64_t rest,
                               T* __restrict__ out, int64_t chi) {
  const int64_t n = chi * chi * rest;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i % rest;
    const int64_t b = (i / rest) % chi;
    const int64_t a = i / (rest * chi);
    out[i] = (a < d1 && b < d2) ? in[(a * d2 + b) * rest + r] : zero_of<T>();
  }
}

__global__ void truncation_kernel(const double* __restrict__ s, int64_t n, int chi_cap,
                                  double cutoff, double* __restrict__ sinv, int chi_out,
                                  int* cut_out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int cut = static_cast<int>(n < chi_cap ? n : chi_cap);
  const double denom = s[0];
  for (int i = 0; i < cut; ++i) {
    if (s[i] / denom > cutoff) {
      sinv[i] = 1.0 / sqrt(s[i]);
    } else {
      cut = i;
      break;
    }
  }
  for (int i = cut; i < chi_out; ++i) sinv[i] = 0.0;
  if (cut_out) *cut_out = cut;
}

template <typename T>
__global__ void scale_cols_kernel(const T* __restrict__ U, int64_t ldu, int64_t rows, int kc,
                                  const double* __restrict__ sinv, bool conj, T* __restrict__ out) {
  const int64_t n = rows * kc;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / kc;
    const int k = static_cast<int>(i - r * kc);
    T v = U[r * ldu + k];
    if (conj) v = conj_of(v);
    out[i] = mul_real(v, sinv[k]);
  }
}

// r[j] = || P1[:, j] - s[j] P2[:, j] ||_2, one block per column j of the
// column-major n-row panels P1, P2 (column j at j*n); fixed reduction order.
__device__ __forceinline__ double abs2_of(double x) { return x * x; }
__device__ __forceinline__ double abs2_of(cplx x) { return x.x * x.x + x.y * x.y; }
__device__ __forceinline__ double sub_scaled_abs2(double a, double s, double b) { return abs2_of(a - s * b); }
__device__ __forceinline__ double sub_scaled_abs2(cplx a, double s, cplx b) {
  return abs2_of(make_double2(a.x - s * b.x, a.y - s * b.y));
}

template <typename T>
__global__ void ritz_residual_kernel(const T* __restrict__ P1, const T* __restrict__ P2,
                                     const double* __restrict__ s, int64_t n, double* __restrict__ r) {
  const int j = blockIdx.x;
  const T* a = P1 + static_cast<int64_t>(j) * n;
  const T* b = P2 + static_cast<int64_t>(j) * n;
  const double sj = s[j];
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += sub_scaled_abs2(a[i], sj, b[i]);
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) r[j] = sqrt(v);
  }
}

template <typename T>
__global__ void scale_rows_kernel(const T* __restrict__ VT, int64_t ldv, int64_t cols, int kc,
                                  const double* __restrict__ sinv, bool conj, T* __restrict__ out) {
  const int64_t n = cols * kc;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t k = i / cols;
    const int64_t c = i - k * cols;
    T v = VT[k * ldv + c];
    if (conj) v = conj_of(v);
    out[i] = mul_real(v, sinv[k]);
  }
}

template <typename T>
__global__ void identity_kernel(T* __restrict__ out, int64_t e) {
  const int64_t n = e * e;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    out[i] = (i / e == i % e) ? one_of<T>() : zero_of<T>();
  }
}

// ---------------------------------------------------------------------------
// One-sided (Hestenes) Jacobi singular values, one CTA per n x n matrix.
// Columns live in shared memory (column-major); each warp orthogonalises
// disjoint column pairs of a round-robin schedule.  Converged when no pair of
// a sweep needed a rotation (|a_p^H a_q| <= n u sqrt(|a_p|^2 |a_q|^2)), or
// after 60 sweeps (the count is reported back).
// ---------------------------------------------------------------------------
// sum of |x|^2 over a shared-memory array (re [, im] planes), whole CTA
template <bool CPLX>
__device__ double block_sumsq(const double* re, const double* im, int len) {
  __shared__ double wsum[32];
  __shared__ double total;
  double a = 0.0;
  for (int i = threadIdx.x; i < len; i += blockDim.x) {
    a += re[i] * re[i];
    if constexpr (CPLX) a += im[i] * im[i];
  }
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x < 32) {
    double b = (threadIdx.x < (blockDim.x >> 5)) ? wsum[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) b += __shfl_xor_sync(0xffffffffu, b, o);
    if (threadIdx.x == 0) total = b;
  }
  __syncthreads();
  return total;
}

template <typename T, bool CPLX>
__global__ void __launch_bounds__(256) jacobi_spectrum_kernel(const T* const* mats, int n,
                                                                double* out, int* sweeps_used) {
  extern __shared__ double sm[];
  double* re = sm;                      // n*n column-major
  double* im = sm + (CPLX ? n * n : 0);  // n*n (complex only)
  double* nrm = sm + (CPLX ? 2 : 1) * n * n;  // n
  __shared__ int rotated;
  const T* M = mats[blockIdx.x];
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    const int r = idx / n, c = idx % n;  // row-major source
    const T v = M[idx];
    re[c * n + r] = re_of(v);
    if constexpr (CPLX) im[c * n + r] = im_of(v);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int np = n + (n & 1);
  const double tol = static_cast<double>(n) * 2.220446049250313e-16;
  const double small2 = tol * tol * block_sumsq<CPLX>(re, im, n * n);  // rounding-noise columns
  int sweep = 0;
  for (; sweep < 60; ++sweep) {
    if (threadIdx.x == 0) rotated = 0;
    __syncthreads();
    for (int rnd = 0; rnd < np - 1; ++rnd) {
      for (int pr = warp; pr < np / 2; pr += nw) {
        auto player = [&](int k) { return k == 0 ? 0 : ((k - 1 + rnd) % (np - 1)) + 1; };
        int p = player(pr), q = player(np - 1 - pr);
        if (p >= n || q >= n) continue;
        if (p > q) {
          int t = p;
          p = q;
          q = t;
        }
        double al = 0, be = 0, gr = 0, gi = 0;
        for (int r = lane; r < n; r += 32) {
          const double pr_ = re[p * n + r], qr_ = re[q * n + r];
          al += pr_ * pr_;
          be += qr_ * qr_;
          gr += pr_ * qr_;
          if constexpr (CPLX) {
            const double pi_ = im[p * n + r], qi_ = im[q * n + r];
            al += pi_ * pi_;
            be += qi_ * qi_;
            gr += pi_ * qi_;
            gi += pr_ * qi_ - pi_ * qr_;  // Im(conj(a_p) a_q)
          }
        }
        for (int o = 16; o > 0; o >>= 1) {
          al += __shfl_xor_sync(0xffffffffu, al, o);
          be += __shfl_xor_sync(0xffffffffu, be, o);
          gr += __shfl_xor_sync(0xffffffffu, gr, o);
          if constexpr (CPLX) gi += __shfl_xor_sync(0xffffffffu, gi, o);
        }
        const double g = CPLX ? hypot(gr, gi) : fabs(gr);
        if (g == 0.0 || al <= small2 || be <= small2 || g <= tol * sqrt(al * be)) continue;
        // phase e^{-i phi} with gamma = |gamma| e^{i phi}
        const double ph_r = CPLX ? gr / g : (gr >= 0 ? 1.0 : -1.0);
        const double ph_i = CPLX ? -gi / g : 0.0;
        const double zeta = (be - al) / (2.0 * g);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
        for (int r = lane; r < n; r += 32) {
          const double apr = re[p * n + r];
          const double api = CPLX ? im[p * n + r] : 0.0;
          const double aqr = re[q * n + r];
          const double aqi = CPLX ? im[q * n + r] : 0.0;
          // b_q = a_q * e^{-i phi}
          const double bqr = aqr * ph_r - aqi * ph_i;
          const double bqi = aqr * ph_i + aqi * ph_r;
          re[p * n + r] = c * apr - s * bqr;
          re[q * n + r] = s * apr + c * bqr;
          if constexpr (CPLX) {
            im[p * n + r] = c * api - s * bqi;
            im[q * n + r] = s * api + c * bqi;
          }
        }
        if (lane == 0) rotated = 1;
      }
      __syncthreads();
    }
    __syncthreads();
    const int any = rotated;
    __syncthreads();
    if (!any) break;
  }
  // column norms, normalised, sorted descending
  for (int c = warp; c < n; c += nw) {
    double a = 0;
    for (int r = lane; r < n; r += 32) {
      a += re[c * n + r] * re[c * n + r];
      if constexpr (CPLX) a += im[c * n + r] * im[c * n + r];
    }
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) nrm[c] = sqrt(a);
  }
  __syncthreads();
  __shared__ double tot;
  if (threadIdx.x < 32) {
    double a = 0;
    for (int c = lane; c < n; c += 32) a += nrm[c] * nrm[c];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) tot = sqrt(a);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    const double v = nrm[c];
    int pos = 0;
    for (int o = 0; o < n; ++o) {
      const double w = nrm[o];
      pos += (w > v) || (w == v && o < c);
    }
    out[static_cast<int64_t>(blockIdx.x) * n + pos] = tot > 0 ? v / tot : 0.0;
  }
  if (threadIdx.x == 0 && sweeps_used) sweeps_used[blockIdx.x] = sweep;
}

template <typename T>
__global__ void counter_normal_kernel(T* __restrict__ out, int64_t rows, int64_t cols, uint64_t key_re,
                                      uint64_t key_im) {
  const int64_t total = rows * cols;
  for (int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; n < total;
       n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = n / cols, j = n - i * cols;
    const double re = counter_gauss(static_cast<uint64_t>(n), key_re);
    T v;
    if constexpr (is_cplx<T>::value) {
      v = make_double2(re, counter_gauss(static_cast<uint64_t>(n), key_im));
    } else {
      v = re;
    }
    out[i + j * rows] = v;
  }
}

template <typename T>
__global__ void upper_to_rh_kernel(const T* __restrict__ acm, int64_t lda, int64_t k, T* __restrict__ out) {
  const int64_t total = k * k;
  for (int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; n < total;
       n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t a = n / k, b = n - a * k;  // out[a, b] = conj(R[b, a]), R upper
    out[n] = (b <= a) ? conj_of(acm[b + a * lda]) : zero_of<T>();
  }
}

// One-sided Jacobi SVD with vectors; see jacobi_svd() in kernels.cuh.
// Column pairs of a round-robin schedule are handled by groups of kJG lanes;
// lane gl of a group holds rows gl + kJG i (i < RPL) of the pair's two
// columns in registers for the round: one batch of loads, the dot product,
// the rotation and the update in registers, one batch of stores (the right
// vectors are loaded only for pairs that rotate).  Squared column norms are
// exact at the start of every sweep and updated with each rotation
// (alpha' = alpha - t g, beta' = beta + t g).
template <typename T, bool CPLX, int kJG, int RPL>
__global__ void __launch_bounds__(kJG == 16 ? 768 : 1024) jacobi_svd_kernel(const T* __restrict__ A, int n, T* __restrict__ U,
                                                          double* __restrict__ S, T* __restrict__ Wout,
                                                          const T* __restrict__ Winit) {
  extern __shared__ double sm[];
  const int nn = n * n;
  double* ar = sm;
  double* ai = sm + nn;                       // complex only
  double* wr = sm + (CPLX ? 2 : 1) * nn;
  double* wi = wr + nn;                       // complex only
  double* nrm = sm + (CPLX ? 4 : 2) * nn;     // n
  int* pos = reinterpret_cast<int*>(nrm + n);  // n
  __shared__ int rotated;
  for (int idx = threadIdx.x; idx < nn; idx += blockDim.x) {
    const int r = idx / n, c = idx % n;
    const T v = A[idx];
    ar[c * n + r] = re_of(v);
    const T w0 = Winit ? Winit[idx] : ((r == c) ? one_of<T>() : zero_of<T>());
    wr[c * n + r] = re_of(w0);
    if constexpr (CPLX) {
      ai[c * n + r] = im_of(v);
      wi[c * n + r] = im_of(w0);
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int np = n + (n & 1);
  const double tol = static_cast<double>(n) * 2.220446049250313e-16, tol2 = tol * tol;
  const double small2 = tol * tol * block_sumsq<CPLX>(ar, ai, nn);  // rounding-noise columns
  const int grp = lane / kJG, gl = lane % kJG;
  for (int sweep = 0; sweep < 60; ++sweep) {
    for (int c = warp; c < n; c += nw) {
      double a = 0;
      for (int r = lane; r < n; r += 32) {
        a += ar[c * n + r] * ar[c * n + r];
        if constexpr (CPLX) a += ai[c * n + r] * ai[c * n + r];
      }
      for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
      if (lane == 0) nrm[c] = a;
    }
    if (threadIdx.x == 0) rotated = 0;
    __syncthreads();
    for (int rnd = 0; rnd < np - 1; ++rnd) {
      for (int base = warp * (32 / kJG); base < np / 2; base += nw * (32 / kJG)) {
        const int pr = base + grp;
        // position kk of the round-robin circle (0 fixed, the others rotating)
        auto player = [&](int kk) {
          if (kk == 0) return 0;
          const int x = kk - 1 + rnd;  // < 2 (np - 1)
          return (x >= np - 1 ? x - (np - 1) : x) + 1;
        };
        int p = 0, q = 0;
        bool valid = pr < np / 2;
        if (valid) {
          p = player(pr);
          q = player(np - 1 - pr);
          valid = p < n && q < n;
          if (p > q) {
            const int t = p;
            p = q;
            q = t;
          }
        }
        double xp[RPL], xq[RPL], yp[CPLX ? RPL : 1], yq[CPLX ? RPL : 1];
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
          const int r = gl + i * kJG;
          const bool ok = valid && r < n;
          xp[i] = ok ? ar[p * n + r] : 0.0;
          xq[i] = ok ? ar[q * n + r] : 0.0;
          if constexpr (CPLX) {
            yp[i] = ok ? ai[p * n + r] : 0.0;
            yq[i] = ok ? ai[q * n + r] : 0.0;
          }
        }
        double gr = 0, gi = 0, gr2 = 0, gi2 = 0;  // two accumulators: shorter FP64 chains
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
          double& a = (i & 1) ? gr2 : gr;
          a = fma(xp[i], xq[i], a);
          if constexpr (CPLX) {
            double& b = (i & 1) ? gi2 : gi;
            a = fma(yp[i], yq[i], a);
            b = fma(xp[i], yq[i], b);
            b = fma(-yp[i], xq[i], b);
          }
        }
        gr += gr2;
        gi += gi2;
#pragma unroll
        for (int o = kJG / 2; o > 0; o >>= 1) {  // reduce within the lane group
          gr += __shfl_xor_sync(0xffffffffu, gr, o, kJG);
          if constexpr (CPLX) gi += __shfl_xor_sync(0xffffffffu, gi, o, kJG);
        }
        const double al = valid ? nrm[p] : 0.0, be = valid ? nrm[q] : 0.0;
        const double g = CPLX ? hypot(gr, gi) : fabs(gr);
        if (!valid || g == 0.0 || al <= small2 || be <= small2 || g * g <= tol2 * al * be) continue;
        // real: the right vectors of the pair, issued before the rotation
        // arithmetic; complex: loaded in the update (register budget)
        double vp[CPLX ? 1 : RPL], vq[CPLX ? 1 : RPL];
        if constexpr (!CPLX) {
#pragma unroll
          for (int i = 0; i < RPL; ++i) {
            const int r = gl + i * kJG;
            const bool ok = r < n;
            vp[i] = ok ? wr[p * n + r] : 0.0;
            vq[i] = ok ? wr[q * n + r] : 0.0;
          }
        }
        // b = phase * a_q with a_p . b = g > 0; the rotation that zeroes it has
        // t = sign(tau) 2g / (|tau| + sqrt(tau^2 + 4 g^2)), tau = beta - alpha
        // (the smaller root of t^2 + 2 zeta t - 1 = 0, zeta = tau / 2g), in
        // rsqrt steps only; c = 1 / sqrt(1 + t^2) keeps c^2 + s^2 = 1 to
        // rounding whatever the accuracy of t
        const double ph_r = CPLX ? gr / g : (gr >= 0 ? 1.0 : -1.0);
        const double ph_i = CPLX ? -gi / g : 0.0;
        const double tau = be - al;
        const double w = fma(tau, tau, 4.0 * g * g);
        const double den = fabs(tau) + w * rsqrt(w);
        const double rd = rsqrt(den);
        const double t = copysign(2.0 * g, tau) * (rd * rd);
        const double c = rsqrt(fma(t, t, 1.0)), s = c * t;
        const double sph = s * ph_r, cph = c * ph_r;
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
          const int r = gl + i * kJG;
          if (r < n) {
            if constexpr (CPLX) {
              const double bqr = xq[i] * ph_r - yq[i] * ph_i, bqi = xq[i] * ph_i + yq[i] * ph_r;
              ar[p * n + r] = c * xp[i] - s * bqr;
              ar[q * n + r] = s * xp[i] + c * bqr;
              ai[p * n + r] = c * yp[i] - s * bqi;
              ai[q * n + r] = s * yp[i] + c * bqi;
              const double vpr = wr[p * n + r], vqr = wr[q * n + r], vpi = wi[p * n + r], vqi = wi[q * n + r];
              const double dqr = vqr * ph_r - vqi * ph_i, dqi = vqr * ph_i + vqi * ph_r;
              wr[p * n + r] = c * vpr - s * dqr;
              wr[q * n + r] = s * vpr + c * dqr;
              wi[p * n + r] = c * vpi - s * dqi;
              wi[q * n + r] = s * vpi + c * dqi;
            } else {  // ph_r = +-1 folded into the coefficients (exact)
              ar[p * n + r] = c * xp[i] - sph * xq[i];
              ar[q * n + r] = s * xp[i] + cph * xq[i];
              wr[p * n + r] = c * vp[i] - sph * vq[i];
              wr[q * n + r] = s * vp[i] + cph * vq[i];
            }
          }
        }
        if (gl == 0) {
          nrm[p] = al - t * g;
          nrm[q] = be + t * g;
          rotated = 1;
        }
      }
      __syncthreads();
    }
    const int any = rotated;
    __syncthreads();
    if (!any) break;
  }
  for (int c = warp; c < n; c += nw) {
    double a = 0;
    for (int r = lane; r < n; r += 32) {
      a += ar[c * n + r] * ar[c * n + r];
      if constexpr (CPLX) a += ai[c * n + r] * ai[c * n + r];
    }
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) nrm[c] = sqrt(a);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    const double v = nrm[c];
    int p = 0;
    for (int o = 0; o < n; ++o) {
      const double w = nrm[o];
      p += (w > v) || (w == v && o < c);
    }
    pos[c] = p;
    S[p] = v;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < nn; idx += blockDim.x) {
    const int r = idx / n, c = idx % n;  // source column c -> output column pos[c]
    const double inv = nrm[c] > 0.0 ? 1.0 / nrm[c] : 0.0;
    const int64_t o = static_cast<int64_t>(r) * n + pos[c];
    if constexpr (CPLX) {
      U[o] = make_double2(ar[c * n + r] * inv, ai[c * n + r] * inv);
      Wout[o] = make_double2(wr[c * n + r], wi[c * n + r]);
    } else {
      U[o] = ar[c * n + r] * inv;
      Wout[o] = wr[c * n + r];
    }
  }
}

template <typename T>
__global__ void add_noise_kernel(T* __restrict__ x, int64_t len, double scale, uint64_t key_re, uint64_t key_im) {
  for (int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; n < len;
       n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    T v = x[n];
    if constexpr (is_cplx<T>::value) {
      v.x += scale * counter_unit_uniform(static_cast<uint64_t>(n), key_re);
      v.y += scale * counter_unit_uniform(static_cast<uint64_t>(n), key_im);
    } else {
      v += scale * counter_unit_uniform(static_cast<uint64_t>(n), key_re);
    }
    x[n] = v;
  }
}

template <typename T>
__global__ void sum_partials_kernel(const T* __restrict__ parts, int nparts, int64_t len, T* __restrict__ out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < len;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int p = 0; p < nparts; ++p) {
      const T v = parts[p * len + i];
      re += re_of(v);
      im += im_of(v);
    }
    if constexpr (is_cplx<T>::value) {
      out[i] = make_double2(re, im);
    } else {
      out[i] = re;
    }
  }
}


// Complex-or-real arithmetic for the blocked factorisation below.
__device__ __forceinline__ double vmul(double a, double b) { return a * b; }
__device__ __forceinline__ cplx vmul(cplx a, cplx b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double vadd(double a, double b) { return a + b; }
__device__ __forceinline__ cplx vadd(cplx a, cplx b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double vsub(double a, double b) { return a - b; }
__device__ __forceinline__ cplx vsub(cplx a, cplx b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double vneg(double a) { return -a; }
__device__ __forceinline__ cplx vneg(cplx a) { return make_double2(-a.x, -a.y); }
__device__ __forceinline__ double shfl_v(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }
__device__ __forceinline__ cplx shfl_v(cplx v, int src) {
  return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// Inverse Cholesky factor of an equilibrated (optionally shifted) Gram
// matrix summed from split-K partials, one CTA, blocked by 8: kp = k rounded up to 8,
// the padding being the identity.  Cholesky (upper, A' = R'^H R'), three
// barriers per 8-column block: warp 0 factors the 8 x 8 diagonal block in
// registers (lane c holds column c, rows exchanged by shuffles), one thread
// per column solves the block row R'_JK = R'_JJ^{-H} A'_JK, all threads
// update the trailing triangle.  Then R' is inverted in place, two barriers
// per block: warp 0 inverts the diagonal block, the column block above it
// becomes -X[0:j0, 0:j0] R'[0:j0, J] X_JJ.  Rinv = D X as before.  One copy
// of the matrix lives in shared memory (kp^2 values), plus an 8 x kp panel.
template <typename T, bool CPLX>
__global__ void __launch_bounds__(512) chol_rinv_blocked_kernel(const T* __restrict__ parts, int nparts, int k,
                                                                 double shift, T* __restrict__ Rinv, int* flag) {
  extern __shared__ __align__(16) unsigned char chol_smem[];
  const int kp = (k + 7) & ~7, nb = kp / 8;
  T* A = reinterpret_cast<T*>(chol_smem);  // kp x kp, row-major
  T* P = A + kp * kp;                      // panel, kp x 8
  double* d = reinterpret_cast<double*>(P + 8 * kp);
  double* dinv = d + kp;  // 1 / R'_ii
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int kk = k * k;
  for (int idx = tid; idx < kp * kp; idx += nt) {
    const int r = idx / kp, c = idx - r * kp;
    T v = (r == c) ? one_of<T>() : zero_of<T>();
    if (r < k && c < k) {
      v = zero_of<T>();
      for (int p = 0; p < nparts; ++p) v = vadd(v, parts[static_cast<int64_t>(p) * kk + r * k + c]);
    }
    A[idx] = v;
  }
  __syncthreads();
  for (int i = tid; i < kp; i += nt) {
    const double g = re_of(A[i * kp + i]);
    d[i] = (i < k && g > 0.0) ? 1.0 / sqrt(g) : 1.0;
  }
  __syncthreads();
  for (int idx = tid; idx < kp * kp; idx += nt) {
    const int r = idx / kp, c = idx - r * kp;
    if (r < k && c < k) {
      T v = mul_real(A[idx], d[r] * d[c]);
      if (r == c) v = vadd(v, mul_real(one_of<T>(), shift));
      A[idx] = v;
    }
  }
  __syncthreads();
  // ---- blocked Cholesky
  for (int J = 0; J < nb; ++J) {
    const int j0 = 8 * J;
    if (warp == 0) {
      const int c = lane & 7;
      T col[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) col[r] = (r <= c) ? A[(j0 + r) * kp + j0 + c] : zero_of<T>();
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        double p = __shfl_sync(0xffffffffu, re_of(col[j]), j);
        if (!(p > 0.0)) {
          if (lane == 0 && flag) atomicExch(flag, 1);
          p = 1.0;
        }
        const double inv = rsqrt(p);  // 1 / R'_jj, kept for the solves below
        if (lane == j) dinv[j0 + j] = inv;
        if (c >= j) col[j] = mul_real(col[j], inv);
#pragma unroll
        for (int r = j + 1; r < 8; ++r) {
          const T rjr = shfl_v(col[j], r);  // R'_{j0+j, j0+r}
          if (c >= r) col[r] = vsub(col[r], vmul(conj_of(rjr), col[j]));
        }
      }
      if (lane < 8) {
#pragma unroll
        for (int r = 0; r < 8; ++r)
          if (r <= c) A[(j0 + r) * kp + j0 + c] = col[r];
      }
    }
    __syncthreads();
    for (int c = j0 + 8 + tid; c < kp; c += nt) {  // block row: solve R'_JJ^H x = a
      T x[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) x[r] = A[(j0 + r) * kp + c];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
#pragma unroll
        for (int m = 0; m < r; ++m) x[r] = vsub(x[r], vmul(conj_of(A[(j0 + m) * kp + j0 + r]), x[m]));
        x[r] = mul_real(x[r], dinv[j0 + r]);
      }
#pragma unroll
      for (int r = 0; r < 8; ++r) A[(j0 + r) * kp + c] = x[r];
    }
    __syncthreads();
    const int n2 = kp - j0 - 8;
    for (int idx = tid; idx < n2 * n2; idx += nt) {  // trailing triangle
      const int r = j0 + 8 + idx / n2, c = j0 + 8 + idx % n2;
      if (c < r) continue;
      T acc = zero_of<T>();
#pragma unroll
      for (int m = 0; m < 8; ++m) acc = vadd(acc, vmul(conj_of(A[(j0 + m) * kp + r]), A[(j0 + m) * kp + c]));
      A[r * kp + c] = vsub(A[r * kp + c], acc);
    }
    __syncthreads();
  }
  // ---- in-place blocked inverse of the upper triangle
  for (int J = 0; J < nb; ++J) {
    const int j0 = 8 * J;
    // Y = X[0:j0, 0:j0] R'[0:j0, J]  (X upper, already inverted)
    for (int idx = tid; idx < j0 * 8; idx += nt) {
      const int i = idx >> 3, c = idx & 7;
      T acc = zero_of<T>();
      for (int m = i; m < j0; ++m) acc = vadd(acc, vmul(A[i * kp + m], A[m * kp + j0 + c]));
      P[idx] = acc;
    }
    if (warp == 0) {  // X_JJ = R'_JJ^{-1}: lane c solves R'_JJ x = e_c
      const int c = lane & 7;
      T x[8];
#pragma unroll
      for (int r = 7; r >= 0; --r) {
        T s = (r == c) ? one_of<T>() : zero_of<T>();
#pragma unroll
        for (int m = r + 1; m < 8; ++m)
          if (m <= c) s = vsub(s, vmul(A[(j0 + r) * kp + j0 + m], x[m]));
        x[r] = (r <= c) ? mul_real(s, dinv[j0 + r]) : zero_of<T>();
      }
      __syncwarp();
      if (lane < 8) {
#pragma unroll
        for (int r = 0; r < 8; ++r)
          if (r <= c) A[(j0 + r) * kp + j0 + c] = x[r];
      }
    }
    __syncthreads();
    // X[0:j0, J] = -Y X_JJ
    for (int idx = tid; idx < j0 * 8; idx += nt) {
      const int i = idx >> 3, c = idx & 7;
      T acc = zero_of<T>();
#pragma unroll
      for (int m = 0; m < 8; ++m)
        if (m <= c) acc = vadd(acc, vmul(P[i * 8 + m], A[(j0 + m) * kp + j0 + c]));
      A[i * kp + j0 + c] = vneg(acc);
    }
    __syncthreads();
  }
  for (int idx = tid; idx < kk; idx += nt) {  // Rinv = D X (upper)
    const int r = idx / k, c = idx - r * k;
    Rinv[idx] = (c >= r) ? mul_real(A[r * kp + c], d[r]) : zero_of<T>();
  }
}

__global__ void spectrum_distance_kernel(const double* a, const double* c, int count, int n,
                                         double* sig) {
  const int b = blockIdx.x;
  if (b >= count) return;
  double acc = 0;
  for (int i = threadIdx.x; i < n; i += 32) {
    const double d = a[static_cast<int64_t>(b) * n + i] - c[static_cast<int64_t>(b) * n + i];
    acc += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (threadIdx.x == 0) sig[b] = sqrt(acc);
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <int BN>
void launch_tc_bn(dim3 grid, const GemmParams<double>& gp, cudaStream_t st) {
  constexpr int bytes = tc::STAGES * (2 * tc::BM * tc::BK * 4 + 2 * BN * tc::BK * 4);
  ensure_dynamic_smem(reinterpret_cast<const void*>(gemm_tc_tf32x3_kernel<BN>), bytes);
  gemm_tc_tf32x3_kernel<BN><<<grid, tc::THREADS, bytes, st>>>(gp);
  TG_CHECK_LAUNCH();
  count_launch();
}

void launch_tc(int bn, dim3 grid, const GemmParams<double>& gp, cudaStream_t st) {
  switch (bn) {
    case 32: launch_tc_bn<32>(grid, gp, st); break;
    case 64: launch_tc_bn<64>(grid, gp, st); break;
    case 96: launch_tc_bn<96>(grid, gp, st); break;
    default: launch_tc_bn<128>(grid, gp, st); break;
  }
}

PFN_cuTensorMapEncodeTiled tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    TG_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (!p || q != cudaDriverEntryPointSuccess) fail(TG_E_CUDA, "cuTensorMapEncodeTiled is not available");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
  }
  return fn;
}

// 2D map over a [rows][kpad] FP32 array: boxes of 32 K x box_rows rows with
// the 128-byte swizzle the tcgen05 descriptors expect
CUtensorMap tf32_map(const float* base, int64_t rows, int64_t kpad, int box_rows) {
  CUtensorMap m;
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(kpad), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(kpad) * 4};
  cuuint32_t box[2] = {static_cast<cuuint32_t>(tma::BK), static_cast<cuuint32_t>(box_rows)};
  cuuint32_t estr[2] = {1, 1};
  const CUresult r = tensor_map_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims,
                                          strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                          CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(TG_E_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(static_cast<int>(r)) + ")");
  return m;
}

template <int BN>
void launch_tma_bn(dim3 grid, const CUtensorMap& ah, const CUtensorMap& al, const CUtensorMap& bh,
                   const CUtensorMap& bl, const TmaGemm& g, cudaStream_t st) {
  constexpr int bytes = tma::STAGES * (2 * tma::A_TILE + 2 * BN * tma::BK * 4) + 1024;
  ensure_dynamic_smem(reinterpret_cast<const void*>(gemm_tma_kernel<BN>), bytes);
  gemm_tma_kernel<BN><<<grid, tma::THREADS, bytes, st>>>(ah, al, bh, bl, g);
  TG_CHECK_LAUNCH();
  count_launch();
}

// C = A B for one real product: both operands split into padded hi / lo TF32
// arrays (split_pack_kernel), then the TMA-fed tcgen05 kernel over 128 x bn
// tiles; K chunks (<= 256 of K, enough of them to give every SM a CTA) are
// reduced in FP64, which keeps the FP32 accumulation error at the level of
// the dropped lo*lo term.
void gemm_tma(const double* A, const double* B, double* C, const GemmDesc& d, int bn, cudaStream_t st) {
  const int64_t kpad = (d.K + tma::BK - 1) / tma::BK * tma::BK, ktiles = kpad / tma::BK;
  const int64_t mpad = (d.M + tma::BM - 1) / tma::BM * tma::BM, npad = (d.N + bn - 1) / bn * bn;
  if (mpad / tma::BM > 65535 || ktiles > (int64_t{1} << 30)) fail(TG_E_INPUT, "gemm: problem too large");
  // operands split by the caller are used as they are; the others are split here
  auto usable = [&](const SplitOperand* s, int64_t rows, int64_t rows_pad_needed) {
    return s && s->hi && s->rows == rows && s->K == d.K && s->kpad == kpad && s->rows_pad >= rows_pad_needed;
  };
  const bool pa = usable(d.preA, d.M, mpad), pb = usable(d.preB, d.N, npad);
  void* sbuf = nullptr;
  const int64_t na = pa ? 0 : mpad * kpad, nbf = pb ? 0 : npad * kpad;
  if (na + nbf > 0) TG_CUDA(cudaMallocAsync(&sbuf, sizeof(float) * 2 * (na + nbf), st));
  float* ah = static_cast<float*>(sbuf);
  float* al = ah + na;
  float* bh = al + na;
  float* bl = bh + nbf;
  int64_t arows = mpad, brows = npad;
  if (pa) {
    ah = const_cast<float*>(d.preA->hi);
    al = const_cast<float*>(d.preA->lo);
    arows = d.preA->rows_pad;
  } else {
    split_pack_kernel<<<dim3(static_cast<unsigned>(kpad / 32), static_cast<unsigned>(mpad / 32)), 256, 0, st>>>(
        A, d.M, d.K, d.sAm, d.sAk, kpad, ah, al);
    TG_CHECK_LAUNCH();
    count_launch();
  }
  if (pb) {
    bh = const_cast<float*>(d.preB->hi);
    bl = const_cast<float*>(d.preB->lo);
    brows = d.preB->rows_pad;
  } else {
    split_pack_kernel<<<dim3(static_cast<unsigned>(kpad / 32), static_cast<unsigned>(npad / 32)), 256, 0, st>>>(
        B, d.N, d.K, d.sBn, d.sBk, kpad, bh, bl);
    TG_CHECK_LAUNCH();
    count_launch();
  }
  const CUtensorMap mah = tf32_map(ah, arows, kpad, tma::BM), mal = tf32_map(al, arows, kpad, tma::BM);
  const CUtensorMap mbh = tf32_map(bh, brows, kpad, bn), mbl = tf32_map(bl, brows, kpad, bn);
  const int64_t tiles = (mpad / tma::BM) * (npad / bn);
  int64_t nch = (ktiles + 7) / 8;  // FP32 accumulation over at most 256 of K
  if (tiles < 148) nch = std::max<int64_t>(nch, std::min<int64_t>((148 + tiles - 1) / tiles, ktiles / 8));
  nch = std::max<int64_t>(1, std::min<int64_t>(nch, ktiles));
  const int64_t per = (ktiles + nch - 1) / nch;
  nch = (ktiles + per - 1) / per;
  TmaGemm g{d.M, d.N, static_cast<int>(per), static_cast<int>(ktiles), C, d.sCm, d.sCn, static_cast<int>(nch),
            d.accumulate};
  void* pbuf = nullptr;
  if (nch > 1) {
    TG_CUDA(cudaMallocAsync(&pbuf, sizeof(double) * nch * d.M * d.N, st));
    g.C = static_cast<double*>(pbuf);
  }
  const dim3 grid(static_cast<unsigned>(npad / bn), static_cast<unsigned>(mpad / tma::BM), static_cast<unsigned>(nch));
  switch (bn) {
    case 32: launch_tma_bn<32>(grid, mah, mal, mbh, mbl, g, st); break;
    case 64: launch_tma_bn<64>(grid, mah, mal, mbh, mbl, g, st); break;
    case 96: launch_tma_bn<96>(grid, mah, mal, mbh, mbl, g, st); break;
    default: launch_tma_bn<128>(grid, mah, mal, mbh, mbl, g, st); break;
  }
  if (nch > 1) {
    splitk_reduce_kernel<double><<<num_blocks(d.M * d.N, 256), 256, 0, st>>>(
        static_cast<double*>(pbuf), static_cast<int>(nch), d.M, d.N, C, d.sCm, d.sCn, d.accumulate);
    TG_CHECK_LAUNCH();
    count_launch();
    TG_CUDA(cudaFreeAsync(pbuf, st));
  }
  if (sbuf) TG_CUDA(cudaFreeAsync(sbuf, st));
}

int64_t split_operand_floats(int64_t rows, int64_t K) {
  const int64_t kpad = (K + tma::BK - 1) / tma::BK * tma::BK, rpad = (rows + tma::BM - 1) / tma::BM * tma::BM;
  return 2 * rpad * kpad;
}

void split_operand(const double* X, int64_t rows, int64_t K, int64_t s_r, int64_t s_k, float* buf,
                   SplitOperand* out, cudaStream_t st) {
  const int64_t kpad = (K + tma::BK - 1) / tma::BK * tma::BK, rpad = (rows + tma::BM - 1) / tma::BM * tma::BM;
  ProfScope ps(PK_GEMM_TC, st, 0.0, 16.0 * static_cast<double>(rows) * K);
  split_pack_kernel<<<dim3(static_cast<unsigned>(kpad / 32), static_cast<unsigned>(rpad / 32)), 256, 0, st>>>(
      X, rows, K, s_r, s_k, kpad, buf, buf + rpad * kpad);
  TG_CHECK_LAUNCH();
  count_launch();
  out->hi = buf;
  out->lo = buf + rpad * kpad;
  out->rows = rows;
  out->K = K;
  out->rows_pad = rpad;
  out->kpad = kpad;
}

// 3xTF32 product on tcgen05 (real).  The longer of M and N goes on the
// 128-row side of the tile (C^T = B^T A^T when N > M); K is split so that
// the CTAs fill the GPU and FP32 accumulation runs over short K chunks, the
// chunks being summed in FP64 (256 of K for single products, 1024 for
// batched ones).  Single products take the TMA-fed kernel, batched ones the
// register-staged kernel.
void gemm_tc(const double* A, const double* B, double* C, GemmDesc d, cudaStream_t st) {
  if (d.N > d.M) {
    GemmDesc s = d;
    s.M = d.N;
    s.N = d.M;
    s.sAm = d.sBn;
    s.sAk = d.sBk;
    s.sBk = d.sAk;
    s.sBn = d.sAm;
    s.sCm = d.sCn;
    s.sCn = d.sCm;
    s.bA = d.bB;
    s.bB = d.bA;
    s.preA = d.preB;
    s.preB = d.preA;
    std::swap(A, B);
    d = s;
  }
  const int bn = d.N <= 32 ? 32 : d.N <= 64 ? 64 : d.N <= 96 ? 96 : 128;
  if (d.batch == 1) {
    gemm_tma(A, B, C, d, bn, st);
    return;
  }
  dim3 grid(static_cast<unsigned>((d.N + bn - 1) / bn), static_cast<unsigned>((d.M + tc::BM - 1) / tc::BM),
            static_cast<unsigned>(d.batch));
  if (grid.y > 65535) fail(TG_E_INPUT, "gemm: M too large");
  const int64_t tiles = static_cast<int64_t>(grid.x) * grid.y * grid.z;
  int64_t split = 1;
  if (d.batch == 1) {
    split = (d.K + 1023) / 1024;
    if (tiles < 296 && d.K >= 512)  // two CTAs per SM
      split = std::max<int64_t>(split, std::min<int64_t>((296 + tiles - 1) / tiles, d.K / 256));
  }
  if (split <= 1) {
    launch_tc(bn, grid, GemmParams<double>{A, B, C, d}, st);
    return;
  }
  const int64_t chunk = (d.K / split + tc::BK - 1) / tc::BK * tc::BK;
  const int64_t nfull = d.K / chunk, rem = d.K - nfull * chunk;
  const int64_t nparts = nfull + (rem > 0 ? 1 : 0);
  void* buf = nullptr;
  TG_CUDA(cudaMallocAsync(&buf, sizeof(double) * nparts * d.M * d.N, st));
  double* parts = static_cast<double*>(buf);
  GemmDesc g = d;
  g.sCm = d.N;
  g.sCn = 1;
  g.accumulate = false;
  g.K = chunk;
  g.batch = nfull;
  g.bA = chunk * d.sAk;
  g.bB = chunk * d.sBk;
  g.bC = d.M * d.N;
  launch_tc(bn, dim3(grid.x, grid.y, static_cast<unsigned>(nfull)), GemmParams<double>{A, B, parts, g}, st);
  if (rem > 0) {
    g.K = rem;
    g.batch = 1;
    launch_tc(bn, grid,
              GemmParams<double>{A + nfull * chunk * d.sAk, B + nfull * chunk * d.sBk, parts + nfull * d.M * d.N, g},
              st);
  }
  splitk_reduce_kernel<double><<<num_blocks(d.M * d.N, 256), 256, 0, st>>>(parts, static_cast<int>(nparts), d.M,
                                                                           d.N, C, d.sCm, d.sCn, d.accumulate);
  TG_CHECK_LAUNCH();
  count_launch();
  TG_CUDA(cudaFreeAsync(buf, st));
}

bool tc_fault_take() {
  int f = 0;
  TG_CUDA(cudaMemcpyFromSymbol(&f, g_tc_fault, sizeof(int)));
  if (f) {
    const int z = 0;
    TG_CUDA(cudaMemcpyToSymbol(g_tc_fault, &z, sizeof(int)));
  }
  return f != 0;
}

// Column-tile width of the narrow FP64 product for this shape, in fragments
// of 8 columns, or 0 for the 64 x 64 tile: real FP64 products with
// 64 < N <= 96, which two 64-wide tiles pad by 33-100%.  (At N <= 64 the
// narrow tile saved nothing measurable: 16.5 us either way at 20000 x 36 x
// 72, and 20.6 against 18.6 us at 1024 x 42 x 1024, whose short split-K
// chunks favour register staging.)
template <typename T>
int narrow_nf(const GemmDesc& d) {
  if (is_cplx<T>::value || d.prec != 0 || d.N <= GBN || d.N > 96) return 0;
  return static_cast<int>((d.N + 7) / 8);
}

template <int NF>
void launch_narrow_nf(dim3 gr, size_t smem, cudaStream_t st, const GemmParams<double>& gp) {
  ensure_dynamic_smem(reinterpret_cast<const void*>(gemm_narrow_kernel<NF>), smem);
  gemm_narrow_kernel<NF><<<gr, 128, smem, st>>>(gp);
}

void launch_narrow(int nf, dim3 gr, size_t smem, cudaStream_t st, const GemmParams<double>& gp) {
  switch (nf) {
    case 9: launch_narrow_nf<9>(gr, smem, st, gp); break;
    case 10: launch_narrow_nf<10>(gr, smem, st, gp); break;
    case 11: launch_narrow_nf<11>(gr, smem, st, gp); break;
    case 12: launch_narrow_nf<12>(gr, smem, st, gp); break;
    default: fail(TG_E_RUNTIME, "gemm: no narrow tile of " + std::to_string(nf) + " fragments");
  }
}

template <typename T>
void gemm(const T* A, const T* B, T* C, const GemmDesc& d, cudaStream_t st) {
  if (d.M <= 0 || d.N <= 0 || d.batch <= 0) return;
  if (d.K <= 0) fail(TG_E_INPUT, "gemm: K must be positive");
  constexpr bool CPLX = is_cplx<T>::value;
  if constexpr (!CPLX) {
    if (gemm_skinny(A, B, C, d, st)) return;
  }
  constexpr int NP = CPLX ? 2 : 1;
  // the narrow tile (one column tile of 8 nf columns) where N pads to fewer columns than 64-wide tiles
  const int nf = narrow_nf<T>(d);
  const size_t smem = nf > 0 ? sizeof(double) * NSTAGE * GBK * (GLD + 8 * nf + 4)
                             : sizeof(double) * 2 * 2 * NP * GBK * GLD;
  if (nf == 0) ensure_dynamic_smem(reinterpret_cast<const void*>(gemm_kernel<T, CPLX>), smem);
  if (d.batch > 65535) fail(TG_E_INPUT, "gemm: batch too large");
  // products taller than the grid's 65535 row tiles run as row chunks
  constexpr int64_t kRowsPerLaunch = int64_t(65535) * GBM;
  if (d.M > kRowsPerLaunch) {
    for (int64_t m0 = 0; m0 < d.M; m0 += kRowsPerLaunch) {
      GemmDesc part = d;
      part.M = std::min(kRowsPerLaunch, d.M - m0);
      gemm<T>(A + m0 * d.sAm, B, C + m0 * d.sCm, part, st);
    }
    return;
  }
  dim3 grid(nf > 0 ? 1u : static_cast<unsigned>((d.N + GBN - 1) / GBN),
            static_cast<unsigned>((d.M + GBM - 1) / GBM), static_cast<unsigned>(d.batch));
  const double macs = static_cast<double>(d.M) * d.N * d.K * d.batch;
  ProfScope ps(d.prec == 1 ? PK_GEMM_TC : PK_GEMM, st, (CPLX ? 8.0 : 2.0) * macs,
               sizeof(T) * static_cast<double>(d.batch) * (d.M * d.K + d.K * d.N + d.M * d.N));
  // Split-K for products whose output tiles cannot fill the 148 SMs (tall-
  // skinny rSVD panels): K is cut into equal chunks written to partial
  // buffers, then summed into C.
  if (CPLX && d.prec != 0) fail(TG_E_INPUT, "gemm: the 3xTF32 product is real-only");
  if constexpr (!CPLX) {
    if (d.prec == 1) {
      gemm_tc(A, B, C, d, st);
      return;
    }
  }
  auto launch = [&](dim3 gr, const GemmParams<T>& gp) {
    if constexpr (!CPLX) {
      if (nf > 0) {
        launch_narrow(nf, gr, smem, st, gp);
        return;
      }
    }
    gemm_kernel<T, CPLX><<<gr, 128, smem, st>>>(gp);
  };
  const int64_t tiles = static_cast<int64_t>(grid.x) * grid.y * grid.z;
  int64_t split = 1;
  // up to two CTAs per SM (the kernel's occupancy), K chunks of at least 128
  if (d.batch == 1 && tiles < 148 && d.K >= 256)
    split = std::min<int64_t>(std::max<int64_t>(1, 296 / tiles), (d.K + 127) / 128);
  if (split <= 1) {
    launch(grid, GemmParams<T>{A, B, C, d});
    TG_CHECK_LAUNCH();
    count_launch();
    return;
  }
  // all chunks in one launch (z = chunk, the last one possibly shorter), then an FP64 sum
  const int64_t chunk = (d.K + split - 1) / split;
  const int64_t chunk16 = (chunk + GBK - 1) / GBK * GBK;  // multiple of the k tile
  const int64_t nparts = (d.K + chunk16 - 1) / chunk16;
  void* buf = nullptr;
  TG_CUDA(cudaMallocAsync(&buf, sizeof(T) * nparts * d.M * d.N, st));
  T* parts = static_cast<T*>(buf);
  GemmDesc g = d;
  g.sCm = d.N;
  g.sCn = 1;
  g.accumulate = false;
  g.K = chunk16;
  g.klast = d.K - (nparts - 1) * chunk16;
  g.batch = nparts;
  g.bA = chunk16 * d.sAk;
  g.bB = chunk16 * d.sBk;
  g.bC = d.M * d.N;
  launch(dim3(grid.x, grid.y, static_cast<unsigned>(nparts)), GemmParams<T>{A, B, parts, g});
  TG_CHECK_LAUNCH();
  splitk_reduce_kernel<T><<<num_blocks(d.M * d.N, 256), 256, 0, st>>>(parts, static_cast<int>(nparts), d.M, d.N,
                                                                       C, d.sCm, d.sCn, d.accumulate);
  TG_CHECK_LAUNCH();
  count_launch(2);
  TG_CUDA(cudaFreeAsync(buf, st));
}

// ---- grouped products: launch of one tile variant, autotuner, entry point
namespace {
constexpr int kGroupVariants = 2;  // real: 64 x 64, 32 x 64; complex: 64 x 32, 32 x 32

template <typename T, int WFM, int WFN>
void launch_group_v(const GroupTab& tab, cudaStream_t st) {
  constexpr bool CPLX = is_cplx<T>::value;
  constexpr int BM = 16 * WFM, BN = 16 * WFN;
  constexpr int LDA = BM + (CPLX ? 2 : 4), LDB = BN + (CPLX ? 2 : 4);
  const size_t smem = sizeof(T) * NSTAGE * GBK * (LDA + LDB);
  const void* fn = reinterpret_cast<const void*>(gemm_group_kernel<T, WFM, WFN>);
  ensure_dynamic_smem(fn, smem);
  // resident CTAs per SM and SM count, per device
  static std::mutex mu;
  static std::map<int, int> slots;
  const int dev = current_device();
  int cap = 0;
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = slots.find(dev);
    if (it == slots.end()) {
      int occ = 0, sms = 0;
      TG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, gemm_group_kernel<T, WFM, WFN>, 128, smem));
      TG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      it = slots.emplace(dev, std::max(1, occ) * std::max(1, sms)).first;
    }
    cap = it->second;
  }
  const int grid = std::min(tab.total, cap);
  gemm_group_kernel<T, WFM, WFN><<<grid, 128, smem, st>>>(tab);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
constexpr int group_bm(int v) { return v == 0 ? 64 : 32; }
template <typename T>
constexpr int group_bn(int) { return is_cplx<T>::value ? 32 : 64; }

template <typename T>
void launch_group(int v, const GroupTab& tab, cudaStream_t st) {
  if constexpr (is_cplx<T>::value) {
    if (v == 0) launch_group_v<T, 4, 2>(tab, st);
    else launch_group_v<T, 2, 2>(tab, st);
  } else {
    if (v == 0) launch_group_v<T, 4, 4>(tab, st);
    else launch_group_v<T, 2, 4>(tab, st);
  }
}

// Work items of a group: every output tile of every problem, problems with
// long K and few tiles cut into K chunks (split-K, summed afterwards in chunk
// order) so that the group's work spreads over about four items per SM.  The
// chunks are sized from 64 x 64 tiles whatever the variant, so every variant
// sums each output element in the same order.  part_off receives each
// problem's offset into the partial-product buffer; returns its size in
// elements.
template <typename T>
int64_t fill_tab(const GroupItem* items, int n, int v, GroupTab& tab, std::vector<int64_t>& part_off) {
  const int bm = group_bm<T>(v), bn = group_bn<T>(v);
  double work = 0.0;  // k tiles over all 64 x 64 output tiles
  for (int i = 0; i < n; ++i) {
    const GroupItem& it = items[i];
    work += static_cast<double>((it.M + 63) / 64 * ((it.N + 63) / 64)) * ((it.K + GBK - 1) / GBK);
  }
  part_off.assign(static_cast<size_t>(n), -1);
  const int64_t chunk_kt = std::max<int64_t>(8, static_cast<int64_t>(std::ceil(work / (4.0 * 148))));
  tab.count = 0;
  tab.total = 0;
  int64_t part = 0;
  for (int i = 0; i < n; ++i) {
    const GroupItem& it = items[i];
    GroupTab::P& p = tab.p[tab.count++];
    p.A = it.A;
    p.B = it.B;
    p.C = it.C;
    p.part = nullptr;
    p.M = it.M;
    p.N = it.N;
    p.K = it.K;
    p.sAm = it.sAm;
    p.sAk = it.sAk;
    p.sBk = it.sBk;
    p.sBn = it.sBn;
    p.sCm = it.sCm;
    p.sCn = it.sCn;
    p.conjA = it.conjA;
    p.conjB = it.conjB;
    p.tn = static_cast<int>((it.N + bn - 1) / bn);
    const int64_t tiles = (it.M + bm - 1) / bm * p.tn;
    const int64_t kt = (it.K + GBK - 1) / GBK;
    int64_t ns = (kt + chunk_kt - 1) / chunk_kt;
    const int64_t ckt = (kt + ns - 1) / ns;  // k tiles of one chunk
    ns = (kt + ckt - 1) / ckt;
    p.kchunk = ckt * GBK;
    p.nsplit = static_cast<int>(ns);
    p.tiles = static_cast<int>(tiles);
    p.tile0 = tab.total;
    if (ns > 1) {
      part_off[static_cast<size_t>(i)] = part;
      part += ns * it.M * it.N;
    }
    if (tab.total + tiles * ns > INT32_MAX / 2) fail(TG_E_INPUT, "gemm_group: too many tiles");
    tab.total += static_cast<int>(tiles * ns);
  }
  return part;
}

// Runs variant v of the group: the product launch, then (if any problem was
// split) the reduction of the partial products into C.
template <typename T>
void run_group(const GroupItem* items, int n, int v, cudaStream_t st) {
  GroupTab tab;
  std::vector<int64_t> off;
  const int64_t part = fill_tab<T>(items, n, v, tab, off);
  void* buf = nullptr;
  if (part > 0) {
    TG_CUDA(cudaMallocAsync(&buf, sizeof(T) * part, st));
    for (int i = 0; i < tab.count; ++i)
      if (off[static_cast<size_t>(i)] >= 0) tab.p[i].part = static_cast<T*>(buf) + off[static_cast<size_t>(i)];
  }
  launch_group<T>(v, tab, st);
  if (part > 0) {
    GroupRed red;
    red.count = 0;
    red.total = 0;
    for (int i = 0; i < tab.count; ++i) {
      const GroupTab::P& p = tab.p[i];
      if (p.nsplit <= 1) continue;
      GroupRed::R& r = red.r[red.count++];
      r.part = p.part;
      r.C = p.C;
      r.M = p.M;
      r.N = p.N;
      r.sCm = p.sCm;
      r.sCn = p.sCn;
      r.nsplit = p.nsplit;
      r.elem0 = red.total;
      red.total += p.M * p.N;
    }
    group_reduce_kernel<T><<<num_blocks(red.total, 256), 256, 0, st>>>(red);
    TG_CHECK_LAUNCH();
    count_launch();
    TG_CUDA(cudaFreeAsync(buf, st));
  }
}

std::mutex g_tune_mu;
std::map<std::vector<int64_t>, int> g_tuned;  // group shape -> variant
int64_t g_tune_count = 0, g_tune_wins[kGroupVariants] = {};
}  // namespace

void gemm_group_stats(int64_t* tuned, int64_t* wins, int nwins) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  if (tuned) *tuned = g_tune_count;
  for (int v = 0; v < nwins && v < kGroupVariants; ++v) wins[v] = g_tune_wins[v];
}

template <typename T>
bool gemm_specialised(const GemmDesc& d) {
  if (is_cplx<T>::value || d.prec != 0 || d.batch != 1) return false;
  const bool skinny = d.K <= 96 && ((d.N <= 96 && d.M >= 2048) || (d.M <= 96 && d.N >= 2048));
  return skinny || narrow_nf<T>(d) > 0;
}

template <typename T>
void gemm_group(const GroupItem* items, int n, cudaStream_t st) {
  std::vector<GroupItem> live;
  for (int i = 0; i < n; ++i) {
    const GroupItem& it = items[i];
    if (it.M <= 0 || it.N <= 0) continue;
    if (it.K <= 0) fail(TG_E_INPUT, "gemm_group: K must be positive");
    if ((it.sAm != 1 && it.sAk != 1) || (it.sBk != 1 && it.sBn != 1))
      fail(TG_E_INPUT, "gemm_group: every operand needs a unit stride");
    live.push_back(it);
  }
  for (size_t off = 0; off < live.size(); off += kGroupMax) {
    const int cnt = static_cast<int>(std::min<size_t>(kGroupMax, live.size() - off));
    const GroupItem* its = live.data() + off;
    double flops = 0.0, bytes = 0.0;
    std::vector<int64_t> key{current_device(), is_cplx<T>::value ? 1 : 0};
    for (int i = 0; i < cnt; ++i) {
      const GroupItem& it = its[i];
      flops += (is_cplx<T>::value ? 8.0 : 2.0) * static_cast<double>(it.M) * it.N * it.K;
      bytes += sizeof(T) * static_cast<double>(it.M * it.K + it.K * it.N + it.M * it.N);
      key.insert(key.end(), {it.M, it.N, it.K, it.sAk == 1, it.sBn == 1, it.sCn == 1});
    }
    ProfScope ps(PK_GEMM, st, flops, bytes);
    int v = -1;
    {
      std::lock_guard<std::mutex> g(g_tune_mu);
      auto f = g_tuned.find(key);
      if (f != g_tuned.end()) v = f->second;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    TG_CUDA(cudaStreamIsCapturing(st, &cs));
    if (v < 0 && cs == cudaStreamCaptureStatusNone && !profile_enabled()) {
      // the autotuner: every variant once to warm up, then once timed (all
      // variants write the same result)
      float best = 0.0f;
      cudaEvent_t e0, e1;
      TG_CUDA(cudaEventCreate(&e0));
      TG_CUDA(cudaEventCreate(&e1));
      for (int c = 0; c < kGroupVariants; ++c) {
        run_group<T>(its, cnt, c, st);
        TG_CUDA(cudaEventRecord(e0, st));
        run_group<T>(its, cnt, c, st);
        TG_CUDA(cudaEventRecord(e1, st));
        TG_CUDA(cudaEventSynchronize(e1));
        float ms = 0.0f;
        TG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (v < 0 || ms < best) {
          v = c;
          best = ms;
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      std::lock_guard<std::mutex> g(g_tune_mu);
      g_tuned[key] = v;
      ++g_tune_count;
      ++g_tune_wins[v];
    }
    if (v < 0) v = 0;  // inside a capture before any eager call: the 64-row tile
    run_group<T>(its, cnt, v, st);
  }
}

template <typename T>
void permute(const T* in, T* out, const Shape& in_shape, const std::vector<int>& perm, bool conj,
             cudaStream_t st) {
  const int r = static_cast<int>(in_shape.size());
  if (r > kMaxRank) fail(TG_E_INPUT, "permute: rank > " + std::to_string(kMaxRank));
  const int64_t total = numel(in_shape);
  if (total == 0) return;
  ProfScope ps(PK_PERMUTE, st, 0.0, 2.0 * sizeof(T) * static_cast<double>(total));
  // Canonical form: drop unit axes, then merge input axes that stay adjacent
  // and in order in the output.
  std::vector<int> newax(static_cast<size_t>(r), -1);
  std::vector<int64_t> sh;
  for (int i = 0; i < r; ++i)
    if (in_shape[i] != 1) {
      newax[i] = static_cast<int>(sh.size());
      sh.push_back(in_shape[i]);
    }
  std::vector<int> pm;
  for (int i = 0; i < r; ++i)
    if (newax[perm[i]] >= 0) pm.push_back(newax[perm[i]]);
  std::vector<std::vector<int>> groups;  // runs of input axes, in output order
  for (int a : pm) {
    if (!groups.empty() && a == groups.back().back() + 1) groups.back().push_back(a);
    else groups.push_back({a});
  }
  std::vector<int> order(groups.size());  // groups sorted by their first input axis
  std::iota(order.begin(), order.end(), 0);
  std::sort(order.begin(), order.end(), [&](int x, int y) { return groups[x][0] < groups[y][0]; });
  const int m = static_cast<int>(groups.size());
  std::vector<int64_t> ms(static_cast<size_t>(m));  // merged input shape
  std::vector<int> rank_of(static_cast<size_t>(m));
  for (int q = 0; q < m; ++q) {
    int64_t e = 1;
    for (int a : groups[order[q]]) e *= sh[a];
    ms[q] = e;
    rank_of[order[q]] = q;
  }
  std::vector<int> mp(static_cast<size_t>(m));  // merged permutation
  for (int g = 0; g < m; ++g) mp[g] = rank_of[g];
  if (m <= 1) {  // a plain copy
    if (!conj) {
      TG_CUDA(cudaMemcpyAsync(out, in, sizeof(T) * static_cast<size_t>(total), cudaMemcpyDeviceToDevice, st));
      return;
    }
  }
  std::vector<int64_t> istr(static_cast<size_t>(std::max(m, 1))), od(static_cast<size_t>(std::max(m, 1))),
      ostr(static_cast<size_t>(std::max(m, 1)));
  std::vector<int> pos(static_cast<size_t>(std::max(m, 1)));
  {
    int64_t s = 1;
    for (int i = m - 1; i >= 0; --i) {
      istr[i] = s;
      s *= ms[i];
    }
    for (int i = 0; i < m; ++i) {
      od[i] = ms[mp[i]];
      pos[mp[i]] = i;
    }
    s = 1;
    for (int i = m - 1; i >= 0; --i) {
      ostr[i] = s;
      s *= od[i];
    }
  }
  if (total >= (int64_t{1} << 31)) {
    PermParams p{};
    p.rank = m;
    p.conj = conj;
    p.total = total;
    for (int i = 0; i < m; ++i) {
      p.out_dims[i] = od[i];
      p.src_stride[i] = istr[mp[i]];
    }
    permute_kernel<T><<<num_blocks(total, 256), 256, 0, st>>>(in, out, p);
    TG_CHECK_LAUNCH();
    count_launch();
    return;
  }
  const int a = m >= 1 ? mp[m - 1] : 0, b = m - 1;
  if (m >= 2 && a != b && ms[a] >= 16 && ms[b] >= 16) {
    TransParams p{};
    p.conj = conj;
    p.na = static_cast<uint32_t>(ms[a]);
    p.nb = static_cast<uint32_t>(ms[b]);
    p.in_a = static_cast<uint32_t>(istr[a]);
    p.out_b = static_cast<uint32_t>(ostr[pos[b]]);
    p.tiles_a = (p.na + 31) / 32;
    p.tiles_b = (p.nb + 31) / 32;
    uint64_t nt = static_cast<uint64_t>(p.tiles_a) * p.tiles_b;
    int nbd = 0;
    for (int d = 0; d < m; ++d) {
      if (d == a || d == b) continue;
      p.bdims[nbd] = static_cast<uint32_t>(ms[d]);
      p.bin[nbd] = static_cast<uint32_t>(istr[d]);
      p.bout[nbd] = static_cast<uint32_t>(ostr[pos[d]]);
      nt *= static_cast<uint64_t>(ms[d]);
      ++nbd;
    }
    p.nbatch_dims = nbd;
    p.ntiles = static_cast<uint32_t>(nt);
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(nt, 148 * 16));
    transpose_tiles_kernel<T><<<grid, 256, 0, st>>>(in, out, p);
    TG_CHECK_LAUNCH();
    count_launch();
    return;
  }
  auto magic_of = [](uint32_t d, uint32_t* mg, uint32_t* sh) {
    if (d <= 1) {
      *mg = 0;
      *sh = 0;
      return;
    }
    uint32_t l = 0;
    while ((uint64_t{1} << l) < d) ++l;  // ceil(log2 d)
    *mg = static_cast<uint32_t>((((uint64_t{1} << 32) * ((uint64_t{1} << l) - d)) / d) + 1);
    *sh = l;
  };
  if (m >= 2 && mp[m - 1] == m - 2 && ms[m - 1] < 16 && ms[m - 2] * ms[m - 1] <= 4096) {
    // the new innermost axis directly before the old one: contiguous blocks
    const int a = m - 2, b = m - 1;
    PermBlockParams p{};
    p.na = static_cast<uint32_t>(ms[a]);
    p.nb = static_cast<uint32_t>(ms[b]);
    p.blk = p.na * p.nb;
    p.out_b = static_cast<uint32_t>(ostr[pos[b]]);
    p.nblocks = static_cast<uint32_t>(total / p.blk);
    p.conj = conj;
    p.nq = (p.blk + kBlkVec - 1) / kBlkVec;
    magic_of(p.nq, &p.q_magic, &p.q_shift);
    magic_of(p.nb, &p.nb_magic, &p.nb_shift);
    int nbd = 0;
    for (int d = 0; d < m; ++d) {
      if (d == a || d == b) continue;
      p.bdims[nbd] = static_cast<uint32_t>(ms[d]);
      p.bin[nbd] = static_cast<uint32_t>(istr[d]);
      p.bout[nbd] = static_cast<uint32_t>(ostr[pos[d]]);
      magic_of(p.bdims[nbd], &p.bmagic[nbd], &p.bshift[nbd]);
      ++nbd;
    }
    p.nbatch = nbd;
    permute_blocks_kernel<T><<<num_blocks(static_cast<int64_t>(p.nblocks) * p.nq, 256, 148 * 16), 256, 0, st>>>(
        in, out, p);
    TG_CHECK_LAUNCH();
    count_launch();
    return;
  }
  if (m >= 2 && mp[m - 1] == m - 1) {  // the innermost axis stays innermost: copy runs
    PermRunParams p{};
    p.nouter = m - 1;
    p.run = static_cast<uint32_t>(ms[m - 1]);
    p.nruns = static_cast<uint32_t>(total / ms[m - 1]);
    p.nchunks = (p.run + kRunChunk - 1) / kRunChunk;
    magic_of(p.nchunks, &p.cmagic, &p.cshift);
    p.conj = conj;
    for (int i = 0; i < m - 1; ++i) {
      p.dims[i] = static_cast<uint32_t>(od[i]);
      p.src_stride[i] = static_cast<uint32_t>(istr[mp[i]]);
      magic_of(p.dims[i], &p.magic[i], &p.shift[i]);
    }
    // the outer strides are multiples of the run, so an even run keeps every run 16-byte aligned
    p.vec = !conj && (p.run % 2 == 0) && (reinterpret_cast<uintptr_t>(in) % 16 == 0) &&
            (reinterpret_cast<uintptr_t>(out) % 16 == 0);
    permute_runs_kernel<T><<<num_blocks(static_cast<int64_t>(p.nruns) * p.nchunks, 256, 148 * 16), 256, 0, st>>>(
        in, out, p);
    TG_CHECK_LAUNCH();
    count_launch();
    return;
  }
  PermParams32 p{};
  p.rank = std::max(m, 1);
  p.conj = conj;
  p.total = static_cast<uint32_t>(total);
  if (m == 0) {
    p.out_dims[0] = 1;
    p.src_stride[0] = 1;
  }
  for (int i = 0; i < m; ++i) {
    p.out_dims[i] = static_cast<uint32_t>(od[i]);
    p.src_stride[i] = static_cast<uint32_t>(istr[mp[i]]);
  }
  permute32_kernel<T><<<num_blocks(total, 256, 148 * 16), 256, 0, st>>>(in, out, p);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
void normalize_max_abs(const T* x, T* out, int64_t n, unsigned long long* scratch, cudaStream_t st) {
  ProfScope ps(PK_NORMALIZE, st, 0.0, 3.0 * sizeof(T) * static_cast<double>(n));
  TG_CUDA(cudaMemsetAsync(scratch, 0, sizeof(unsigned long long), st));
  const int nb = num_blocks(n, 256, 148 * 4);
  maxabs_kernel<T><<<nb, 256, 0, st>>>(x, n, scratch);
  TG_CHECK_LAUNCH();
  divide_kernel<T><<<num_blocks(n, 256), 256, 0, st>>>(x, out, n, scratch);
  TG_CHECK_LAUNCH();
  count_launch(2);
}

template <typename T>
void fit_chi(const T* in, int64_t d1, int64_t d2, int64_t rest, T* out, int64_t chi,
             cudaStream_t st) {
  fit_chi_kernel<T><<<num_blocks(chi * chi * rest, 256), 256, 0, st>>>(in, d1, d2, rest, out, chi);
  TG_CHECK_LAUNCH();
  count_launch();
}

void truncation(const double* s, int64_t n, int chi_cap, double cutoff, double* sinv, int chi_out,
                int* cut_out, cudaStream_t st) {
  truncation_kernel<<<1, 32, 0, st>>>(s, n, chi_cap, cutoff, sinv, chi_out, cut_out);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
void scale_cols(const T* U, int64_t ldu, int64_t rows, int kc, const double* sinv, bool conj,
                T* out, cudaStream_t st) {
  scale_cols_kernel<T><<<num_blocks(rows * kc, 256), 256, 0, st>>>(U, ldu, rows, kc, sinv, conj, out);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
void scale_rows(const T* VT, int64_t ldv, int64_t cols, int kc, const double* sinv, bool conj,
                T* out, cudaStream_t st) {
  scale_rows_kernel<T><<<num_blocks(cols * kc, 256), 256, 0, st>>>(VT, ldv, cols, kc, sinv, conj, out);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
void ritz_residual(const T* P1, const T* P2, const double* s, int64_t n, int w, double* r, cudaStream_t st) {
  if (w < 1) return;
  ritz_residual_kernel<T><<<w, 256, 0, st>>>(P1, P2, s, n, r);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
void identity(T* out, int64_t e, cudaStream_t st) {
  identity_kernel<T><<<num_blocks(e * e, 256), 256, 0, st>>>(out, e);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
void batched_spectrum(const T* const* mats, int count, int n, double* out, int* sweeps_used,
                      cudaStream_t st) {
  if (count <= 0) return;
  constexpr bool CPLX = is_cplx<T>::value;
  // the matrix lives in shared memory: n <= 160 (real), 112 (complex)
  const int nmax = CPLX ? 112 : 160;
  if (n > nmax || n < 1)
    fail(TG_E_INPUT, "batched_spectrum: 1 <= chi <= " + std::to_string(nmax) + " required");
  const size_t smem = sizeof(double) * ((CPLX ? 2 : 1) * n * n + n);
  ensure_dynamic_smem(reinterpret_cast<const void*>(jacobi_spectrum_kernel<T, CPLX>), smem);
  ProfScope ps(PK_SPECTRUM, st, 0.0, sizeof(T) * static_cast<double>(count) * n * n);
  jacobi_spectrum_kernel<T, CPLX><<<count, 256, smem, st>>>(mats, n, out, sweeps_used);
  TG_CHECK_LAUNCH();
  count_launch();
}

void spectrum_distance(const double* a, const double* c, int count, int n, double* sig,
                       cudaStream_t st) {
  if (count <= 0) return;
  spectrum_distance_kernel<<<count, 32, 0, st>>>(a, c, count, n, sig);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
void axpy(T* y, const T* x, double alpha, int64_t n, cudaStream_t st) {
  axpy_kernel<T><<<num_blocks(n, 256), 256, 0, st>>>(y, x, alpha, n);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
void scale(T* x, int64_t n, double alpha, cudaStream_t st) {
  scale_kernel<T><<<num_blocks(n, 256), 256, 0, st>>>(x, n, alpha);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
void scale_leg(T* x, int64_t outer, int64_t dim, int64_t inner, const double* v, cudaStream_t st) {
  scale_leg_kernel<T><<<num_blocks(outer * dim * inner, 256), 256, 0, st>>>(x, outer, dim, inner, v);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
void counter_normal(T* out, int64_t rows, int64_t cols, uint64_t seed, uint64_t stream, cudaStream_t st) {
  const uint64_t k_re = seed * 0x9E3779B97F4A7C15ull + stream * 0xBF58476D1CE4E5B9ull;
  const uint64_t k_im = seed * 0x9E3779B97F4A7C15ull + (stream + 1) * 0xBF58476D1CE4E5B9ull;
  counter_normal_kernel<T><<<num_blocks(rows * cols, 256), 256, 0, st>>>(out, rows, cols, k_re, k_im);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
void upper_to_rh(const T* acm, int64_t lda, int64_t k, T* out, cudaStream_t st) {
  upper_to_rh_kernel<T><<<num_blocks(k * k, 256), 256, 0, st>>>(acm, lda, k, out);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
int jacobi_svd_max_k() {
  // A and W (re [, im]) plus norms / positions must fit in 227 KB of smem
  return is_cplx<T>::value ? 84 : 119;
}

template <typename T>
void jacobi_svd(const T* A, int64_t k, T* U, double* S, T* W, cudaStream_t st, const T* Winit) {
  constexpr bool CPLX = is_cplx<T>::value;
  if (k < 1 || k > jacobi_svd_max_k<T>()) fail(TG_E_INPUT, "jacobi_svd: k out of range");
  const size_t smem = sizeof(double) * ((CPLX ? 4 : 2) * k * k + k) + sizeof(int) * k;
  ProfScope ps(PK_SOLVER, st, (CPLX ? 4.0 : 1.0) * 10.0 * static_cast<double>(k) * k * k, 0.0);
  const int npairs = static_cast<int>((k + 1) / 2);
  // up to 96 columns: 16 lanes a pair, 3, 4 or 6 rows a lane; up to 160: 32 lanes, 5 rows
  auto run = [&](auto kernel, int lanes) {
    ensure_dynamic_smem(reinterpret_cast<const void*>(kernel), smem);
    const int threads = static_cast<int>(std::min<int64_t>(1024, (static_cast<int64_t>(npairs) * lanes + 31) / 32 * 32));
    kernel<<<1, threads, smem, st>>>(A, static_cast<int>(k), U, S, W, Winit);
  };
  // rows a lane holds: the fewest that cover k (masked rows add exact zeros,
  // so the sums -- and the result -- are those of any larger choice)
  if (k <= 48)
    run(jacobi_svd_kernel<T, CPLX, 16, 3>, 16);
  else if (k <= 64)
    run(jacobi_svd_kernel<T, CPLX, 16, 4>, 16);
  else if (k <= 96)
    run(jacobi_svd_kernel<T, CPLX, 16, 6>, 16);
  else
    run(jacobi_svd_kernel<T, CPLX, 32, 5>, 32);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
void add_noise(T* x, int64_t len, double scale, uint64_t stream, cudaStream_t st) {
  const uint64_t k_re = noise_key_re(stream), k_im = noise_key_im(stream);
  add_noise_kernel<T><<<num_blocks(len, 256), 256, 0, st>>>(x, len, scale, k_re, k_im);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
void sum_partials(const T* parts, int nparts, int64_t len, T* out, cudaStream_t st) {
  sum_partials_kernel<T><<<num_blocks(len, 256), 256, 0, st>>>(parts, nparts, len, out);
  TG_CHECK_LAUNCH();
  count_launch();
}

template <typename T>
void chol_rinv(const T* parts, int nparts, int64_t k, int64_t n, int shift, T* Rinv, int* flag, cudaStream_t st) {
  constexpr bool CPLX = is_cplx<T>::value;
  if (k < 1 || k > jacobi_svd_max_k<T>()) fail(TG_E_INPUT, "chol_rinv: k out of range");
  const int64_t kp = (k + 7) / 8 * 8;
  const size_t smem = sizeof(T) * static_cast<size_t>(kp * kp + 8 * kp) + sizeof(double) * static_cast<size_t>(2 * kp);
  ensure_dynamic_smem(reinterpret_cast<const void*>(chol_rinv_blocked_kernel<T, CPLX>), smem);
  // shifted CholeskyQR (Fukaya et al., SIAM J. Sci. Comput. 42 (2020) A477):
  // s = 11 (m n + n (n+1)) u ||X||_2^2 with ||X||_2^2 <= k for unit columns
  const double u = 1.1102230246251565e-16;
  const double s = shift ? 11.0 * (static_cast<double>(n) * k + static_cast<double>(k) * (k + 1)) * u * k : 0.0;
  ProfScope ps(PK_SOLVER, st, (CPLX ? 4.0 : 1.0) * 2.0 * static_cast<double>(k) * k * k / 3.0, 0.0);
  chol_rinv_blocked_kernel<T, CPLX><<<1, 512, smem, st>>>(parts, nparts, static_cast<int>(k), s, Rinv, flag);
  TG_CHECK_LAUNCH();
  count_launch();
}

#define TG_INST(T)                                                                               \
  template void sum_partials<T>(const T*, int, int64_t, T*, cudaStream_t);                       \
  template void add_noise<T>(T*, int64_t, double, uint64_t, cudaStream_t);                    \
  template void chol_rinv<T>(const T*, int, int64_t, int64_t, int, T*, int*, cudaStream_t);        \
  template void counter_normal<T>(T*, int64_t, int64_t, uint64_t, uint64_t, cudaStream_t);       \
  template void upper_to_rh<T>(const T*, int64_t, int64_t, T*, cudaStream_t);                    \
  template int jacobi_svd_max_k<T>();                                                            \
  template void jacobi_svd<T>(const T*, int64_t, T*, double*, T*, cudaStream_t, const T*);       \
  template void gemm<T>(const T*, const T*, T*, const GemmDesc&, cudaStream_t);                  \
  template void gemm_group<T>(const GroupItem*, int, cudaStream_t);                             \
  template bool gemm_specialised<T>(const GemmDesc&);                                            \
  template void permute<T>(const T*, T*, const Shape&, const std::vector<int>&, bool,            \
                           cudaStream_t);                                                        \
  template void normalize_max_abs<T>(const T*, T*, int64_t, unsigned long long*, cudaStream_t);            \
  template void fit_chi<T>(const T*, int64_t, int64_t, int64_t, T*, int64_t, cudaStream_t);      \
  template void scale_cols<T>(const T*, int64_t, int64_t, int, const double*, bool, T*,          \
                              cudaStream_t);                                                     \
  template void scale_rows<T>(const T*, int64_t, int64_t, int, const double*, bool, T*,          \
                              cudaStream_t);                                                     \
  template void identity<T>(T*, int64_t, cudaStream_t);                                          \
  template void ritz_residual<T>(const T*, const T*, const double*, int64_t, int, double*, cudaStream_t); \
  template void batched_spectrum<T>(const T* const*, int, int, double*, int*, cudaStream_t);     \
  template void scale<T>(T*, int64_t, double, cudaStream_t);                                     \
  template void axpy<T>(T*, const T*, double, int64_t, cudaStream_t);                            \
  template void scale_leg<T>(T*, int64_t, int64_t, int64_t, const double*, cudaStream_t);

TG_INST(double)
TG_INST(cplx)

}  // namespace tg
