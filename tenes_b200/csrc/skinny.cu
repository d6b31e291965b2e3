// FP64 products with one small operand and one very long one: the
// contractions of an environment tensor with a corner or a site tensor that
// build the enlarged corners (rows chi * chi * D^2, the other sides <= 96).
//
// C (rows x n) = Big (rows x K) * Small (K x n), n, K <= 96: Small stays in
// shared memory, Big streams through in 64-row tiles (three cp.async stages,
// persistent CTAs), eight warps each compute one 8-row block of the tile on
// DMMA m8n8k4, and the tile goes out through shared memory so that the
// stores run along C's unit stride.  A product whose left operand is the
// small one is taken as its transpose, C^T = B^T A^T.  At these shapes the
// DMMA rate and the HBM bandwidth bound the product about equally.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.cuh"

namespace tg {
namespace {

constexpr int SK_R = 64;         // rows of Big per tile
constexpr int SK_THREADS = 256;  // 8 warps, one 8-row block each
constexpr int SK_STAGES = 3;
constexpr int SK_NMAX = 96;      // n and K at most this
constexpr int SK_NB = SK_NMAX / 8;

struct SkinnyParams {
  const double* big;  // element (r, k) at big[r * sr + k * sk], sr == 1 or sk == 1
  int64_t rows, sr, sk;
  const double* small;  // element (k, j) at small[k * ssk + j * ssn]
  int64_t ssk, ssn;
  double* C;  // element (r, j) at C[r * scr + j * scn], scr == 1 or scn == 1
  int64_t scr, scn;
  int K, n;
  bool accumulate;
};

__device__ __forceinline__ void sk_dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}
__device__ __forceinline__ void sk_cp8(double* dst, const double* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void sk_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void sk_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__host__ __device__ inline int sk_ld(int x) { return x + ((20 - (x & 15)) & 15); }  // = 4 (mod 16)

__global__ void __launch_bounds__(SK_THREADS, 1) skinny_kernel(SkinnyParams p) {
  extern __shared__ __align__(16) double sk_smem[];
  const int K = p.K, n = p.n;
  const int K4 = (K + 3) & ~3, n8 = (n + 7) & ~7, nb = n8 >> 3;
  const int ldb = sk_ld(K4), lds = sk_ld(n8);
  double* S = sk_smem;                     // K4 x lds
  double* Bt = S + K4 * lds;               // SK_STAGES x SK_R x ldb
  double* Cs = Bt + SK_STAGES * SK_R * ldb;  // SK_R x lds
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  for (int idx = tid; idx < K4 * n8; idx += SK_THREADS) {
    const int k = idx / n8, j = idx - k * n8;
    S[k * lds + j] = (k < K && j < n) ? p.small[k * p.ssk + j * p.ssn] : 0.0;
  }
  const int64_t ntiles = (p.rows + SK_R - 1) / SK_R;
  const int64_t my = ntiles > blockIdx.x ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  auto tile_of = [&](int64_t i) { return blockIdx.x + i * gridDim.x; };
  auto load_tile = [&](int64_t tile, int stage) {
    const int64_t r0 = tile * SK_R;
    double* dst = Bt + stage * SK_R * ldb;
    if (p.sk == 1) {  // rows contiguous along K
      for (int r = warp; r < SK_R; r += SK_THREADS / 32)
        for (int k = lane; k < K4; k += 32) {
          if (r0 + r < p.rows && k < K)
            sk_cp8(dst + r * ldb + k, p.big + (r0 + r) * p.sr + k);
          else
            dst[r * ldb + k] = 0.0;
        }
    } else {  // contiguous along the rows
      for (int k = warp; k < K4; k += SK_THREADS / 32)
        for (int r = lane; r < SK_R; r += 32) {
          if (r0 + r < p.rows && k < K)
            sk_cp8(dst + r * ldb + k, p.big + (r0 + r) + k * p.sk);
          else
            dst[r * ldb + k] = 0.0;
        }
    }
  };
#pragma unroll
  for (int s = 0; s < SK_STAGES - 1; ++s) {
    if (s < my) load_tile(tile_of(s), s);
    sk_commit();
  }
  for (int64_t i = 0; i < my; ++i) {
    if (i + SK_STAGES - 1 < my) load_tile(tile_of(i + SK_STAGES - 1), static_cast<int>((i + SK_STAGES - 1) % SK_STAGES));
    sk_commit();
    sk_wait<SK_STAGES - 1>();
    __syncthreads();  // tile i (and, before the first, S) in shared memory
    const double* bs = Bt + static_cast<int>(i % SK_STAGES) * SK_R * ldb + (8 * warp + g) * ldb + t;
    double acc[SK_NB][2];
#pragma unroll
    for (int cb = 0; cb < SK_NB; ++cb) acc[cb][0] = acc[cb][1] = 0.0;
    for (int k4 = 0; k4 < K4; k4 += 4) {
      const double a = bs[k4];
      const double* sp = S + (k4 + t) * lds + g;
#pragma unroll
      for (int cb = 0; cb < SK_NB; ++cb)
        if (cb < nb) sk_dmma(acc[cb][0], acc[cb][1], a, sp[8 * cb]);
    }
#pragma unroll
    for (int cb = 0; cb < SK_NB; ++cb)
      if (cb < nb) {
        double* c = Cs + (8 * warp + g) * lds + 8 * cb + 2 * t;
        c[0] = acc[cb][0];
        c[1] = acc[cb][1];
      }
    __syncthreads();  // the tile's C block staged
    const int64_t r0 = tile_of(i) * SK_R;
    const int nr = static_cast<int>(p.rows - r0 < SK_R ? p.rows - r0 : SK_R);
    if (p.scn == 1) {  // C rows contiguous along n
      for (int r = warp; r < nr; r += SK_THREADS / 32)
        for (int j = lane; j < n; j += 32) {
          double* dst = p.C + (r0 + r) * p.scr + j;
          *dst = p.accumulate ? *dst + Cs[r * lds + j] : Cs[r * lds + j];
        }
    } else {  // contiguous along the rows
      for (int j = warp; j < n; j += SK_THREADS / 32)
        for (int r = lane; r < nr; r += 32) {
          double* dst = p.C + (r0 + r) + j * p.scn;
          *dst = p.accumulate ? *dst + Cs[r * lds + j] : Cs[r * lds + j];
        }
    }
    // the next iteration's barrier orders these reads of Cs before its rewrite
    // and every warp's reads of stage i % SK_STAGES before its refill
  }
}

size_t skinny_smem(int K, int n) {
  const int K4 = (K + 3) & ~3, n8 = (n + 7) & ~7;
  return sizeof(double) * (static_cast<size_t>(K4) * sk_ld(n8) + static_cast<size_t>(SK_STAGES) * SK_R * sk_ld(K4) +
                           static_cast<size_t>(SK_R) * sk_ld(n8));
}

}  // namespace

bool gemm_skinny(const double* A, const double* B, double* C, const GemmDesc& d, cudaStream_t st) {
  if (d.batch != 1 || d.K < 1 || d.K > SK_NMAX) return false;
  SkinnyParams p{};
  p.K = static_cast<int>(d.K);
  p.accumulate = d.accumulate;
  constexpr int64_t kLong = 4096;
  if (d.N <= SK_NMAX && d.M >= kLong) {  // C = A B, A the long operand
    p.big = A;
    p.rows = d.M;
    p.sr = d.sAm;
    p.sk = d.sAk;
    p.small = B;
    p.ssk = d.sBk;
    p.ssn = d.sBn;
    p.C = C;
    p.scr = d.sCm;
    p.scn = d.sCn;
    p.n = static_cast<int>(d.N);
  } else if (d.M <= SK_NMAX && d.N >= kLong) {  // C^T = B^T A^T, B the long operand
    p.big = B;
    p.rows = d.N;
    p.sr = d.sBn;
    p.sk = d.sBk;
    p.small = A;
    p.ssk = d.sAk;
    p.ssn = d.sAm;
    p.C = C;
    p.scr = d.sCn;
    p.scn = d.sCm;
    p.n = static_cast<int>(d.M);
  } else {
    return false;
  }
  if ((p.sr != 1 && p.sk != 1) || (p.scr != 1 && p.scn != 1)) return false;
  const size_t smem = skinny_smem(p.K, p.n);
  if (smem > 227 * 1024) return false;
  static size_t attr_bytes = 0;
  if (smem > attr_bytes) {
    TG_CUDA(cudaFuncSetAttribute(skinny_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    attr_bytes = smem;
  }
  ProfScope ps(PK_GEMM, st, 2.0 * static_cast<double>(d.M) * d.N * d.K,
               sizeof(double) * static_cast<double>(d.M * d.K + d.K * d.N + d.M * d.N));
  const int64_t ntiles = (p.rows + SK_R - 1) / SK_R;
  const unsigned grid = static_cast<unsigned>(std::min<int64_t>(ntiles, 148));
  skinny_kernel<<<grid, SK_THREADS, smem, st>>>(p);
  TG_CHECK_LAUNCH();
  count_launch();
  return true;
}

}  // namespace tg
