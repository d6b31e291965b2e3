// FP64 products with one small operand and one very long one: the
// contractions of an environment tensor with a corner or a site tensor that
// build the enlarged corners (rows chi * chi * D^2, the other sides <= 96).
//
// C (rows x n) = Big (rows x K) * Small (K x n), n, K <= 96: Small stays in
// shared memory, Big streams through in 64-row tiles (cp.async stages,
// persistent CTAs, two per SM where shared memory allows), eight warps each
// compute one 8-row block of the tile on DMMA m8n8k4 with the next k step's
// fragments loaded ahead of the current step's MMAs, and C is stored
// straight from the accumulator fragments.  A product whose left operand is
// the small one is taken as its transpose, C^T = B^T A^T.  At these shapes
// the DMMA rate and the HBM bandwidth bound the product about equally.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "kernels.cuh"

namespace tg {
namespace {

constexpr int SK_R = 64;         // rows of Big per tile
constexpr int SK_THREADS = 256;  // 8 warps, one 8-row block each
constexpr int SK_NMAX = 96;      // n and K at most this
constexpr size_t SK_SMEM_2CTA = 113 * 1024;  // two CTAs per SM at or below this

struct SkinnyParams {
  const double* big;  // element (r, k) at big[r * sr + k * sk], sr == 1 or sk == 1
  int64_t rows, sr, sk;
  const double* small;  // element (k, j) at small[k * ssk + j * ssn]
  int64_t ssk, ssn;
  double* C;  // element (r, j) at C[r * scr + j * scn]
  int64_t scr, scn;
  int K, n;
  bool accumulate;
  bool pairs;  // 16-byte copies of Big (its unit-stride runs start at even elements)
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
__device__ __forceinline__ void sk_cp16(double* dst, const double* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void sk_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void sk_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__host__ __device__ inline int sk_ld(int x) { return x + ((20 - (x & 15)) & 15); }  // = 4 (mod 16)

// A stage of Big holds the tile k-major (element (r, k) at k * SK_LDR + r)
// when Big is contiguous along its rows, row-major (r * ldb + k) when it is
// contiguous along K; either way the A-fragment loads are conflict-free.
constexpr int SK_LDR = SK_R + 4;

// NB = ceil(n / 8) column blocks, a template parameter so that the MMA
// loops carry no predicated-off work
template <int STAGES, int NB>
__global__ void __launch_bounds__(SK_THREADS, 2) skinny_kernel(SkinnyParams p) {
  extern __shared__ __align__(16) double sk_smem[];
  const int K = p.K, n = p.n;
  const int K4 = (K + 3) & ~3, n8 = NB * 8;
  const bool kmajor = p.sk != 1;  // Big contiguous along its rows
  const int ldb = sk_ld(K4), lds = sk_ld(n8);
  const int stage_len = kmajor ? K4 * SK_LDR : SK_R * ldb;
  double* S = sk_smem;        // K4 x lds
  double* Bt = S + K4 * lds;  // STAGES x stage_len
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  for (int idx = tid; idx < K4 * n8; idx += SK_THREADS) {
    const int k = idx / n8, j = idx - k * n8;
    S[k * lds + j] = (k < K && j < n) ? p.small[k * p.ssk + j * p.ssn] : 0.0;
  }
  const int64_t ntiles = (p.rows + SK_R - 1) / SK_R;
  const int my = ntiles > blockIdx.x ? static_cast<int>((ntiles - 1 - blockIdx.x) / gridDim.x + 1) : 0;
  auto row0 = [&](int i) { return (static_cast<int64_t>(blockIdx.x) + static_cast<int64_t>(i) * gridDim.x) * SK_R; };
  auto load_tile = [&](int i, int stage) {
    const int64_t r0 = row0(i);
    double* dst = Bt + stage * stage_len;
    const int nr = static_cast<int>(p.rows - r0 < SK_R ? p.rows - r0 : SK_R);
    if (kmajor) {  // K4 runs of SK_R consecutive rows
      const double* src = p.big + r0;
      if (p.pairs) {
        for (int idx = tid; idx < K4 * (SK_R / 2); idx += SK_THREADS) {
          const int k = idx >> 5, r = 2 * (idx & 31);
          double* d = dst + k * SK_LDR + r;
          if (k < K && r + 1 < nr) {
            sk_cp16(d, src + r + k * p.sk);
          } else {
            d[0] = (k < K && r < nr) ? src[r + k * p.sk] : 0.0;
            d[1] = 0.0;
          }
        }
      } else {
        for (int idx = tid; idx < K4 * SK_R; idx += SK_THREADS) {
          const int k = idx >> 6, r = idx & 63;
          double* d = dst + k * SK_LDR + r;
          if (k < K && r < nr)
            sk_cp8(d, src + r + k * p.sk);
          else
            *d = 0.0;
        }
      }
    } else {  // SK_R runs of K consecutive elements, one row per warp at a time
      const double* src = p.big + r0 * p.sr;
      for (int r = warp; r < SK_R; r += SK_THREADS / 32) {
        double* d = dst + r * ldb;
        const double* srow = src + r * p.sr;
        if (p.pairs) {
          for (int k = 2 * lane; k < K4; k += 64) {
            if (r < nr && k + 1 < K) {
              sk_cp16(d + k, srow + k);
            } else {
              d[k] = (r < nr && k < K) ? srow[k] : 0.0;
              d[k + 1] = 0.0;
            }
          }
        } else {
          for (int k = lane; k < K4; k += 32) {
            if (r < nr && k < K)
              sk_cp8(d + k, srow + k);
            else
              d[k] = 0.0;
          }
        }
      }
    }
  };
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < my) load_tile(s, s);
    sk_commit();
  }
  int stage = 0, pstage = STAGES - 1;
  const int astep = kmajor ? 4 * SK_LDR : 4;
#ifdef TG_SK_TRACE  // per-phase cycle counts for tuning builds (off in the library)
  long long ph[5] = {0, 0, 0, 0, 0}, tc = clock64();
#define SKT(q)                \
  {                           \
    long long c_ = clock64(); \
    ph[q] += c_ - tc;         \
    tc = c_;                  \
  }
#else
#define SKT(q)
#endif
  for (int i = 0; i < my; ++i) {
    if (i + STAGES - 1 < my) load_tile(i + STAGES - 1, pstage);
    pstage = pstage + 1 == STAGES ? 0 : pstage + 1;
    sk_commit();
    SKT(0)
    sk_wait<STAGES - 1>();
    __syncthreads();  // tile i (and, before the first, S) in shared memory
    SKT(1)
    const double* bst = Bt + stage * stage_len;
    stage = stage + 1 == STAGES ? 0 : stage + 1;
    double acc[NB][2];
#pragma unroll
    for (int c = 0; c < NB; ++c) acc[c][0] = acc[c][1] = 0.0;
    const double* ap = kmajor ? bst + t * SK_LDR + 8 * warp + g : bst + (8 * warp + g) * ldb + t;
    const double* sp = S + t * lds + g;
    // the fragments of the next k step are loaded before this step's MMAs
    double a0 = *ap, b0[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) b0[c] = sp[8 * c];
#pragma unroll 2
    for (int k4 = 0; k4 < K4; k4 += 4) {
      const bool more = k4 + 4 < K4;
      ap += astep;
      sp += 4 * lds;
      const double a1 = more ? *ap : 0.0;
      double b1[NB];
#pragma unroll
      for (int c = 0; c < NB; ++c) b1[c] = more ? sp[8 * c] : 0.0;
#pragma unroll
      for (int c = 0; c < NB; ++c) sk_dmma(acc[c][0], acc[c][1], a0, b0[c]);
      a0 = a1;
#pragma unroll
      for (int c = 0; c < NB; ++c) b0[c] = b1[c];
    }
    SKT(2)
    __syncthreads();  // every warp done with this stage before it is refilled
    SKT(3)
    // C straight from the accumulators: lane (g, t) holds row 8 warp + g,
    // columns 8 c + 2 t, +1; along either unit stride of C the 32 lanes
    // write whole 32-byte sectors
    const int64_t r = row0(i) + 8 * warp + g;
    if (r < p.rows) {
      double* crow = p.C + r * p.scr;
#pragma unroll
      for (int c = 0; c < NB; ++c) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int j = 8 * c + 2 * t + e;
          if (j < n) {
            double* dst = crow + j * p.scn;
            *dst = p.accumulate ? *dst + acc[c][e] : acc[c][e];
          }
        }
      }
    }
    SKT(4)
  }
#ifdef TG_SK_TRACE
  if (blockIdx.x == 0 && tid == 0 && my > 0)
    printf("skinny rows=%lld K=%d n=%d tiles=%d grid=%d cycles/tile: issue %lld wait %lld mma %lld sync %lld store %lld\n",
           (long long)p.rows, K, n, my, (int)gridDim.x, ph[0] / my, ph[1] / my, ph[2] / my, ph[3] / my, ph[4] / my);
#endif
#undef SKT
}

size_t skinny_smem(int K, int n, bool kmajor, int stages) {
  const int K4 = (K + 3) & ~3, n8 = (n + 7) & ~7;
  const size_t stage = kmajor ? static_cast<size_t>(K4) * SK_LDR : static_cast<size_t>(SK_R) * sk_ld(K4);
  return sizeof(double) * (static_cast<size_t>(K4) * sk_ld(n8) + stages * stage);
}

template <int STAGES, int NB>
void launch_skinny_nb(const SkinnyParams& p, size_t smem, cudaStream_t st) {
  ensure_dynamic_smem(reinterpret_cast<const void*>(skinny_kernel<STAGES, NB>), smem);
  const int64_t ntiles = (p.rows + SK_R - 1) / SK_R;
  const int per_sm = smem <= SK_SMEM_2CTA ? 2 : 1;
  const unsigned grid = static_cast<unsigned>(std::min<int64_t>(ntiles, 148 * per_sm));
  skinny_kernel<STAGES, NB><<<grid, SK_THREADS, smem, st>>>(p);
}

template <int STAGES>
void launch_skinny(const SkinnyParams& p, size_t smem, cudaStream_t st) {
  switch ((p.n + 7) / 8) {
    case 1: launch_skinny_nb<STAGES, 1>(p, smem, st); break;
    case 2: launch_skinny_nb<STAGES, 2>(p, smem, st); break;
    case 3: launch_skinny_nb<STAGES, 3>(p, smem, st); break;
    case 4: launch_skinny_nb<STAGES, 4>(p, smem, st); break;
    case 5: launch_skinny_nb<STAGES, 5>(p, smem, st); break;
    case 6: launch_skinny_nb<STAGES, 6>(p, smem, st); break;
    case 7: launch_skinny_nb<STAGES, 7>(p, smem, st); break;
    case 8: launch_skinny_nb<STAGES, 8>(p, smem, st); break;
    case 9: launch_skinny_nb<STAGES, 9>(p, smem, st); break;
    case 10: launch_skinny_nb<STAGES, 10>(p, smem, st); break;
    case 11: launch_skinny_nb<STAGES, 11>(p, smem, st); break;
    default: launch_skinny_nb<STAGES, 12>(p, smem, st); break;
  }
}

}  // namespace

bool gemm_skinny(const double* A, const double* B, double* C, const GemmDesc& d, cudaStream_t st) {
  if (d.batch != 1 || d.K < 1 || d.K > SK_NMAX) return false;
  SkinnyParams p{};
  p.K = static_cast<int>(d.K);
  p.accumulate = d.accumulate;
  constexpr int64_t kLong = 2048;
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
  const bool kmajor = p.sk != 1;
  // 16-byte copies: every unit-stride run of Big starts 16-byte aligned
  const int64_t lead = kmajor ? p.sk : p.sr;
  p.pairs = (reinterpret_cast<uintptr_t>(p.big) % 16 == 0) && (lead % 2 == 0);
  // three stages if two CTAs still fit on an SM, else two
  size_t smem = skinny_smem(p.K, p.n, kmajor, 3);
  const bool three = smem <= SK_SMEM_2CTA;
  if (!three) smem = skinny_smem(p.K, p.n, kmajor, 2);
  if (smem > 227 * 1024) return false;
  ProfScope ps(PK_GEMM, st, 2.0 * static_cast<double>(d.M) * d.N * d.K,
               sizeof(double) * static_cast<double>(d.M * d.K + d.K * d.N + d.M * d.N));
  if (three)
    launch_skinny<3>(p, smem, st);
  else
    launch_skinny<2>(p, smem, st);
  TG_CHECK_LAUNCH();
  count_launch();
  return true;
}

}  // namespace tg
