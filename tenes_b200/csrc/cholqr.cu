// Orthonormalisation of a tall FP64 panel by shifted CholeskyQR, every pass
// in one launch of one thread-block cluster.
//
// The panel Y (column-major n x k) is split into CS row ranges, one per CTA
// of a CS-CTA cluster (CS = 16 where the device allows it, else 8).  A pass is
//   1. Gram partial Y_c^H Y_c of the CTA's rows (upper 8 x 8 blocks, DMMA
//      m8n8k4 from a shared-memory copy of the rows);
//   2. a fixed-order sum of the CS partials over distributed shared memory,
//      each CTA summing one slice of the entries;
//   3. CTA 0 gathers the slices, equilibrates (D = diag(G)^-1/2), adds the
//      shift to the diagonal and factors D G D (+shift) = R'^H R' (blocked by
//      8), then inverts the 8 x 8 diagonal blocks of R';
//   4. every CTA copies R' and D from CTA 0;
//   5. every warp solves X R' = Y D for 8-row blocks of the CTA's rows
//      (blocked forward substitution: X_J = (Y_J D_J - sum_{I<J} X_I R'_IJ)
//      R'_JJ^{-1}, all products on DMMA), writing X over Y.
// After the first pass the counter-based perturbation of the engine's
// CholeskyQR (add_noise: same keys, same element counters) is added to the
// stored X.
// Cluster barriers order the phases; no CTA waits on anything else.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "counter_rng.cuh"
#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace tg {
namespace {

constexpr int CQ_THREADS = 256;  // 8 warps: up to 255 registers a thread
constexpr int CQ_WARPS = CQ_THREADS / 32;
constexpr int CQ_NBMAX = 12;  // k rounded up to 8 is at most 96
constexpr int CQ_KPMAX = 8 * CQ_NBMAX;
constexpr int CQ_RB = 176;          // rows of Y staged per chunk of the Gram phase
constexpr int CQ_LDY = CQ_RB + 4;   // 180 = 4 (mod 16): conflict-free fragment loads
constexpr int CQ_SLOTS = (CQ_NBMAX * (CQ_NBMAX + 1) / 2 + CQ_WARPS - 1) / CQ_WARPS;
constexpr int CQ_NU = 3;  // 8-row blocks a warp solves together

__device__ __forceinline__ void dmma_acc(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// accumulator fragment (row lane/4, columns 2(lane%4) + {0,1}) of an 8 x 8
// block -> the two A fragments (row lane/4, column 4 ks + lane%4) of its
// k-steps ks = 0, 1
__device__ __forceinline__ void acc_to_afrag(double c0, double c1, int lane, double& f0, double& f1) {
  const int src = (lane & ~3) + ((lane & 3) >> 1);
  const double v0 = __shfl_sync(0xffffffffu, c0, src), v1 = __shfl_sync(0xffffffffu, c1, src);
  const double w0 = __shfl_sync(0xffffffffu, c0, src + 2), w1 = __shfl_sync(0xffffffffu, c1, src + 2);
  f0 = (lane & 1) ? v1 : v0;
  f1 = (lane & 1) ? w1 : w0;
}

__device__ __forceinline__ int row_stride(int kp) { return kp + ((20 - (kp & 15)) & 15); }  // = 4 (mod 16)

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }


// Upper Cholesky factor of the kp x kp matrix A (row stride ld, upper
// triangle referenced) in place, blocked by 8.  For block J every warp that
// owns columns of the block row (or warp 0) factors the 8 x 8 diagonal block
// redundantly in registers -- each lane holds the whole upper triangle, so a
// pivot step is rsqrt -> scale -> update with no communication -- and applies
// the same steps to its own block-row column.  The trailing triangle is then
// updated on DMMA, two 8 x 8 blocks per warp task.  dinv[i] = 1/R'_ii.  At the
// end the diagonal blocks are replaced by their inverses (lower parts zero).
// btab lists the upper 8 x 8 blocks row by row, so the trailing blocks of
// block J are its suffix starting at (J+1) nb - J (J+1) / 2.
__device__ __forceinline__ void cholesky_blocked(double* A, int kp, int ld, double* dinv, const int* btab, int* flag) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const int nb = kp / 8, nblk = nb * (nb + 1) / 2;
  const int g = lane >> 2, t = lane & 3;
  for (int J = 0; J < nb; ++J) {
    const int j0 = 8 * J, ncol = kp - j0 - 8;
    double a[8][8];
    if (warp == 0 || warp * 32 < ncol) {
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = r; c < 8; ++c) a[r][c] = A[(j0 + r) * ld + j0 + c];
      const int col = j0 + 8 + warp * 32 + lane;
      const bool has = warp * 32 + lane < ncol;
      double p[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) p[r] = has ? A[(j0 + r) * ld + col] : 0.0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        double piv = a[j][j];
        if (!(piv > 0.0)) {
          if (tid == 0 && flag) atomicExch(flag, 1);
          piv = 1.0;
        }
        const double inv = rsqrt(piv);
        if (tid == 0) dinv[j0 + j] = inv;
        a[j][j] = piv * inv;
#pragma unroll
        for (int c = j + 1; c < 8; ++c) a[j][c] *= inv;
        p[j] *= inv;
#pragma unroll
        for (int r = j + 1; r < 8; ++r) {
#pragma unroll
          for (int c = r; c < 8; ++c) a[r][c] -= a[j][r] * a[j][c];
          p[r] -= a[j][r] * p[j];
        }
      }
      if (has) {  // each block-row column is read and written by its owner lane only
#pragma unroll
        for (int r = 0; r < 8; ++r) A[(j0 + r) * ld + col] = p[r];
      }
    }
    __syncthreads();  // every warp has loaded the diagonal block
    if (warp == 0 && lane < 8) {  // lane c writes column c of R'_JJ (no trailing block touches it)
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (c == lane) {
#pragma unroll
          for (int r = 0; r <= c; ++r) A[(j0 + r) * ld + j0 + c] = a[r][c];
        }
    }
    // trailing blocks (K, L), J < K <= L: A_KL -= R'_JK^H R'_JL
    for (int b = (J + 1) * nb - J * (J + 1) / 2 + warp; b < nblk; b += 2 * nw) {
      const bool two = b + nw < nblk;  // a second, independent block task
      const int bb0 = btab[b], bb1 = btab[two ? b + nw : b];
      const int K0 = bb0 >> 8, L0 = bb0 & 255, K1 = bb1 >> 8, L1 = bb1 & 255;
      double* cp0 = A + (8 * K0 + g) * ld + 8 * L0 + 2 * t;
      double* cp1 = A + (8 * K1 + g) * ld + 8 * L1 + 2 * t;
      double c0 = cp0[0], c1 = cp0[1], e0 = cp1[0], e1 = cp1[1];
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        const double* rowk = A + (j0 + 4 * ks + t) * ld + g;
        dmma_acc(c0, c1, -rowk[8 * K0], rowk[8 * L0]);
        dmma_acc(e0, e1, -rowk[8 * K1], rowk[8 * L1]);
      }
      cp0[0] = c0;
      cp0[1] = c1;
      if (two) {
        cp1[0] = e0;
        cp1[1] = e1;
      }
    }
    __syncthreads();
  }
  // diagonal blocks -> their inverses: warp J, lane c solves R'_JJ x = e_c
  for (int J = warp; J < nb; J += nw) {
    const int j0 = 8 * J, c = lane & 7;
    double x[8];
#pragma unroll
    for (int r = 7; r >= 0; --r) {
      double s = (r == c) ? 1.0 : 0.0;
#pragma unroll
      for (int m = r + 1; m < 8; ++m)
        if (m <= c) s -= A[(j0 + r) * ld + j0 + m] * x[m];
      x[r] = (r <= c) ? s * dinv[j0 + r] : 0.0;
    }
    __syncwarp();
    if (lane < 8) {
#pragma unroll
      for (int r = 0; r < 8; ++r) A[(j0 + r) * ld + j0 + c] = x[r];
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(CQ_THREADS, 1)
    cholqr_cluster_kernel(double* Y, double* scratch, int n, int k, int passes, int shifted, double shift,
                          double noise_scale, unsigned long long noise_key, int* flag) {
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = static_cast<int>(cluster.block_rank());
  const int cs = static_cast<int>(cluster.num_blocks());
  extern __shared__ __align__(16) double cq_smem[];
  const int kp = (k + 7) & ~7, nb = kp >> 3, ld = row_stride(kp);
  double* U = cq_smem;           // rows of Y / X, column by column (kp x CQ_LDY)
  double* Rs = U + kp * CQ_LDY;  // Gram partial, reduced slice, then R' with inverted diagonal blocks (kp x ld)
  double* ds = Rs + kp * ld;     // equilibration D
  double* dinv = ds + kp;        // 1 / R'_ii
  int* btab = reinterpret_cast<int*>(dinv + kp);  // (bi << 8) | bj of the upper 8 x 8 blocks
  const int nblk = nb * (nb + 1) / 2, total = nblk * 64;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    int q = 0;
    for (int bi = 0; bi < nb; ++bi)
      for (int bj = bi; bj < nb; ++bj) btab[q++] = (bi << 8) | bj;
  }
  auto entry = [&](int e) {  // element e of the upper blocks -> offset in a kp x ld matrix
    const int b = btab[e >> 6], w = e & 63;
    return ((b >> 8) * 8 + (w >> 3)) * ld + (b & 255) * 8 + (w & 7);
  };
  const int rows_per = ((n + cs - 1) / cs + 7) & ~7;
  const int r0 = min(n, rank * rows_per), r1 = min(n, r0 + rows_per);
  const int nch = (r1 - r0 + CQ_RB - 1) / CQ_RB;  // chunks of the CTA's rows
  const bool resident = nch <= 1;                 // the rows stay in shared memory across passes
  const int per = (total + cs - 1) / cs;          // entries summed by each CTA
  // rows [rc, rc + nr) of Y -> U, zero-padded to a multiple of 8 rows and to kp columns
  auto stage = [&](int rc, int nr) {
    const int nr8 = (nr + 7) & ~7;
    for (int idx = tid; idx < kp * nr8; idx += CQ_THREADS) {
      const int c = idx / nr8, r = idx - c * nr8;
      double* dst = U + c * CQ_LDY + r;
      if (r < nr && c < k)
        cp_async8(dst, Y + static_cast<size_t>(c) * n + rc + r);
      else
        *dst = 0.0;
    }
    cp_async_wait_all();
    __syncthreads();
  };
  auto unstage = [&](int rc, int nr) {
    for (int idx = tid; idx < k * nr; idx += CQ_THREADS) {
      const int c = idx / nr, r = idx - c * nr;
      Y[static_cast<size_t>(c) * n + rc + r] = U[c * CQ_LDY + r];
    }
  };
  __syncthreads();
  if (resident && nch == 1) stage(r0, r1 - r0);

  for (int pass = 0; pass < passes; ++pass) {
    // ---- 1. Gram partial of rows [r0, r1)
    double acc[CQ_SLOTS][2];
#pragma unroll
    for (int s = 0; s < CQ_SLOTS; ++s) acc[s][0] = acc[s][1] = 0.0;
    for (int ch = 0; ch < nch; ++ch) {
      const int rc = r0 + ch * CQ_RB, nr = min(CQ_RB, r1 - rc), nr8 = (nr + 7) & ~7;
      if (!resident) stage(rc, nr);
      int oa[CQ_SLOTS], ob[CQ_SLOTS];
#pragma unroll
      for (int s = 0; s < CQ_SLOTS; ++s) {
        const int b = warp + s * CQ_WARPS;
        const int bb = b < nblk ? btab[b] : 0;
        oa[s] = ((bb >> 8) * 8 + (lane >> 2)) * CQ_LDY + (lane & 3);
        ob[s] = ((bb & 255) * 8 + (lane >> 2)) * CQ_LDY + (lane & 3);
      }
      for (int r = 0; r < nr8; r += 4) {
#pragma unroll
        for (int s = 0; s < CQ_SLOTS; ++s)
          if (warp + s * CQ_WARPS < nblk) dmma_acc(acc[s][0], acc[s][1], U[oa[s] + r], U[ob[s] + r]);
      }
      if (!resident) __syncthreads();  // before the next chunk is staged
    }
    // CTA 0's R' of the previous pass is read by the others until here
    if (pass > 0) cluster.sync();
#pragma unroll
    for (int s = 0; s < CQ_SLOTS; ++s) {
      const int b = warp + s * CQ_WARPS;
      if (b < nblk) {
        const int bb = btab[b];
        const int row = (bb >> 8) * 8 + (lane >> 2), col = (bb & 255) * 8 + 2 * (lane & 3);
        Rs[row * ld + col] = acc[s][0];
        Rs[row * ld + col + 1] = acc[s][1];
      }
    }
    cluster.sync();
    // ---- 2. sum slice [e0, e1) of the entries over the cluster, in rank order
    {
      const int e0 = rank * per, e1 = min(total, e0 + per);
      for (int e = e0 + tid; e < e1; e += CQ_THREADS) {
        const int off = entry(e);
        double v = 0.0;
#pragma unroll
        for (int q = 0; q < 16; ++q)
          if (q < cs) v += cluster.map_shared_rank(Rs, q)[off];
        Rs[off] = v;
      }
    }
    cluster.sync();
    // ---- 3. CTA 0: gather, equilibrate, shift, factor
    if (rank == 0) {
#pragma unroll 4
      for (int e = tid; e < total; e += CQ_THREADS) {
        const int owner = e / per;
        if (owner != 0) {
          const int off = entry(e);
          Rs[off] = cluster.map_shared_rank(Rs, owner)[off];
        }
      }
      __syncthreads();
      for (int i = tid; i < kp; i += CQ_THREADS) {
        if (i >= k) Rs[i * ld + i] = 1.0;  // padding columns: identity
        const double g = Rs[i * ld + i];
        ds[i] = (i < k && g > 0.0) ? 1.0 / sqrt(g) : 1.0;
      }
      __syncthreads();
      for (int e = tid; e < total; e += CQ_THREADS) {
        const int b = btab[e >> 6], w = e & 63;
        const int r = (b >> 8) * 8 + (w >> 3), c = (b & 255) * 8 + (w & 7);
        if (r < k && c < k) {
          double v = Rs[r * ld + c] * (ds[r] * ds[c]);
          if (r == c && pass < shifted) v += shift;
          Rs[r * ld + c] = v;
        }
      }
      __syncthreads();
      cholesky_blocked(Rs, kp, ld, dinv, btab, flag);
      // R' and D to the global scratch, read from L2 by the other CTAs (a
      // broadcast from one SM's shared memory would serialise on that SM)
      for (int e = tid; e < total; e += CQ_THREADS) {
        const int off = entry(e);
        scratch[off] = Rs[off];
      }
      for (int i = tid; i < kp; i += CQ_THREADS) scratch[kp * ld + i] = ds[i];
      __threadfence();
    }
    cluster.sync();
    // ---- 4. R' and D from the scratch (L2 only: the lines change every pass)
    if (rank != 0) {
#pragma unroll 4
      for (int e = tid; e < total; e += CQ_THREADS) {
        const int off = entry(e);
        Rs[off] = __ldcg(scratch + off);
      }
      for (int i = tid; i < kp; i += CQ_THREADS) ds[i] = __ldcg(scratch + kp * ld + i);
      __syncthreads();
    }
    // ---- 5. X R' = Y D on 8-row blocks, X written over the rows in U
    const bool noisy = (pass == 0 && noise_scale != 0.0);
    for (int ch = 0; ch < nch; ++ch) {
      const int rc = r0 + ch * CQ_RB, nr = min(CQ_RB, r1 - rc), nr8 = (nr + 7) & ~7;
      if (!resident) stage(rc, nr);
      const int nrb = nr8 / 8;
      const int g = lane >> 2, t = lane & 3;
      for (int rb0 = warp; rb0 < nrb; rb0 += CQ_NU * CQ_WARPS) {
        // row blocks rb0 + u CQ_WARPS, u < CQ_NU: independent chains; an
        // absent block recomputes the rows of the first and stores nothing.
        // The solved blocks X_I are read back from U as A fragments.
        bool val[CQ_NU];
        int rb8[CQ_NU];
#pragma unroll
        for (int u = 0; u < CQ_NU; ++u) {
          val[u] = rb0 + u * CQ_WARPS < nrb;
          rb8[u] = (val[u] ? rb0 + u * CQ_WARPS : rb0) * 8 + g;
        }
#pragma unroll 1
        for (int J = 0; J < nb; ++J) {
          const int c0 = 8 * J + 2 * t;
          double a0[CQ_NU], a1[CQ_NU], b0[CQ_NU], b1[CQ_NU];
#pragma unroll
          for (int u = 0; u < CQ_NU; ++u) {
            a0[u] = U[c0 * CQ_LDY + rb8[u]] * ds[c0];
            a1[u] = U[(c0 + 1) * CQ_LDY + rb8[u]] * ds[c0 + 1];
            b0[u] = b1[u] = 0.0;
          }
          // a -= X_I R'_IJ over I < J, even I into a, odd I into b
#pragma unroll 1
          for (int I = 0; I < J; I += 2) {
            const bool odd = I + 1 < J;
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
              const int ra = 8 * I + 4 * ks + t, rb = ra + 8;
              const double bva = Rs[ra * ld + 8 * J + g];
              const double bvb = odd ? Rs[rb * ld + 8 * J + g] : 0.0;
#pragma unroll
              for (int u = 0; u < CQ_NU; ++u) {
                dmma_acc(a0[u], a1[u], -U[ra * CQ_LDY + rb8[u]], bva);
                if (odd) dmma_acc(b0[u], b1[u], -U[rb * CQ_LDY + rb8[u]], bvb);
              }
            }
          }
          const double d0 = Rs[(8 * J + t) * ld + 8 * J + g];
          const double d1 = Rs[(8 * J + 4 + t) * ld + 8 * J + g];
#pragma unroll
          for (int u = 0; u < CQ_NU; ++u) {
            double f0, f1;
            acc_to_afrag(a0[u] + b0[u], a1[u] + b1[u], lane, f0, f1);
            double x0 = 0.0, x1 = 0.0;
            dmma_acc(x0, x1, f0, d0);
            dmma_acc(x0, x1, f1, d1);
            if (val[u]) {
              U[c0 * CQ_LDY + rb8[u]] = x0;
              U[(c0 + 1) * CQ_LDY + rb8[u]] = x1;
            }
          }
          __syncwarp();  // X_J visible to the warp's later A-fragment loads
        }
      }
      if (noisy) {  // after the solve, which needs the unperturbed X
        __syncthreads();
        for (int idx = tid; idx < k * nr; idx += CQ_THREADS) {
          const int c = idx / nr, r = idx - c * nr;
          U[c * CQ_LDY + r] += noise_scale * counter_unit_uniform(static_cast<size_t>(c) * n + rc + r, noise_key);
        }
      }
      __syncthreads();
      if (!resident || pass == passes - 1) {
        unstage(rc, nr);
        if (!resident) __syncthreads();
      }
    }
  }
  cluster.sync();  // CTA 0's shared memory is read by the others until here
#undef CQ_T
}

size_t cholqr_smem_bytes(int kp) {
  const int ld = kp + ((20 - (kp & 15)) & 15);
  const int nb = kp / 8;
  return sizeof(double) * (static_cast<size_t>(kp) * CQ_LDY + static_cast<size_t>(kp) * ld + 2 * kp) +
         sizeof(int) * static_cast<size_t>(nb * (nb + 1) / 2);
}

// cluster size the current device runs this kernel with (16, else 8, else
// 0).  Both the attributes and the occupancy query belong to the current
// device's context, so the answer is probed and kept per device.
int probe_cluster_size() {
  const size_t smem = cholqr_smem_bytes(CQ_KPMAX);
  if (cudaFuncSetAttribute(cholqr_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem)) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaFuncSetAttribute(cholqr_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaGetLastError();
  for (int c : {16, 8}) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c);
    cfg.blockDim = dim3(CQ_THREADS);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = c;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, cholqr_cluster_kernel, &cfg) == cudaSuccess && nclusters > 0)
      return c;
    cudaGetLastError();
  }
  return 0;
}

int cholqr_cluster_size() {
  static std::mutex mu;
  static int cs[kMaxDevices];
  static bool probed[kMaxDevices] = {};
  const int dev = current_device();
  std::lock_guard<std::mutex> g(mu);
  if (!probed[dev]) {
    cs[dev] = probe_cluster_size();
    probed[dev] = true;
  }
  return cs[dev];
}

}  // namespace

bool cholqr_cluster_supported(int64_t n, int64_t k) {
  return k >= 1 && k <= CQ_KPMAX && n >= 1 && n * k < (int64_t(1) << 31) && cholqr_cluster_size() > 0;
}

int64_t cholqr_scratch_doubles(int64_t k) {
  const int64_t kp = (k + 7) / 8 * 8;
  return kp * (kp + ((20 - (kp & 15)) & 15)) + kp;
}

void cholqr_cluster(double* Y, int64_t n, int64_t k, int passes, int shifted_passes, uint64_t noise_stream,
                    double noise_scale, double* scratch, int* flag, cudaStream_t st) {
  if (!cholqr_cluster_supported(n, k)) fail(TG_E_INPUT, "cholqr_cluster: unsupported panel shape");
  const int cs = cholqr_cluster_size();
  const int kp = static_cast<int>((k + 7) / 8 * 8);
  const size_t smem = cholqr_smem_bytes(kp);
  // shifted CholeskyQR (Fukaya et al., SIAM J. Sci. Comput. 42 (2020) A477):
  // s = 11 (m n + n (n+1)) u ||X||_2^2 with ||X||_2^2 <= k for unit columns
  const double u = 1.1102230246251565e-16;
  const double s = 11.0 * (static_cast<double>(n) * k + static_cast<double>(k) * (k + 1)) * u * k;
  ProfScope ps(PK_SOLVER, st, passes * (2.0 * static_cast<double>(n) * k * k + k * k * k / 3.0), 0.0);
  {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(CQ_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    TG_CUDA(cudaLaunchKernelEx(&cfg, cholqr_cluster_kernel, Y, scratch, static_cast<int>(n), static_cast<int>(k), passes,
                               shifted_passes, s, noise_scale,
                               static_cast<unsigned long long>(noise_key_re(noise_stream)), flag));
    count_launch();
  }
}

}  // namespace tg
