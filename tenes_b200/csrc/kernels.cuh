// Launchers of the hand-written sm_100a kernels used by the CTMRG driver.
#pragma once

#include "common.hpp"

namespace tg {

// An FP64 operand X(r, k) = X[r*s_r + k*s_k] split once into TF32 hi / lo
// arrays of shape [rows_pad][kpad] (rows padded to 128, K to 32), for
// operands that several 3xTF32 products share.
struct SplitOperand {
  const float* hi = nullptr;
  const float* lo = nullptr;
  int64_t rows = 0, K = 0, rows_pad = 0, kpad = 0;
};
// floats of buffer split_operand needs for rows x K
int64_t split_operand_floats(int64_t rows, int64_t K);
void split_operand(const double* X, int64_t rows, int64_t K, int64_t s_r, int64_t s_k, float* buf,
                   SplitOperand* out, cudaStream_t st);

// Strided batched matrix product C[b] (+)= op(A[b]) * op(B[b]) on the FP64
// tensor cores (DMMA m8n8k4).  Element (m,k) of A is A[m*sAm + k*sAk]; one of
// sAm / sAk must be 1 for coalesced tile loads, the other stride is free.
struct GemmDesc {
  int64_t M, N, K, batch;
  int64_t sAm, sAk, sBk, sBn, sCm, sCn;
  int64_t bA, bB, bC;
  bool conjA, conjB, accumulate;
  int prec = 0;  // 0: FP64 DMMA; 1: 3xTF32 on tcgen05, FP32 accumulation over K chunks <= 256
                 //    summed in FP64 (real only; conjugation flags are ignored)
  // prec 1, single products: already-split copies of A (rows M) / B (rows N, i.e. B^T), if any
  const SplitOperand* preA = nullptr;
  const SplitOperand* preB = nullptr;
  // FP64 product, > 0: the last batch entry contracts only klast of its K (split-K chunks of one launch)
  int64_t klast = 0;
};

template <typename T>
void gemm(const T* A, const T* B, T* C, const GemmDesc& d, cudaStream_t st);

// Grouped FP64 products: up to kGroupMax independent C_p = op(A_p) op(B_p)
// (batch 1, C overwritten) in ONE persistent launch whose CTAs take the
// output tiles of every problem in turn, so the products of all rows of a
// move share one wave instead of running one launch each.  Problems with
// long K and few output tiles are cut into K chunks whose partial products a
// second launch sums in chunk order.  Strides as in
// GemmDesc (one of each operand's strides 1).  Complex products run as three
// real DMMA products per tile (3M: Re = ArBr - AiBi, Im = (Ar+Ai)(Br+Bi) -
// ArBr - AiBi).  The tile shape is chosen per group by timing the candidate
// shapes once on the group's own operands (outside stream capture; cached
// per device and group shape); every candidate accumulates each output
// element in the same order, so the choice never changes a result.
constexpr int kGroupMax = 24;
struct GroupItem {
  const void* A = nullptr;
  const void* B = nullptr;
  void* C = nullptr;
  int64_t M = 0, N = 0, K = 0;
  int64_t sAm = 0, sAk = 0, sBk = 0, sBn = 0, sCm = 0, sCn = 0;
  bool conjA = false, conjB = false;
};
template <typename T>
void gemm_group(const GroupItem* items, int n, cudaStream_t st);
// autotuner record: groups tuned so far and, per tile variant, how often it won
void gemm_group_stats(int64_t* tuned, int64_t* wins, int nwins);
// True for a product that gemm() runs on a specialised kernel a grouped
// launch would do worse than: real FP64 shapes of the streaming kernel
// (skinny.cu: K <= 96, one side <= 96 and the other >= 2048) or of the
// narrow tile (64 < N <= 96).
template <typename T>
bool gemm_specialised(const GemmDesc& d);

// FP64 product with one operand of at most 96 x 96 and the other at least
// 2048 long (batch 1, a unit stride on the long operand and on C): the
// streaming kernel of skinny.cu.  Returns false, launching nothing, for any
// other shape.  gemm() tries it first at both precisions (it is exact FP64).
bool gemm_skinny(const double* A, const double* B, double* C, const GemmDesc& d, cudaStream_t st);

// True (and cleared) when a tcgen05 product gave up waiting for its tensor
// cores since the last call.  Synchronises the device.
bool tc_fault_take();

// out[i0..i_{r-1}] = in[...] with out.shape[i] = in.shape[perm[i]] (row-major),
// optionally conjugated.
template <typename T>
void permute(const T* in, T* out, const Shape& in_shape, const std::vector<int>& perm, bool conj,
             cudaStream_t st);

// out = x / max_i |x_i|  (the max_abs normalisation of ctm.cpp:514-517,
// 550-551); out may be x.  `scratch` holds one uint64 on the device.
template <typename T>
void normalize_max_abs(const T* x, T* out, int64_t n, unsigned long long* scratch, cudaStream_t st);

// out(chi, chi, r...) = zero-padded / sliced in(d1, d2, r...)  (extend / slice
// of the environment initialisation, ctm.cpp:998-1012).
template <typename T>
void fit_chi(const T* in, int64_t d1, int64_t d2, int64_t rest, T* out, int64_t chi,
             cudaStream_t st);

// Projector truncation (ctm.cpp:245-256, 275-288): given descending singular
// values s[0..n), keep cut = min(n, chi_cap) values, stopping at the first
// s_i / s_0 <= cutoff; sinv[k] = 1/sqrt(s_k) for k < cut, 0 for cut <= k < chi_out.
// cut is written to *cut_out (device int).
void truncation(const double* s, int64_t n, int chi_cap, double cutoff, double* sinv,
                int chi_out, int* cut_out, cudaStream_t st);

// U_c[i, k] = U[i*ldu + k] * sinv[k], k < kc (conj optional)  -> (rows x kc)
template <typename T>
void scale_cols(const T* U, int64_t ldu, int64_t rows, int kc, const double* sinv, bool conj,
                T* out, cudaStream_t st);
// VT_c[k, j] = VT[k*ldv + j] * sinv[k], k < kc  -> (kc x cols)
template <typename T>
void scale_rows(const T* VT, int64_t ldv, int64_t cols, int kc, const double* sinv, bool conj,
                T* out, cudaStream_t st);

// Residuals of a Rayleigh-Ritz check: r[j] = || P1[:, j] - s[j] P2[:, j] ||_2
// for j < w, with P1, P2 column-major n-row panels (column j at j*n).
template <typename T>
void ritz_residual(const T* P1, const T* P2, const double* s, int64_t n, int w, double* r, cudaStream_t st);

// One simple-update bond step (core::Simple_update_bond) in one thread
// block, in place on the two site tensors; the weights of every (site, leg)
// are read from and the new bond weights written to the device table
// lam[(site * 4 + leg) * lam_ld + j].  *flag is set to 1 (tensors and
// weights left unchanged) if Theta's Jacobi SVD does not converge.
struct SuBondArgs {
  void* tn1;
  void* tn2;
  double* lam;
  int lam_ld;
  int site1, site2, connect1;
  int dims1[5], dims2[5];  // (l, u, r, b, p) of the two tensors
  const void* op;          // op12 (d1, d2, d1, d2), row-major
  double lambda_cut;       // Inverse_lambda_cut
  int* flag;
};
template <typename T>
bool su_bond_fused_supported(const int* dims1, const int* dims2, int connect1, int lam_ld);
template <typename T>
void su_bond_fused(const SuBondArgs& a, cudaStream_t st);
// Bond steps on pairwise disjoint site pairs (they commute: none reads a
// weight or a tensor another writes), one thread block each, in one launch.
constexpr int kSuBatchMax = 16;
struct SuBondBatch {
  SuBondArgs a[kSuBatchMax];
};
template <typename T>
void su_bonds_fused(const SuBondArgs* a, int n, cudaStream_t st);

// Identity projector reshaped to (e, 1, 1, e) (ctm.cpp:303-317).
template <typename T>
void identity(T* out, int64_t e, cudaStream_t st);

// Batched L2-normalised singular values of `count` n x n matrices by one-sided
// Jacobi (one CTA per matrix, matrix resident in shared memory).  Values are
// written descending to out[b*n + i].  n <= 160 (real), 112 (complex).
template <typename T>
void batched_spectrum(const T* const* mats, int count, int n, double* out, int* sweeps_used,
                      cudaStream_t st);

// sig[b] = || a[b*n : (b+1)*n] - c[b*n : (b+1)*n] ||_2
void spectrum_distance(const double* a, const double* c, int count, int n, double* sig,
                       cudaStream_t st);

// Counter-based standard normals (splitmix64 hash + Box-Muller) in a
// column-major rows x cols array: element (i, j) uses counters 2n, 2n+1 of the
// row-major index n = i*cols + j under key (seed, stream); complex arrays take
// their imaginary parts from stream + 1.  The CPU oracle draws the same numbers.
template <typename T>
void counter_normal(T* out_colmajor, int64_t rows, int64_t cols, uint64_t seed, uint64_t stream,
                    cudaStream_t st);

// out (row-major k x k) = R^H, R = upper triangle of the first k rows of the
// column-major factored matrix `acm` (leading dimension lda) left by geqrf.
template <typename T>
void upper_to_rh(const T* acm, int64_t lda, int64_t k, T* out, cudaStream_t st);

// SVD of one row-major k x k matrix by one-sided Jacobi with accumulated
// right vectors, in one CTA with A and W resident in shared memory:
// A W = U S, singular values descending.  U, W written row-major (k x k,
// column j = j-th singular vector), S (k).  k <= jacobi_svd_max_k<T>().
// With Winit the accumulated rotations start from Winit instead of the
// identity: pass A = B Winit (Winit unitary) and the result is the SVD of B,
// B W = U S -- a warm start when Winit already nearly diagonalises B.
template <typename T>
void jacobi_svd(const T* A, int64_t k, T* U, double* S, T* W, cudaStream_t st, const T* Winit = nullptr);
template <typename T>
int jacobi_svd_max_k();

// x[i] += scale * u_i, u_i counter-based uniform numbers of mean 0 and
// variance 1 (key derived from `stream`; complex entries get independent real
// and imaginary parts)
template <typename T>
void add_noise(T* x, int64_t len, double scale, uint64_t stream, cudaStream_t st);

// out[i] = sum_p parts[p*len + i]
template <typename T>
void sum_partials(const T* parts, int nparts, int64_t len, T* out, cudaStream_t st);

// One CTA: sums the nparts partial Gram matrices (row-major k x k each) of an
// n-row panel Y into G = Y^H Y, equilibrates its columns (D = diag(G)^-1/2),
// adds shift * 11 (n k + k (k+1)) u * k to the diagonal when shift != 0, and
// writes Rinv = D R'^{-1} (upper, row-major) with D G D (+shift) = R'^H R',
// so that Y Rinv has orthonormal columns up to the CholeskyQR error.
// flag[0] is set to 1 if a pivot is not positive.  k <= jacobi_svd_max_k<T>().
template <typename T>
void chol_rinv(const T* parts, int nparts, int64_t k, int64_t n, int shift, T* Rinv, int* flag, cudaStream_t st);

// Shifted CholeskyQR of a real column-major n x k panel Y in place, all
// `passes` passes in one launch of one thread-block cluster: the first
// `shifted_passes` add the shift of chol_rinv, and after the first pass the
// perturbation noise_scale * u of add_noise(stream noise_stream) is added.
// flag[0] = 1 if a pivot is not positive.  Callable when
// cholqr_cluster_supported(n, k) (k <= 96 and a device that runs clusters of
// 8 or 16 CTAs with the kernel's shared memory).
// `scratch` holds cholqr_scratch_doubles(k) doubles of device memory.
bool cholqr_cluster_supported(int64_t n, int64_t k);
int64_t cholqr_scratch_doubles(int64_t k);
void cholqr_cluster(double* Y, int64_t n, int64_t k, int passes, int shifted_passes, uint64_t noise_stream,
                    double noise_scale, double* scratch, int* flag, cudaStream_t st);

// y += alpha x (alpha real)
template <typename T>
void axpy(T* y, const T* x, double alpha, int64_t n, cudaStream_t st);

// x *= alpha (scalar, real)
template <typename T>
void scale(T* x, int64_t n, double alpha, cudaStream_t st);

// multiply leg `ax` of a tensor viewed as (outer, dim, inner) by v[dim]
template <typename T>
void scale_leg(T* x, int64_t outer, int64_t dim, int64_t inner, const double* v, cudaStream_t st);

}  // namespace tg
