// Device backend of the CTMRG energy adjoint: the tape of adjoint.hpp over
// DT<double> tensors, with the products on the library's DMMA / 3xTF32
// tensordot and the adjoint-only steps as the small kernels below.
#include <cuda_runtime.h>

#include <cmath>
#include <utility>

#include "adjoint_device.hpp"
#include "kernels.cuh"

namespace tg {
namespace {

inline int blocks_for(int64_t n, int threads = 256) {
  const int64_t b = (n + threads - 1) / threads;
  return static_cast<int>(std::min<int64_t>(std::max<int64_t>(b, 1), 148 * 8));
}

#define GRID_STRIDE(i, n)                                                                  \
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < (n); \
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)

// out[i*nb + j] = a[i] b[j]  (tensordot without contracted legs)
__global__ void outer_kernel(const double* __restrict__ a, int64_t na, const double* __restrict__ b, int64_t nb,
                             double* __restrict__ out) {
  GRID_STRIDE(i, na * nb) { out[i] = a[i / nb] * b[i % nb]; }
}

// Adjoint of c = a / m, m = max_i |a_i| attained first at index I:
// ga = gc / m - sign(a_I) (gc . c) / m e_I.  One CTA of kNormThreads threads;
// the reductions run in a fixed order, so the result is reproducible.
constexpr int kNormThreads = 1024;
__global__ void __launch_bounds__(kNormThreads) normalize_bwd_kernel(const double* __restrict__ a,
                                                                     const double* __restrict__ c,
                                                                     const double* __restrict__ gc,
                                                                     double* __restrict__ ga, int64_t n) {
  __shared__ double s_m[32], s_d[32];
  __shared__ long long s_i[32];
  double m = -1.0, dot = 0.0;
  long long idx = n;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = fabs(a[i]);
    if (v > m) {
      m = v;
      idx = i;
    }
    dot = fma(gc[i], c[i], dot);
  }
  for (int off = 16; off > 0; off >>= 1) {
    const double m2 = __shfl_down_sync(0xffffffffu, m, off);
    const long long i2 = __shfl_down_sync(0xffffffffu, idx, off);
    dot += __shfl_down_sync(0xffffffffu, dot, off);
    if (m2 > m || (m2 == m && i2 < idx)) {
      m = m2;
      idx = i2;
    }
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  if (lane == 0) {
    s_m[warp] = m;
    s_i[warp] = idx;
    s_d[warp] = dot;
  }
  __syncthreads();
  if (warp == 0) {
    m = lane < nwarp ? s_m[lane] : -1.0;
    idx = lane < nwarp ? s_i[lane] : n;
    dot = lane < nwarp ? s_d[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) {
      const double m2 = __shfl_down_sync(0xffffffffu, m, off);
      const long long i2 = __shfl_down_sync(0xffffffffu, idx, off);
      dot += __shfl_down_sync(0xffffffffu, dot, off);
      if (m2 > m || (m2 == m && i2 < idx)) {
        m = m2;
        idx = i2;
      }
    }
    if (lane == 0) {
      s_m[0] = m;
      s_i[0] = idx;
      s_d[0] = dot;
    }
  }
  __syncthreads();
  const double M = s_m[0], D = s_d[0];
  const long long I = s_i[0];
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    double v = gc[i] / M;
    if (i == I) v -= (a[i] < 0.0 ? -D : D) / M;
    ga[i] = v;
  }
}

// adjoint of fit_chi: gin(d1, d2, rest) = gout(chi, chi, rest) sliced / zero-padded back
__global__ void unfit_kernel(const double* __restrict__ g, int64_t chi, int64_t d1, int64_t d2, int64_t rest,
                             double* __restrict__ out) {
  GRID_STRIDE(i, d1 * d2 * rest) {
    const int64_t r = i % rest;
    const int64_t b = (i / rest) % d2;
    const int64_t a = i / (rest * d2);
    out[i] = (a < chi && b < chi) ? g[(a * chi + b) * rest + r] : 0.0;
  }
}

// gU (m x k) = [gUc diag(sinv), 0], gVT (k x n) = [diag(sinv) gVTc; 0]
__global__ void svd_prep_kernel(const double* __restrict__ gUc, const double* __restrict__ gVTc,
                                const double* __restrict__ sinv, int64_t m, int64_t n, int64_t k, int64_t w,
                                double* __restrict__ gU, double* __restrict__ gVT) {
  GRID_STRIDE(i, m * k) {
    const int64_t j = i % k;
    gU[i] = j < w ? gUc[(i / k) * w + j] * sinv[j] : 0.0;
  }
  GRID_STRIDE(i, k * n) {
    const int64_t j = i / n;
    gVT[i] = j < w ? sinv[j] * gVTc[j * n + (i % n)] : 0.0;
  }
}

// gs_j = d/ds_j of s_j^-1/2 times (gUc[:, j] . U[:, j] + gVTc[j, :] . VT[j, :]),
// zero where the value was cut (sinv_j = 0).  One CTA per j.
__global__ void svd_gs_kernel(const double* __restrict__ gUc, const double* __restrict__ gVTc,
                              const double* __restrict__ U, const double* __restrict__ VT,
                              const double* __restrict__ sinv, int64_t m, int64_t n, int64_t k, int64_t w,
                              double* __restrict__ gs) {
  __shared__ double red[32];
  const int64_t j = blockIdx.x;
  if (j >= k) return;
  if (j >= w) {
    if (threadIdx.x == 0) gs[j] = 0.0;
    return;
  }
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < m; i += blockDim.x) acc = fma(gUc[i * w + j], U[i * k + j], acc);
  for (int64_t l = threadIdx.x; l < n; l += blockDim.x) acc = fma(gVTc[j * n + l], VT[j * n + l], acc);
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  if (warp == 0) {
    acc = lane < nwarp ? red[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) {
      const double si = sinv[j];
      gs[j] = -0.5 * si * si * si * acc;
    }
  }
}

// core_ij = delta_ij gs_i + F_ij (J_ij - J_ji) s_j + s_i F_ij (K_ij - K_ji),
// F_ij = (s_j^2 - s_i^2) / ((s_j^2 - s_i^2)^2 + eps (s_i^2 + s_j^2)^2), F_ii = 0
// (the broadening relative to the pair's own scale, so that it acts on
// near-degenerate pairs only, whatever the matrix's norm)
__global__ void svd_core_kernel(const double* __restrict__ J, const double* __restrict__ K,
                                const double* __restrict__ s, const double* __restrict__ gs, int64_t k, double eps,
                                double* __restrict__ core) {
  GRID_STRIDE(idx, k * k) {
    const int64_t i = idx / k, j = idx % k;
    if (i == j) {
      core[idx] = gs[i];
    } else {
      const double d = s[j] * s[j] - s[i] * s[i], q = s[j] * s[j] + s[i] * s[i];
      const double den = d * d + eps * q * q;
      const double F = den > 0.0 ? d / den : 0.0;
      const int64_t t = j * k + i;
      core[idx] = F * (J[idx] - J[t]) * s[j] + s[i] * F * (K[idx] - K[t]);
    }
  }
}

// Ur = U with the columns of vanishing singular values (s_j <= tol s_0)
// zeroed, VTr = VT with those rows zeroed
__global__ void svd_rank_mask_kernel(const double* __restrict__ U, const double* __restrict__ VT,
                                     const double* __restrict__ s, int64_t m, int64_t n, int64_t k, double tol,
                                     double* __restrict__ Ur, double* __restrict__ VTr) {
  const double thr = tol * s[0];
  GRID_STRIDE(i, m * k) { Ur[i] = s[i % k] > thr ? U[i] : 0.0; }
  GRID_STRIDE(i, k * n) { VTr[i] = s[i / n] > thr ? VT[i] : 0.0; }
}

// X(rows x k) columns j scaled by sinv_j^2 = 1 / s_j (0 beyond w or where cut)
__global__ void scale_cols_sq_kernel(double* __restrict__ X, int64_t rows, int64_t k, const double* __restrict__ sinv,
                                     int64_t w) {
  GRID_STRIDE(i, rows * k) {
    const int64_t j = i % k;
    X[i] *= j < w ? sinv[j] * sinv[j] : 0.0;
  }
}
// X(k x cols) rows j scaled by sinv_j^2
__global__ void scale_rows_sq_kernel(double* __restrict__ X, int64_t k, int64_t cols, const double* __restrict__ sinv,
                                     int64_t w) {
  GRID_STRIDE(i, k * cols) {
    const int64_t j = i / cols;
    X[i] *= j < w ? sinv[j] * sinv[j] : 0.0;
  }
}

#undef GRID_STRIDE

struct DevBackend {
  using Ten = DT<double>;
  cudaStream_t st;
  const SvdFn& svd_fn;
  DT<unsigned long long> maxbuf;
  DT<int> cutbuf;

  DevBackend(cudaStream_t s, const SvdFn& f) : st(s), svd_fn(f), maxbuf({1}, s), cutbuf({1}, s) {}

  static const Shape& shape(const Ten& t) { return t.sh; }
  static bool empty(const Ten& t) { return t.p == nullptr; }

  Ten zeros(const Shape& s) { return tg::zeros<double>(s, st); }
  Ten td(const Ten& a, const Ten& b, const ad::Axes& x, const ad::Axes& y, int prec) {
    if (!x.empty()) return tensordot<double>(a, b, x, y, st, false, false, prec);
    Shape s = a.sh;
    s.insert(s.end(), b.sh.begin(), b.sh.end());
    Ten out(s, st);
    outer_kernel<<<blocks_for(out.size()), 256, 0, st>>>(a.p, a.size(), b.p, b.size(), out.p);
    TG_CHECK_LAUNCH();
    count_launch();
    return out;
  }
  Ten tr(const Ten& a, const ad::Axes& p) { return transpose<double>(a, p, st); }
  Ten reshape(const Ten& a, const Shape& s) { return tg::reshape(a, s); }
  void axpy(Ten& y, const Ten& x, double alpha) {
    if (y.size() != x.size()) fail(TG_E_RUNTIME, "energy gradient: adjoint size mismatch");
    tg::axpy<double>(y.p, x.p, alpha, y.size(), st);
  }
  Ten normalize(const Ten& a) {
    Ten c(a.sh, st);
    normalize_max_abs<double>(a.p, c.p, a.size(), maxbuf.p, st);
    return c;
  }
  Ten normalize_bwd(const Ten& a, const Ten& c, const Ten& gc) {
    Ten ga(a.sh, st);
    normalize_bwd_kernel<<<1, kNormThreads, 0, st>>>(a.p, c.p, gc.p, ga.p, a.size());
    TG_CHECK_LAUNCH();
    count_launch();
    return ga;
  }
  Ten fit(const Ten& a, int64_t d1, int64_t d2, int64_t rest, const Shape& out) {
    Ten o(out, st);
    fit_chi<double>(a.p, d1, d2, rest, o.p, out[0], st);
    return o;
  }
  Ten unfit(const Ten& g, int64_t d1, int64_t d2, int64_t rest, int64_t chi, const Shape& in_shape) {
    Ten o(in_shape, st);
    unfit_kernel<<<blocks_for(o.size()), 256, 0, st>>>(g.p, chi, d1, d2, rest, o.p);
    TG_CHECK_LAUNCH();
    count_launch();
    return o;
  }
  void svd_trunc(const Ten& M, int64_t m, int64_t n, int chi, double cutoff, Ten& U, Ten& s, Ten& VT, Ten& sinv,
                 Ten& Uc, Ten& VTc) {
    Ten A = clone(M, st);
    svd_fn(A, m, n, U, s, VT);
    const int64_t k = std::min(m, n);
    const int w = static_cast<int>(std::min<int64_t>(k, chi));
    sinv = Ten({w}, st);
    truncation(s.p, k, chi, cutoff, sinv.p, w, cutbuf.p, st);
    Uc = Ten({m, w}, st);
    scale_cols<double>(U.p, k, m, w, sinv.p, false, Uc.p, st);
    VTc = Ten({w, n}, st);
    scale_rows<double>(VT.p, n, n, w, sinv.p, false, VTc.p, st);
  }
  void svd_prep(const Ten& gUc, const Ten& gVTc, const Ten& U, const Ten& VT, const Ten& sinv, int64_t m, int64_t n,
                int64_t k, int64_t w, Ten& gU, Ten& gVT, Ten& gs) {
    gU = Ten({m, k}, st);
    gVT = Ten({k, n}, st);
    gs = Ten({k}, st);
    svd_prep_kernel<<<blocks_for(std::max(m * k, k * n)), 256, 0, st>>>(gUc.p, gVTc.p, sinv.p, m, n, k, w, gU.p,
                                                                        gVT.p);
    TG_CHECK_LAUNCH();
    svd_gs_kernel<<<static_cast<unsigned>(k), 256, 0, st>>>(gUc.p, gVTc.p, U.p, VT.p, sinv.p, m, n, k, w, gs.p);
    TG_CHECK_LAUNCH();
    count_launch(2);
  }
  void svd_rank_mask(const Ten& U, const Ten& VT, const Ten& s, double tol, Ten& Ur, Ten& VTr) {
    const int64_t m = U.dim(0), k = U.dim(1), n = VT.dim(1);
    Ur = Ten({m, k}, st);
    VTr = Ten({k, n}, st);
    svd_rank_mask_kernel<<<blocks_for(std::max(m * k, k * n)), 256, 0, st>>>(U.p, VT.p, s.p, m, n, k, tol, Ur.p,
                                                                             VTr.p);
    TG_CHECK_LAUNCH();
    count_launch();
  }
  Ten svd_core(const Ten& J, const Ten& K, const Ten& s, const Ten& gs, int64_t k, double eps) {
    Ten core({k, k}, st);
    svd_core_kernel<<<blocks_for(k * k), 256, 0, st>>>(J.p, K.p, s.p, gs.p, k, eps, core.p);
    TG_CHECK_LAUNCH();
    count_launch();
    return core;
  }
  void scale_cols_sq(Ten& X, const Ten& sinv, int64_t w) {
    scale_cols_sq_kernel<<<blocks_for(X.size()), 256, 0, st>>>(X.p, X.dim(0), X.dim(1), sinv.p, w);
    TG_CHECK_LAUNCH();
    count_launch();
  }
  void scale_rows_sq(Ten& X, const Ten& sinv, int64_t w) {
    scale_rows_sq_kernel<<<blocks_for(X.size()), 256, 0, st>>>(X.p, X.dim(0), X.dim(1), sinv.p, w);
    TG_CHECK_LAUNCH();
    count_launch();
  }
  Ten identity_projector(int64_t e) {
    Ten o({e, 1, 1, e}, st);
    identity<double>(o.p, e, st);
    return o;
  }
  Ten from_host(const Shape& s, const double* h) {
    Ten t(s, st);
    TG_CUDA(cudaMemcpyAsync(t.p, h, sizeof(double) * static_cast<size_t>(t.size()), cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaStreamSynchronize(st));
    return t;
  }
  double scalar(const Ten& t) {
    double v = 0.0;
    TG_CUDA(cudaMemcpyAsync(&v, t.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    return v;
  }
};

}  // namespace

double energy_grad_device(cudaStream_t st, const Lattice& lat, const std::vector<DT<double>>& Tn,
                          const std::vector<ad::WindowTerm>& terms, const ad::Options& o, const SvdFn& svd,
                          std::vector<DT<double>>* grads) {
  DevBackend bk(st, svd);
  return ad::energy_grad(bk, lat, Tn, terms, o, grads);
}

}  // namespace tg
