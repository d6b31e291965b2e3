// Host tensors and the host backend of the library's backend-generic tensor
// algorithms (tenes_b200/csrc/adjoint.hpp, full_update.hpp), for tests on the
// CPU: naive loops, a one-sided Jacobi SVD, and the adjoint's helper kernels
// restated as loops.  Test infrastructure; included by the host check programs.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "adjoint.hpp"

namespace {

using tg::Shape;
using tg::ad::Axes;

struct HT {
  Shape sh;
  std::shared_ptr<std::vector<double>> d;
  double* p() const { return d->data(); }
  int64_t size() const { return tg::numel(sh); }
};

HT make(const Shape& s) { return HT{s, std::make_shared<std::vector<double>>(static_cast<size_t>(tg::numel(s)), 0.0)}; }

HT permute(const HT& a, const Axes& perm) {
  const int r = static_cast<int>(perm.size());
  Shape os(static_cast<size_t>(r));
  for (int i = 0; i < r; ++i) os[i] = a.sh[perm[i]];
  HT o = make(os);
  std::vector<int64_t> istr(static_cast<size_t>(r), 1);
  for (int i = r - 2; i >= 0; --i) istr[i] = istr[i + 1] * a.sh[i + 1];
  std::vector<int64_t> idx(static_cast<size_t>(r), 0);
  for (int64_t lin = 0; lin < o.size(); ++lin) {
    int64_t src = 0;
    for (int i = 0; i < r; ++i) src += idx[i] * istr[perm[i]];
    o.p()[lin] = a.p()[src];
    for (int i = r - 1; i >= 0; --i) {
      if (++idx[i] < os[i]) break;
      idx[i] = 0;
    }
  }
  return o;
}

// one-sided Jacobi SVD of a row-major m x n matrix with m >= n: U (m x n,
// orthonormal, completed where a singular value vanishes), s descending, VT (n x n)
// When set, singular vectors of vanishing values are left as zero vectors
// instead of completing the basis (a solver that does not complete them).
inline bool g_zero_null = false;

void jacobi_svd_tall(const std::vector<double>& A, int64_t m, int64_t n, std::vector<double>& U,
                     std::vector<double>& s, std::vector<double>& VT) {
  std::vector<double> W(A), V(static_cast<size_t>(n * n), 0.0);
  for (int64_t i = 0; i < n; ++i) V[i * n + i] = 1.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0;
    for (int64_t p = 0; p < n; ++p)
      for (int64_t q = p + 1; q < n; ++q) {
        double al = 0, be = 0, ga = 0;
        for (int64_t i = 0; i < m; ++i) {
          const double x = W[i * n + p], y = W[i * n + q];
          al += x * x;
          be += y * y;
          ga += x * y;
        }
        if (ga == 0.0 || std::fabs(ga) <= 1e-15 * std::sqrt(al * be)) continue;
        off = std::max(off, std::fabs(ga) / std::sqrt(al * be));
        const double z = (be - al) / (2 * ga);
        const double t = (z >= 0 ? 1.0 : -1.0) / (std::fabs(z) + std::sqrt(1 + z * z));
        const double c = 1 / std::sqrt(1 + t * t), sn = c * t;
        for (int64_t i = 0; i < m; ++i) {
          const double x = W[i * n + p], y = W[i * n + q];
          W[i * n + p] = c * x - sn * y;
          W[i * n + q] = sn * x + c * y;
        }
        for (int64_t i = 0; i < n; ++i) {
          const double x = V[i * n + p], y = V[i * n + q];
          V[i * n + p] = c * x - sn * y;
          V[i * n + q] = sn * x + c * y;
        }
      }
    if (off < 1e-15) break;
  }
  std::vector<double> nrm(static_cast<size_t>(n));
  for (int64_t j = 0; j < n; ++j) {
    double a = 0;
    for (int64_t i = 0; i < m; ++i) a += W[i * n + j] * W[i * n + j];
    nrm[j] = std::sqrt(a);
  }
  std::vector<int64_t> ord(static_cast<size_t>(n));
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) { return nrm[a] > nrm[b]; });
  U.assign(static_cast<size_t>(m * n), 0.0);
  s.assign(static_cast<size_t>(n), 0.0);
  VT.assign(static_cast<size_t>(n * n), 0.0);
  const double tiny = 1e-13 * (nrm[ord[0]] > 0 ? nrm[ord[0]] : 1.0);
  for (int64_t k = 0; k < n; ++k) {
    const int64_t j = ord[k];
    s[k] = nrm[j];
    for (int64_t i = 0; i < n; ++i) VT[k * n + i] = V[i * n + j];
    // u minus its components along the columns before (two passes); returns the norm left
    auto project_out = [&](std::vector<double>& u) {
      for (int rep = 0; rep < 2; ++rep)
        for (int64_t l = 0; l < k; ++l) {
          double dp = 0;
          for (int64_t i = 0; i < m; ++i) dp += U[i * n + l] * u[i];
          for (int64_t i = 0; i < m; ++i) u[i] -= dp * U[i * n + l];
        }
      double a = 0;
      for (int64_t i = 0; i < m; ++i) a += u[i] * u[i];
      return std::sqrt(a);
    };
    std::vector<double> u(static_cast<size_t>(m));
    double a = 0;
    if (nrm[j] > tiny) {
      for (int64_t i = 0; i < m; ++i) u[i] = W[i * n + j] / nrm[j];
      a = project_out(u);
    } else if (g_zero_null) {
      continue;
    } else {
      // a vanishing value: complete the basis with the standard basis vector
      // that keeps the most norm outside the columns so far
      for (int64_t e = 0; e < m; ++e) {
        std::vector<double> c(static_cast<size_t>(m), 0.0);
        c[static_cast<size_t>(e)] = 1.0;
        const double ce = project_out(c);
        if (ce > a) {
          a = ce;
          u = c;
        }
      }
    }
    for (int64_t i = 0; i < m; ++i) U[i * n + k] = u[i] / a;
  }
}

// Householder QR of a row-major m x n matrix with LAPACK's reflector
// convention (dlarfg: beta = -sign(alpha) |x|), Q = H_1 ... H_k (m x k), R (k x n)
void householder_qr(const std::vector<double>& A, int64_t m, int64_t n, std::vector<double>& Q,
                    std::vector<double>& R) {
  const int64_t k = std::min(m, n);
  std::vector<double> a(A);
  std::vector<std::vector<double>> vs;
  std::vector<double> taus;
  for (int64_t j = 0; j < k; ++j) {
    double alpha = a[j * n + j], xn = 0.0;
    for (int64_t i = j + 1; i < m; ++i) xn += a[i * n + j] * a[i * n + j];
    xn = std::sqrt(xn);
    std::vector<double> v(static_cast<size_t>(m - j), 0.0);
    v[0] = 1.0;
    double tau = 0.0;
    if (xn != 0.0) {
      const double beta = -(alpha >= 0 ? 1.0 : -1.0) * std::hypot(alpha, xn);
      tau = (beta - alpha) / beta;
      for (int64_t i = j + 1; i < m; ++i) v[static_cast<size_t>(i - j)] = a[i * n + j] / (alpha - beta);
      // apply H = I - tau v v^T to columns j..n-1
      for (int64_t c = j; c < n; ++c) {
        double dot = 0.0;
        for (int64_t i = j; i < m; ++i) dot += v[static_cast<size_t>(i - j)] * a[i * n + c];
        for (int64_t i = j; i < m; ++i) a[i * n + c] -= tau * v[static_cast<size_t>(i - j)] * dot;
      }
    }
    vs.push_back(v);
    taus.push_back(tau);
  }
  R.assign(static_cast<size_t>(k * n), 0.0);
  for (int64_t i = 0; i < k; ++i)
    for (int64_t c = i; c < n; ++c) R[i * n + c] = a[i * n + c];
  Q.assign(static_cast<size_t>(m * k), 0.0);
  for (int64_t i = 0; i < k; ++i) Q[i * k + i] = 1.0;
  for (int64_t j = k - 1; j >= 0; --j) {
    const auto& v = vs[static_cast<size_t>(j)];
    for (int64_t c = 0; c < k; ++c) {
      double dot = 0.0;
      for (int64_t i = j; i < m; ++i) dot += v[static_cast<size_t>(i - j)] * Q[i * k + c];
      for (int64_t i = j; i < m; ++i) Q[i * k + c] -= taus[static_cast<size_t>(j)] * v[static_cast<size_t>(i - j)] * dot;
    }
  }
}

// cyclic Jacobi eigendecomposition of a symmetric n x n matrix: ascending w,
// Z (n x n, column j the eigenvector of w_j)
void jacobi_eigh(const std::vector<double>& A, int64_t n, std::vector<double>& w, std::vector<double>& Z) {
  std::vector<double> a(A), v(static_cast<size_t>(n * n), 0.0);
  for (int64_t i = 0; i < n; ++i) v[i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int64_t i = 0; i < n; ++i)
      for (int64_t j = 0; j < n; ++j) (i == j ? tot : off) += a[i * n + j] * a[i * n + j];
    if (off <= 1e-32 * (tot + off) || off == 0.0) break;
    for (int64_t p = 0; p < n; ++p)
      for (int64_t q = p + 1; q < n; ++q) {
        const double apq = a[p * n + q];
        if (apq == 0.0) continue;
        const double th = (a[q * n + q] - a[p * n + p]) / (2 * apq);
        const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1));
        const double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int64_t k = 0; k < n; ++k) {  // columns p, q
          const double x = a[k * n + p], y = a[k * n + q];
          a[k * n + p] = c * x - s * y;
          a[k * n + q] = s * x + c * y;
        }
        for (int64_t k = 0; k < n; ++k) {  // rows p, q
          const double x = a[p * n + k], y = a[q * n + k];
          a[p * n + k] = c * x - s * y;
          a[q * n + k] = s * x + c * y;
        }
        for (int64_t k = 0; k < n; ++k) {
          const double x = v[k * n + p], y = v[k * n + q];
          v[k * n + p] = c * x - s * y;
          v[k * n + q] = s * x + c * y;
        }
      }
  }
  std::vector<int64_t> ord(static_cast<size_t>(n));
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int64_t x, int64_t y) { return a[x * n + x] < a[y * n + y]; });
  w.resize(static_cast<size_t>(n));
  Z.assign(static_cast<size_t>(n * n), 0.0);
  for (int64_t j = 0; j < n; ++j) {
    w[static_cast<size_t>(j)] = a[ord[j] * n + ord[j]];
    for (int64_t i = 0; i < n; ++i) Z[i * n + j] = v[i * n + ord[j]];
  }
}

struct HostBackend {
  using Ten = HT;
  using Scalar = double;
  Ten conj(const Ten& a) { return a; }
  static const Shape& shape(const Ten& t) { return t.sh; }
  static bool empty(const Ten& t) { return !t.d; }

  Ten zeros(const Shape& s) { return make(s); }
  Ten td(const Ten& a, const Ten& b, const Axes& x, const Axes& y, int) {
    const Axes fa = tg::ad::free_legs(static_cast<int>(a.sh.size()), x);
    const Axes fb = tg::ad::free_legs(static_cast<int>(b.sh.size()), y);
    Axes pa(fa), pb(y);
    pa.insert(pa.end(), x.begin(), x.end());
    pb.insert(pb.end(), fb.begin(), fb.end());
    const HT A = permute(a, pa), B = permute(b, pb);
    int64_t M = 1, N = 1, K = 1;
    Shape os;
    for (int l : fa) {
      M *= a.sh[l];
      os.push_back(a.sh[l]);
    }
    for (int l : fb) {
      N *= b.sh[l];
      os.push_back(b.sh[l]);
    }
    for (int l : x) K *= a.sh[l];
    HT o = make(os);
    for (int64_t i = 0; i < M; ++i)
      for (int64_t k = 0; k < K; ++k) {
        const double av = A.p()[i * K + k];
        for (int64_t j = 0; j < N; ++j) o.p()[i * N + j] += av * B.p()[k * N + j];
      }
    return o;
  }
  Ten tr(const Ten& a, const Axes& p) { return permute(a, p); }
  Ten reshape(const Ten& a, const Shape& s) {
    HT o = a;
    o.sh = s;
    return o;
  }
  void axpy(Ten& y, const Ten& x, double alpha) {
    for (int64_t i = 0; i < y.size(); ++i) y.p()[i] += alpha * x.p()[i];
  }
  Ten normalize(const Ten& a) {
    double m = 0;
    for (int64_t i = 0; i < a.size(); ++i) m = std::max(m, std::fabs(a.p()[i]));
    HT c = make(a.sh);
    for (int64_t i = 0; i < a.size(); ++i) c.p()[i] = a.p()[i] / m;
    return c;
  }
  Ten normalize_bwd(const Ten& a, const Ten& c, const Ten& gc) {
    double m = -1;
    int64_t I = 0;
    double dot = 0;
    for (int64_t i = 0; i < a.size(); ++i) {
      if (std::fabs(a.p()[i]) > m) {
        m = std::fabs(a.p()[i]);
        I = i;
      }
      dot += gc.p()[i] * c.p()[i];
    }
    HT g = make(a.sh);
    for (int64_t i = 0; i < a.size(); ++i) g.p()[i] = gc.p()[i] / m;
    g.p()[I] -= (a.p()[I] < 0 ? -dot : dot) / m;
    return g;
  }
  Ten fit(const Ten& a, int64_t d1, int64_t d2, int64_t rest, const Shape& out) {
    HT o = make(out);
    const int64_t chi = out[0];
    for (int64_t i = 0; i < chi; ++i)
      for (int64_t j = 0; j < chi; ++j)
        for (int64_t r = 0; r < rest; ++r)
          o.p()[(i * chi + j) * rest + r] = (i < d1 && j < d2) ? a.p()[(i * d2 + j) * rest + r] : 0.0;
    return o;
  }
  Ten unfit(const Ten& g, int64_t d1, int64_t d2, int64_t rest, int64_t chi, const Shape& in_shape) {
    HT o = make(in_shape);
    for (int64_t i = 0; i < d1; ++i)
      for (int64_t j = 0; j < d2; ++j)
        for (int64_t r = 0; r < rest; ++r)
          o.p()[(i * d2 + j) * rest + r] = (i < chi && j < chi) ? g.p()[(i * chi + j) * rest + r] : 0.0;
    return o;
  }
  void svd_trunc(const Ten& M, int64_t m, int64_t n, int chi, double cutoff, Ten& U, Ten& s, Ten& VT, Ten& sinv,
                 Ten& Uc, Ten& VTc) {
    const int64_t k = std::min(m, n);
    std::vector<double> u, sv, vt;
    if (m >= n) {
      jacobi_svd_tall(*M.d, m, n, u, sv, vt);
      U = make({m, k});
      *U.d = u;
      VT = make({k, n});
      *VT.d = vt;
    } else {  // M^T = U' s VT'  ->  M = VT'^T s U'^T
      const HT Mt = permute(M, {1, 0});
      jacobi_svd_tall(*Mt.d, n, m, u, sv, vt);
      HT Ut = make({n, k});
      *Ut.d = u;
      HT Vt = make({k, m});
      *Vt.d = vt;
      U = permute(Vt, {1, 0});
      VT = permute(Ut, {1, 0});
    }
    s = make({k});
    *s.d = sv;
    const int64_t w = std::min<int64_t>(k, chi);
    sinv = make({w});
    int64_t cut = w;
    for (int64_t i = 0; i < w; ++i) {
      if (sv[i] / sv[0] > cutoff) {
        sinv.p()[i] = 1.0 / std::sqrt(sv[i]);
      } else {
        cut = i;
        break;
      }
    }
    for (int64_t i = cut; i < w; ++i) sinv.p()[i] = 0.0;
    Uc = make({m, w});
    for (int64_t i = 0; i < m; ++i)
      for (int64_t j = 0; j < w; ++j) Uc.p()[i * w + j] = U.p()[i * k + j] * sinv.p()[j];
    VTc = make({w, n});
    for (int64_t j = 0; j < w; ++j)
      for (int64_t l = 0; l < n; ++l) VTc.p()[j * n + l] = VT.p()[j * n + l] * sinv.p()[j];
  }
  void svd_prep(const Ten& gUc, const Ten& gVTc, const Ten& U, const Ten& VT, const Ten& sinv, int64_t m, int64_t n,
                int64_t k, int64_t w, Ten& gU, Ten& gVT, Ten& gs) {
    gU = make({m, k});
    gVT = make({k, n});
    gs = make({k});
    for (int64_t i = 0; i < m; ++i)
      for (int64_t j = 0; j < w; ++j) gU.p()[i * k + j] = gUc.p()[i * w + j] * sinv.p()[j];
    for (int64_t j = 0; j < w; ++j)
      for (int64_t l = 0; l < n; ++l) gVT.p()[j * n + l] = sinv.p()[j] * gVTc.p()[j * n + l];
    for (int64_t j = 0; j < w; ++j) {
      double a = 0;
      for (int64_t i = 0; i < m; ++i) a += gUc.p()[i * w + j] * U.p()[i * k + j];
      for (int64_t l = 0; l < n; ++l) a += gVTc.p()[j * n + l] * VT.p()[j * n + l];
      const double si = sinv.p()[j];
      gs.p()[j] = -0.5 * si * si * si * a;
    }
  }
  void svd_rank_mask(const Ten& U, const Ten& VT, const Ten& s, double tol, Ten& Ur, Ten& VTr) {
    const int64_t m = U.sh[0], k = U.sh[1], n = VT.sh[1];
    Ur = make({m, k});
    VTr = make({k, n});
    for (int64_t j = 0; j < k; ++j) {
      const bool keep = s.p()[j] > tol * s.p()[0];
      for (int64_t i = 0; i < m; ++i) Ur.p()[i * k + j] = keep ? U.p()[i * k + j] : 0.0;
      for (int64_t l = 0; l < n; ++l) VTr.p()[j * n + l] = keep ? VT.p()[j * n + l] : 0.0;
    }
  }
  Ten svd_core(const Ten& J, const Ten& K, const Ten& s, const Ten& gs, int64_t k, double eps) {
    HT c = make({k, k});
    for (int64_t i = 0; i < k; ++i)
      for (int64_t j = 0; j < k; ++j) {
        if (i == j) {
          c.p()[i * k + j] = gs.p()[i];
          continue;
        }
        const double d = s.p()[j] * s.p()[j] - s.p()[i] * s.p()[i];
        const double q = s.p()[j] * s.p()[j] + s.p()[i] * s.p()[i];
        const double den = d * d + eps * q * q;
        const double F = den > 0.0 ? d / den : 0.0;
        c.p()[i * k + j] = F * (J.p()[i * k + j] - J.p()[j * k + i]) * s.p()[j] +
                           s.p()[i] * F * (K.p()[i * k + j] - K.p()[j * k + i]);
      }
    return c;
  }
  void scale_cols_sq(Ten& X, const Ten& sinv, int64_t w) {
    const int64_t rows = X.sh[0], k = X.sh[1];
    for (int64_t i = 0; i < rows; ++i)
      for (int64_t j = 0; j < k; ++j) X.p()[i * k + j] *= j < w ? sinv.p()[j] * sinv.p()[j] : 0.0;
  }
  void scale_rows_sq(Ten& X, const Ten& sinv, int64_t w) {
    const int64_t k = X.sh[0], cols = X.sh[1];
    for (int64_t j = 0; j < k; ++j)
      for (int64_t l = 0; l < cols; ++l) X.p()[j * cols + l] *= j < w ? sinv.p()[j] * sinv.p()[j] : 0.0;
  }
  Ten identity_projector(int64_t e) {
    HT o = make({e, 1, 1, e});
    for (int64_t i = 0; i < e; ++i) o.p()[i * e + i] = 1.0;
    return o;
  }
  Ten from_host(const Shape& s, const double* h) {
    HT o = make(s);
    for (int64_t i = 0; i < o.size(); ++i) o.p()[i] = h[i];
    return o;
  }
  double scalar(const Ten& t) { return t.p()[0]; }

  // ---- matrix factorisations and leg operations used by full_update.hpp
  void qr_matrix(const Ten& M, Ten& Q, Ten& R) {
    const int64_t m = M.sh[0], n = M.sh[1], k = std::min(m, n);
    std::vector<double> q, r;
    householder_qr(*M.d, m, n, q, r);
    Q = make({m, k});
    *Q.d = q;
    R = make({k, n});
    *R.d = r;
  }
  void svd_matrix(const Ten& M, Ten& U, std::vector<double>& s, Ten& VT) {
    const int64_t m = M.sh[0], n = M.sh[1], k = std::min(m, n);
    std::vector<double> u, vt;
    if (m >= n) {
      jacobi_svd_tall(*M.d, m, n, u, s, vt);
      U = make({m, k});
      *U.d = u;
      VT = make({k, n});
      *VT.d = vt;
    } else {
      const HT Mt = permute(M, {1, 0});
      jacobi_svd_tall(*Mt.d, n, m, u, s, vt);
      HT Ut = make({n, k});
      *Ut.d = u;
      HT Vt = make({k, m});
      *Vt.d = vt;
      U = permute(Vt, {1, 0});
      VT = permute(Ut, {1, 0});
    }
  }
  void eigh_matrix(const Ten& M, std::vector<double>& w, Ten& Z) {
    const int64_t n = M.sh[0];
    std::vector<double> z;
    jacobi_eigh(*M.d, n, w, z);
    Z = make({n, n});
    *Z.d = z;
  }
  Ten mulvec(const Ten& A, const std::vector<double>& v, int leg) {
    HT o = make(A.sh);
    int64_t inner = 1;
    for (size_t i = static_cast<size_t>(leg) + 1; i < A.sh.size(); ++i) inner *= A.sh[i];
    const int64_t dim = A.sh[static_cast<size_t>(leg)];
    for (int64_t i = 0; i < A.size(); ++i) o.p()[i] = A.p()[i] * v[static_cast<size_t>((i / inner) % dim)];
    return o;
  }
  void scale(Ten& A, double alpha) {
    for (int64_t i = 0; i < A.size(); ++i) A.p()[i] *= alpha;
  }
  Ten slice(const Ten& A, int leg, int64_t n) {
    Shape s = A.sh;
    s[static_cast<size_t>(leg)] = n;
    HT o = make(s);
    int64_t inner = 1;
    for (size_t i = static_cast<size_t>(leg) + 1; i < A.sh.size(); ++i) inner *= A.sh[i];
    const int64_t dim = A.sh[static_cast<size_t>(leg)];
    for (int64_t i = 0; i < o.size(); ++i) {
      const int64_t r = i % inner, x = (i / inner) % n, outer = i / (inner * n);
      o.p()[i] = A.p()[(outer * dim + x) * inner + r];
    }
    return o;
  }
};

}  // namespace
