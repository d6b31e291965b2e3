// Complex host tensors and the complex host backend of the full-update bond
// step (tenes_b200/csrc/full_update.hpp), for tests on the CPU: naive loops,
// QR by Gram-Schmidt with re-orthogonalisation, one-sided complex Jacobi SVD,
// Hermitian Jacobi eigendecomposition.  The bond step depends on the sign /
// phase conventions of these factorisations only through a gauge on the
// updated bond, which the tests remove.  Test infrastructure.
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <memory>
#include <numeric>
#include <vector>

#include "common.hpp"

namespace {

using cd = std::complex<double>;

struct HTC {
  tg::Shape sh;
  std::shared_ptr<std::vector<cd>> d;
  cd* p() const { return d->data(); }
  int64_t size() const { return tg::numel(sh); }
};

HTC makec(const tg::Shape& s) {
  return HTC{s, std::make_shared<std::vector<cd>>(static_cast<size_t>(tg::numel(s)), cd(0.0, 0.0))};
}

HTC permutec(const HTC& a, const std::vector<int>& perm) {
  const int r = static_cast<int>(perm.size());
  tg::Shape os(static_cast<size_t>(r));
  for (int i = 0; i < r; ++i) os[i] = a.sh[perm[i]];
  HTC o = makec(os);
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

// u minus its components along the first k columns of the row-major m x ld
// matrix Q (two passes); returns the norm left
double project_out_c(const std::vector<cd>& Q, int64_t m, int64_t ld, int64_t k, std::vector<cd>& u) {
  for (int rep = 0; rep < 2; ++rep)
    for (int64_t l = 0; l < k; ++l) {
      cd dp = 0.0;
      for (int64_t i = 0; i < m; ++i) dp += std::conj(Q[i * ld + l]) * u[i];
      for (int64_t i = 0; i < m; ++i) u[i] -= dp * Q[i * ld + l];
    }
  double a = 0.0;
  for (int64_t i = 0; i < m; ++i) a += std::norm(u[i]);
  return std::sqrt(a);
}

// a unit vector orthogonal to the first k columns of Q: the standard basis
// vector that keeps the most norm, orthogonalised
std::vector<cd> completion_c(const std::vector<cd>& Q, int64_t m, int64_t ld, int64_t k) {
  std::vector<cd> best(static_cast<size_t>(m), cd(0.0));
  double bn = -1.0;
  for (int64_t e = 0; e < m; ++e) {
    std::vector<cd> c(static_cast<size_t>(m), cd(0.0));
    c[static_cast<size_t>(e)] = 1.0;
    const double n = project_out_c(Q, m, ld, k, c);
    if (n > bn) {
      bn = n;
      best = c;
    }
  }
  for (auto& x : best) x /= bn;
  return best;
}

// thin QR of a row-major m x n matrix: Q (m x k), R (k x n), k = min(m, n)
void gs_qr_c(const std::vector<cd>& A, int64_t m, int64_t n, std::vector<cd>& Q, std::vector<cd>& R) {
  const int64_t k = std::min(m, n);
  Q.assign(static_cast<size_t>(m * k), cd(0.0));
  R.assign(static_cast<size_t>(k * n), cd(0.0));
  const double scale = [&] {
    double a = 0.0;
    for (const cd& x : A) a = std::max(a, std::abs(x));
    return a > 0 ? a : 1.0;
  }();
  for (int64_t j = 0; j < k; ++j) {
    std::vector<cd> u(static_cast<size_t>(m));
    for (int64_t i = 0; i < m; ++i) u[i] = A[i * n + j];
    const double nr = project_out_c(Q, m, k, j, u);
    if (nr > 1e-13 * scale) {
      for (int64_t i = 0; i < m; ++i) Q[i * k + j] = u[i] / nr;
    } else {
      const std::vector<cd> c = completion_c(Q, m, k, j);
      for (int64_t i = 0; i < m; ++i) Q[i * k + j] = c[i];
    }
  }
  for (int64_t i = 0; i < k; ++i)
    for (int64_t c = i; c < n; ++c) {
      cd dp = 0.0;
      for (int64_t r = 0; r < m; ++r) dp += std::conj(Q[r * k + i]) * A[r * n + c];
      R[i * n + c] = dp;
    }
}

// one-sided Jacobi SVD of a row-major m x n matrix with m >= n:
// U (m x n), s descending, VT = V^H (n x n)
void jacobi_svd_tall_c(const std::vector<cd>& A, int64_t m, int64_t n, std::vector<cd>& U, std::vector<double>& s,
                       std::vector<cd>& VT) {
  std::vector<cd> W(A), V(static_cast<size_t>(n * n), cd(0.0));
  for (int64_t i = 0; i < n; ++i) V[i * n + i] = 1.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0;
    for (int64_t p = 0; p < n; ++p)
      for (int64_t q = p + 1; q < n; ++q) {
        double al = 0, be = 0;
        cd ga = 0.0;
        for (int64_t i = 0; i < m; ++i) {
          al += std::norm(W[i * n + p]);
          be += std::norm(W[i * n + q]);
          ga += std::conj(W[i * n + p]) * W[i * n + q];
        }
        const double g = std::abs(ga);
        if (g == 0.0 || g <= 1e-15 * std::sqrt(al * be)) continue;
        off = std::max(off, g / std::sqrt(al * be));
        const cd e = std::conj(ga / g);  // column q times e makes a_p^H a_q real
        const double z = (be - al) / (2 * g);
        const double t = (z >= 0 ? 1.0 : -1.0) / (std::fabs(z) + std::sqrt(1 + z * z));
        const double c = 1 / std::sqrt(1 + t * t), sn = c * t;
        for (int64_t i = 0; i < m; ++i) {
          const cd x = W[i * n + p], y = W[i * n + q] * e;
          W[i * n + p] = c * x - sn * y;
          W[i * n + q] = sn * x + c * y;
        }
        for (int64_t i = 0; i < n; ++i) {
          const cd x = V[i * n + p], y = V[i * n + q] * e;
          V[i * n + p] = c * x - sn * y;
          V[i * n + q] = sn * x + c * y;
        }
      }
    if (off < 1e-15) break;
  }
  std::vector<double> nrm(static_cast<size_t>(n));
  for (int64_t j = 0; j < n; ++j) {
    double a = 0;
    for (int64_t i = 0; i < m; ++i) a += std::norm(W[i * n + j]);
    nrm[j] = std::sqrt(a);
  }
  std::vector<int64_t> ord(static_cast<size_t>(n));
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) { return nrm[a] > nrm[b]; });
  U.assign(static_cast<size_t>(m * n), cd(0.0));
  s.assign(static_cast<size_t>(n), 0.0);
  VT.assign(static_cast<size_t>(n * n), cd(0.0));
  const double tiny = 1e-13 * (nrm[ord[0]] > 0 ? nrm[ord[0]] : 1.0);
  for (int64_t k = 0; k < n; ++k) {
    const int64_t j = ord[k];
    s[k] = nrm[j];
    for (int64_t i = 0; i < n; ++i) VT[k * n + i] = std::conj(V[i * n + j]);
    std::vector<cd> u(static_cast<size_t>(m));
    double a = 0.0;
    if (nrm[j] > tiny) {
      for (int64_t i = 0; i < m; ++i) u[i] = W[i * n + j] / nrm[j];
      a = project_out_c(U, m, n, k, u);
      for (auto& x : u) x /= a;
    } else {
      u = completion_c(U, m, n, k);
    }
    for (int64_t i = 0; i < m; ++i) U[i * n + k] = u[i];
  }
}

// Hermitian Jacobi eigendecomposition of an n x n matrix: ascending w,
// Z (n x n, column j the eigenvector of w_j)
void jacobi_eigh_c(const std::vector<cd>& H, int64_t n, std::vector<double>& w, std::vector<cd>& Z) {
  std::vector<cd> a(H), v(static_cast<size_t>(n * n), cd(0.0));
  for (int64_t i = 0; i < n; ++i) v[i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int64_t i = 0; i < n; ++i)
      for (int64_t j = 0; j < n; ++j) (i == j ? tot : off) += std::norm(a[i * n + j]);
    if (off == 0.0 || off <= 1e-32 * (tot + off)) break;
    for (int64_t p = 0; p < n; ++p)
      for (int64_t q = p + 1; q < n; ++q) {
        const cd h = a[p * n + q];
        const double g = std::abs(h);
        if (g == 0.0) continue;
        const cd e = std::conj(h / g);  // column q times e, row q times conj(e): a_pq -> |h|
        for (int64_t k = 0; k < n; ++k) a[k * n + q] *= e;
        for (int64_t k = 0; k < n; ++k) a[q * n + k] *= std::conj(e);
        for (int64_t k = 0; k < n; ++k) v[k * n + q] *= e;
        const double th = (a[q * n + q].real() - a[p * n + p].real()) / (2 * g);
        const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1));
        const double c = 1 / std::sqrt(t * t + 1), sn = t * c;
        for (int64_t k = 0; k < n; ++k) {
          const cd x = a[k * n + p], y = a[k * n + q];
          a[k * n + p] = c * x - sn * y;
          a[k * n + q] = sn * x + c * y;
        }
        for (int64_t k = 0; k < n; ++k) {
          const cd x = a[p * n + k], y = a[q * n + k];
          a[p * n + k] = c * x - sn * y;
          a[q * n + k] = sn * x + c * y;
        }
        for (int64_t k = 0; k < n; ++k) {
          const cd x = v[k * n + p], y = v[k * n + q];
          v[k * n + p] = c * x - sn * y;
          v[k * n + q] = sn * x + c * y;
        }
      }
  }
  std::vector<int64_t> ord(static_cast<size_t>(n));
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(),
                   [&](int64_t x, int64_t y) { return a[x * n + x].real() < a[y * n + y].real(); });
  w.resize(static_cast<size_t>(n));
  Z.assign(static_cast<size_t>(n * n), cd(0.0));
  for (int64_t j = 0; j < n; ++j) {
    w[static_cast<size_t>(j)] = a[ord[j] * n + ord[j]].real();
    for (int64_t i = 0; i < n; ++i) Z[i * n + j] = v[i * n + ord[j]];
  }
}

struct HostBackendC {
  using Ten = HTC;
  using Scalar = cd;
  static const tg::Shape& shape(const Ten& t) { return t.sh; }

  Ten td(const Ten& a, const Ten& b, const std::vector<int>& x, const std::vector<int>& y, int) {
    std::vector<int> fa, fb;
    for (int i = 0; i < static_cast<int>(a.sh.size()); ++i)
      if (std::find(x.begin(), x.end(), i) == x.end()) fa.push_back(i);
    for (int i = 0; i < static_cast<int>(b.sh.size()); ++i)
      if (std::find(y.begin(), y.end(), i) == y.end()) fb.push_back(i);
    std::vector<int> pa(fa), pb(y);
    pa.insert(pa.end(), x.begin(), x.end());
    pb.insert(pb.end(), fb.begin(), fb.end());
    const HTC A = permutec(a, pa), B = permutec(b, pb);
    int64_t M = 1, N = 1, K = 1;
    tg::Shape os;
    for (int l : fa) {
      M *= a.sh[l];
      os.push_back(a.sh[l]);
    }
    for (int l : fb) {
      N *= b.sh[l];
      os.push_back(b.sh[l]);
    }
    for (int l : x) K *= a.sh[l];
    HTC o = makec(os);
    for (int64_t i = 0; i < M; ++i)
      for (int64_t k = 0; k < K; ++k) {
        const cd av = A.p()[i * K + k];
        for (int64_t j = 0; j < N; ++j) o.p()[i * N + j] += av * B.p()[k * N + j];
      }
    return o;
  }
  Ten tr(const Ten& a, const std::vector<int>& p) { return permutec(a, p); }
  Ten reshape(const Ten& a, const tg::Shape& s) {
    HTC o = a;
    o.sh = s;
    return o;
  }
  Ten conj(const Ten& a) {
    HTC o = makec(a.sh);
    for (int64_t i = 0; i < a.size(); ++i) o.p()[i] = std::conj(a.p()[i]);
    return o;
  }
  void axpy(Ten& y, const Ten& x, double alpha) {
    for (int64_t i = 0; i < y.size(); ++i) y.p()[i] += alpha * x.p()[i];
  }
  void scale(Ten& A, double alpha) {
    for (int64_t i = 0; i < A.size(); ++i) A.p()[i] *= alpha;
  }
  cd scalar(const Ten& t) { return t.p()[0]; }
  void qr_matrix(const Ten& M, Ten& Q, Ten& R) {
    const int64_t m = M.sh[0], n = M.sh[1], k = std::min(m, n);
    std::vector<cd> q, r;
    gs_qr_c(*M.d, m, n, q, r);
    Q = makec({m, k});
    *Q.d = q;
    R = makec({k, n});
    *R.d = r;
  }
  void svd_matrix(const Ten& M, Ten& U, std::vector<double>& s, Ten& VT) {
    const int64_t m = M.sh[0], n = M.sh[1], k = std::min(m, n);
    std::vector<cd> u, vt;
    if (m >= n) {
      jacobi_svd_tall_c(*M.d, m, n, u, s, vt);
      U = makec({m, k});
      *U.d = u;
      VT = makec({k, n});
      *VT.d = vt;
    } else {  // M^H = U' s V'^H  ->  M = V' s U'^H
      const HTC Mh = conj(permutec(M, {1, 0}));
      jacobi_svd_tall_c(*Mh.d, n, m, u, s, vt);
      HTC Up = makec({n, k});
      *Up.d = u;
      HTC Vh = makec({k, m});
      *Vh.d = vt;
      U = conj(permutec(Vh, {1, 0}));
      VT = conj(permutec(Up, {1, 0}));
    }
  }
  void eigh_matrix(const Ten& M, std::vector<double>& w, Ten& Z) {
    const int64_t n = M.sh[0];
    std::vector<cd> z;
    jacobi_eigh_c(*M.d, n, w, z);
    Z = makec({n, n});
    *Z.d = z;
  }
  Ten mulvec(const Ten& A, const std::vector<double>& v, int leg) {
    HTC o = makec(A.sh);
    int64_t inner = 1;
    for (size_t i = static_cast<size_t>(leg) + 1; i < A.sh.size(); ++i) inner *= A.sh[i];
    const int64_t dim = A.sh[static_cast<size_t>(leg)];
    for (int64_t i = 0; i < A.size(); ++i) o.p()[i] = A.p()[i] * v[static_cast<size_t>((i / inner) % dim)];
    return o;
  }
  Ten slice(const Ten& A, int leg, int64_t n) {
    tg::Shape s = A.sh;
    s[static_cast<size_t>(leg)] = n;
    HTC o = makec(s);
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
