// Host instantiation of the CTMRG energy adjoint (tenes_b200/csrc/adjoint.hpp)
// for tests on the CPU: the same tape, moves, windows and checkpoint scheme as
// the device build, over plain host tensors (naive loops and a one-sided
// Jacobi SVD).  Reads a problem from stdin, prints E and dE/dTn.
//
// Input (whitespace separated):
//   LX LY skew chi iterations checkpoint_every
//   cutoff eps
//   per site: pdim D0 D1 D2 D3
//   per site: D0*D1*D2*D3*pdim values (row-major)
//   nterms, then per term: source nrow ncol source_row source_col coeff nops,
//     then per operator: row col d, d*d values
// Output: "E <energy>" and one line "G <values>" per site.  With the argument
// "zero-null" the host SVD leaves the singular vectors of vanishing values
// as zero vectors.
#include <cmath>
#include <cstdio>
#include <iostream>
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
bool g_zero_null = false;

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

struct HostBackend {
  using Ten = HT;
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
        const double F = d / (d * d + eps);
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
};

}  // namespace

int main(int argc, char** argv) {
  g_zero_null = argc > 1 && std::string(argv[1]) == "zero-null";
  int LX, LY, skew, chi, iters, ckpt;
  double cutoff, eps;
  std::cin >> LX >> LY >> skew >> chi >> iters >> ckpt >> cutoff >> eps;
  tg::Lattice lat(LX, LY, skew);
  lat.pdim.resize(lat.N);
  lat.vdim.resize(lat.N);
  for (int i = 0; i < lat.N; ++i) {
    std::cin >> lat.pdim[i];
    for (int l = 0; l < 4; ++l) std::cin >> lat.vdim[i][l];
  }
  lat.check_dims();
  std::vector<HT> Tn;
  for (int i = 0; i < lat.N; ++i) {
    const auto& v = lat.vdim[i];
    HT t = make({v[0], v[1], v[2], v[3], lat.pdim[i]});
    for (int64_t q = 0; q < t.size(); ++q) std::cin >> t.p()[q];
    Tn.push_back(t);
  }
  int nterms;
  std::cin >> nterms;
  std::vector<tg::ad::WindowTerm> terms(static_cast<size_t>(nterms));
  for (auto& t : terms) {
    int nops;
    std::cin >> t.source >> t.nrow >> t.ncol >> t.source_row >> t.source_col >> t.coeff >> nops;
    for (int q = 0; q < nops; ++q) {
      int r, c, d;
      std::cin >> r >> c >> d;
      std::vector<double> op(static_cast<size_t>(d * d));
      for (auto& x : op) std::cin >> x;
      t.op_row.push_back(r);
      t.op_col.push_back(c);
      t.ops.push_back(op);
    }
  }
  tg::ad::Options o;
  o.chi = chi;
  o.cutoff = cutoff;
  o.eps = eps;
  o.iterations = iters;
  o.checkpoint_every = ckpt;
  HostBackend bk;
  std::vector<HT> g;
  const double E = tg::ad::energy_grad(bk, lat, Tn, terms, o, &g);
  std::printf("E %.17g\n", E);
  for (const HT& x : g) {
    std::printf("G");
    for (int64_t q = 0; q < x.size(); ++q) std::printf(" %.17g", x.p()[q]);
    std::printf("\n");
  }
  return 0;
}
