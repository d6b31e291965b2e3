// Local gauge fixing of the simple update (TeNeS core::fix_local_gauge and
// boundary_tensor, src/iTPS/core/local_gauge.cpp:44-224; the sweep of
// iTPS::fix_local_gauge, src/iTPS/simple_update.cpp:49-101), written once
// over a tensor backend BK like the full update (full_update.hpp): the library
// instantiates it on device tensors (engine.cu), the tests on host tensors.
//
// Backend API used here: Ten, shape(t), td(a, b, x, y, prec) (free legs of a,
// then of b), tr(a, perm), conj(a), mulvec(a, v, leg) (leg scaled by a real
// vector), eigh_matrix(M, w, Z) (ascending w, eigenvectors in the columns of
// Z), svd_matrix(M, U, s, VT) (thin SVD).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <vector>

namespace tg {
namespace gauge {

using Axes = std::vector<int>;
using Weights = std::array<std::vector<double>, 4>;  // the four bond weights of a site

template <class BK>
struct LocalGauge {
  using Ten = typename BK::Ten;
  BK& bk;
  double lambda_cut;  // Inverse_lambda_cut

  std::vector<double> inv(const std::vector<double>& v) const {
    std::vector<double> r(v.size());
    for (size_t i = 0; i < v.size(); ++i) r[i] = v[i] > lambda_cut ? 1.0 / v[i] : 0.0;
    return r;
  }

  // boundary_tensor (:190-224): the weights on the three other legs and the
  // inverse weight on `connect`, contracted with the conjugate over every leg
  // but `connect`; M[a, b] = sum conj(T)[.., a, ..] T[.., b, ..]
  Ten boundary(const Ten& T, const Weights& lam, int connect) {
    Ten X = T;
    for (int leg = 0; leg < 4; ++leg) X = bk.mulvec(X, leg == connect ? inv(lam[leg]) : lam[leg], leg);
    Axes rest;
    for (int l = 0; l < 5; ++l)
      if (l != connect) rest.push_back(l);
    return bk.td(bk.conj(X), X, rest, rest, 0);
  }

  // the contracted leg (last, after the physical one) back to `connect`
  static Axes back(int connect) {
    switch (connect) {
      case 0: return {4, 0, 1, 2, 3};
      case 1: return {0, 4, 1, 2, 3};
      case 2: return {0, 1, 4, 2, 3};
      default: return {0, 1, 2, 4, 3};
    }
  }

  // fix_local_gauge (:44-158) for the bond (Tn1 leg connect1, Tn2 leg
  // connect1 + 2).  As in the reference, the boundary eigenvalues are
  // square-rooted and inverted without a cutoff, and the inverse weight of
  // Tn2 is gated on lambda1[connect2] (:136-142).
  void bond(const Ten& Tn1, const Ten& Tn2, const Weights& lambda1, const Weights& lambda2, int connect1, Ten& n1,
            Ten& n2, std::vector<double>& lambda_c) {
    const int connect2 = (connect1 + 2) % 4;
    const Ten M1 = boundary(Tn1, lambda1, connect1);
    const Ten M2 = boundary(Tn2, lambda2, connect2);
    std::vector<double> D1, D2;
    Ten U1, U2;
    bk.eigh_matrix(M1, D1, U1);
    bk.eigh_matrix(M2, D2, U2);
    std::vector<double> D1inv(D1.size()), D2inv(D2.size());
    for (size_t i = 0; i < D1.size(); ++i) {
      D1[i] = std::sqrt(D1[i]);
      D1inv[i] = 1.0 / D1[i];
    }
    for (size_t i = 0; i < D2.size(); ++i) {
      D2[i] = std::sqrt(D2[i]);
      D2inv[i] = 1.0 / D2[i];
    }
    const Ten U1s = bk.mulvec(bk.mulvec(U1, lambda1[static_cast<size_t>(connect1)], 0), D1, 1);
    const Ten U2s = bk.mulvec(bk.mulvec(U2, lambda2[static_cast<size_t>(connect2)], 0), D2, 1);
    Ten W1, W2;
    bk.svd_matrix(bk.td(bk.conj(U1s), bk.conj(U2s), {0}, {0}, 0), W1, lambda_c, W2);
    double norm = 0.0;
    for (size_t i = lambda_c.size(); i-- > 0;) norm += lambda_c[i] * lambda_c[i];
    norm = std::sqrt(norm);
    for (double& l : lambda_c) l = std::sqrt(l / norm);
    W1 = bk.mulvec(W1, D1inv, 0);
    W2 = bk.mulvec(W2, D2inv, 1);

    const Ten X1 = bk.td(U1, W1, {1}, {0}, 0);
    n1 = bk.td(bk.mulvec(Tn1, inv(lambda1[static_cast<size_t>(connect1)]), connect1), X1, {connect1}, {0}, 0);
    n1 = bk.mulvec(bk.tr(n1, back(connect1)), lambda_c, connect1);

    const auto& g = lambda1[static_cast<size_t>(connect2)];
    const auto& l2 = lambda2[static_cast<size_t>(connect2)];
    std::vector<double> inv2(l2.size());
    for (size_t i = 0; i < l2.size(); ++i) inv2[i] = g[i] > lambda_cut ? 1.0 / l2[i] : 0.0;
    const Ten X2 = bk.td(U2, W2, {1}, {1}, 0);
    n2 = bk.td(bk.mulvec(Tn2, inv2, connect2), X2, {connect2}, {0}, 0);
    n2 = bk.mulvec(bk.tr(n2, back(connect2)), lambda_c, connect2);
  }

  // max |eigenvalue - 1| of the boundary tensors of legs of dimension > 1
  // (the convergence check, simple_update.cpp:80-97)
  double score(const std::vector<Ten>& Tn, const std::vector<Weights>& lam, const std::vector<std::array<int, 4>>& vdim) {
    double s = 0.0;
    for (size_t site = 0; site < Tn.size(); ++site)
      for (int leg = 0; leg < 4; ++leg) {
        if (vdim[site][static_cast<size_t>(leg)] <= 1) continue;
        std::vector<double> w;
        Ten Z;
        bk.eigh_matrix(boundary(Tn[site], lam[site], leg), w, Z);
        for (double d : w) s = std::max(s, std::abs(d - 1.0));
      }
    return s;
  }

  // iTPS::fix_local_gauge (simple_update.cpp:49-101): sweeps over the bonds
  // (sites of parity +1 then -1; source legs 2 then 1) until the score is
  // below eps, at most maxiter sweeps.  neighbor(site, leg) and parity(site)
  // describe the lattice.  Returns the sweeps done; *out_score the last score.
  template <class Neighbor, class Parity>
  int run(std::vector<Ten>& Tn, std::vector<Weights>& lam, const std::vector<std::array<int, 4>>& vdim,
          Neighbor neighbor, Parity parity, int maxiter, double eps, double* out_score) {
    double s = NAN;
    for (int it = 0; it < maxiter; ++it) {
      for (int par : {1, -1})
        for (int sleg : {2, 1}) {
          const int tleg = (sleg + 2) % 4;
          for (size_t src = 0; src < Tn.size(); ++src) {
            const int si = static_cast<int>(src);
            if (parity(si) != par || vdim[src][static_cast<size_t>(sleg)] <= 1) continue;
            const size_t tgt = static_cast<size_t>(neighbor(si, sleg));
            Ten a, b;
            std::vector<double> lc;
            bond(Tn[src], Tn[tgt], lam[src], lam[tgt], sleg, a, b, lc);
            lam[src][static_cast<size_t>(sleg)] = lc;
            lam[tgt][static_cast<size_t>(tleg)] = lc;
            Tn[src] = a;
            Tn[tgt] = b;
          }
        }
      s = score(Tn, lam, vdim);
      if (s < eps) {
        if (out_score) *out_score = s;
        return it + 1;
      }
    }
    if (out_score) *out_score = s;
    return maxiter;
  }
};

}  // namespace gauge
}  // namespace tg
