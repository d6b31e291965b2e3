// Full update of one bond (core::Full_update_bond, src/iTPS/core/full_update.cpp:31-455)
// over a tensor backend BK, real or complex tensors (BK::Scalar).
//
// The bond (Tn1 leg 2 -- Tn2 leg 0 after rotation) is updated by:
//   1. QR splits Tn1 = Q1 R1 over (0,1,3 | 2,4), Tn2 = Q2 R2 over (1,2,3 | 0,4);
//   2. Theta = (R1 R2) op12;
//   3. the bond environment of Q1, Q2 in the CTM environment
//      (Create_Environment_two_sites, :50-83), Hermitised, made positive by an
//      eigendecomposition that drops eigenvalues at or below Inverse_Env_cut
//      of the largest, and (Full_Gauge_Fix) brought to a gauge where its
//      square root is orthonormal through two QRs and their pseudo-inverses;
//   4. an initial R1, R2 from the SVD of Theta truncated to the bond
//      dimension, then alternating least squares R1 <- N1^+ W1, R2 <- N2^+ W2
//      (pseudo-inverses of the Hermitian normal matrices by SVD, cut at
//      Full_Inverse_precision) until the cost changes by less than
//      Full_Convergence_Epsilon of <Theta|E|Theta> or Full_max_iteration;
//   5. the gauge removed, R1, R2 balanced through QR + SVD of r1 r2^T with the
//      bond weights normalised, and the new tensors put back together.
//
// The backend supplies tensordot / transpose / reshape / conj / axpy / scale,
// leg slicing and scaling by host vectors, and thin matrix QR, SVD and
// Hermitian eigendecomposition (ascending) of row-major matrices.  The
// result does not depend on the sign / phase conventions of these
// factorisations beyond a gauge on the updated bond.  Tests instantiate it
// on host tensors; no CUDA code in this header.
#pragma once

#include <cmath>
#include <complex>
#include <cstdint>
#include <utility>
#include <vector>

#include "common.hpp"

namespace tg {
namespace fu {

using Axes = std::vector<int>;

struct Params {
  double inverse_env_cut = 1e-12;      // Inverse_Env_cut
  double inverse_precision = 1e-12;    // Full_Inverse_precision
  double convergence_epsilon = 1e-6;   // Full_Convergence_Epsilon
  int max_iteration = 100;             // Full_max_iteration
  bool gauge_fix = true;               // Full_Gauge_Fix
};

struct Stats {
  int iterations = 0;
  bool converged = false;
};

template <class BK>
struct FullUpdate {
  using Ten = typename BK::Ten;
  using S = typename BK::Scalar;  // double or std::complex<double>
  BK& bk;
  Params p;

  Ten cj(const Ten& a) { return bk.conj(a); }

  Ten td(const Ten& a, const Ten& b, const Axes& x, const Axes& y) { return bk.td(a, b, x, y, 0); }
  Ten tr(const Ten& a, const Axes& q) { return bk.tr(a, q); }
  static int64_t prod(const Shape& s, const Axes& legs) {
    int64_t n = 1;
    for (int l : legs) n *= s[static_cast<size_t>(l)];
    return n;
  }
  // A as the matrix (rows | cols) and the shapes of the two groups
  Ten matrix(const Ten& A, const Axes& rows, const Axes& cols, Shape& rs, Shape& cs) {
    const Shape& s = BK::shape(A);
    Axes perm(rows);
    perm.insert(perm.end(), cols.begin(), cols.end());
    rs.clear();
    cs.clear();
    for (int l : rows) rs.push_back(s[static_cast<size_t>(l)]);
    for (int l : cols) cs.push_back(s[static_cast<size_t>(l)]);
    return bk.reshape(tr(A, perm), {prod(s, rows), prod(s, cols)});
  }
  static Shape cat(Shape a, const Shape& b) {
    a.insert(a.end(), b.begin(), b.end());
    return a;
  }
  // qr over (rows | cols): Q (rows..., k), R (k, cols...)
  std::pair<Ten, Ten> qr(const Ten& A, const Axes& rows, const Axes& cols) {
    Shape rs, cs;
    const Ten M = matrix(A, rows, cols, rs, cs);
    Ten Q, R;
    bk.qr_matrix(M, Q, R);
    const int64_t k = BK::shape(Q)[1];
    return {bk.reshape(Q, cat(rs, {k})), bk.reshape(R, cat({k}, cs))};
  }
  // svd over (rows | cols): U (rows..., k), s, VT (k, cols...)
  void svd(const Ten& A, const Axes& rows, const Axes& cols, Ten& U, std::vector<double>& s, Ten& VT) {
    Shape rs, cs;
    const Ten M = matrix(A, rows, cols, rs, cs);
    bk.svd_matrix(M, U, s, VT);
    const int64_t k = static_cast<int64_t>(s.size());
    U = bk.reshape(U, cat(rs, {k}));
    VT = bk.reshape(VT, cat({k}, cs));
  }
  // Hermitian eigendecomposition over (rows | cols): ascending w, Z (rows..., k)
  void eigh(const Ten& A, const Axes& rows, const Axes& cols, std::vector<double>& w, Ten& Z) {
    Shape rs, cs;
    const Ten M = matrix(A, rows, cols, rs, cs);
    bk.eigh_matrix(M, w, Z);
    Z = bk.reshape(Z, cat(rs, {static_cast<int64_t>(w.size())}));
  }
  S trace(const Ten& A, const Ten& B, const Axes& x, const Axes& y) { return bk.scalar(td(A, B, x, y)); }

  // the transposed pseudo-inverse conj(u s^-1) conj(vt) of A = u s vt (:158-184)
  Ten pinv_t(const Ten& A) {
    Ten u, vt;
    std::vector<double> s;
    bk.svd_matrix(A, u, s, vt);
    std::vector<double> si(s.size());
    for (size_t i = 0; i < s.size(); ++i) si[i] = s[i] / s[0] > p.inverse_env_cut ? 1.0 / s[i] : 0.0;
    return td(cj(bk.mulvec(u, si, 1)), cj(vt), {1}, {0});
  }

  // Create_Environment_two_sites (:50-83), legs (t1, t2, tc1, tc2)
  Ten environment(const Ten& C1, const Ten& C2, const Ten& C3, const Ten& C4, const Ten& eT1, const Ten& eT2,
                  const Ten& eT3, const Ten& eT4, const Ten& eT5, const Ten& eT6, const Ten& Q1, const Ten& Q2) {
    const Ten right =
        td(td(C2, eT2, {0}, {1}),
           td(td(td(td(C3, eT4, {1}, {0}), eT3, {0}, {1}), cj(Q2), {2, 5}, {3, 2}), Q2, {1, 3}, {3, 2}), {0, 2, 3},
           {1, 5, 3});
    const Ten left =
        td(td(C1, eT1, {1}, {0}),
           td(td(td(td(C4, eT6, {1}, {0}), eT5, {0}, {1}), cj(Q1), {2, 5}, {0, 2}), Q1, {1, 3}, {0, 2}), {0, 2, 3},
           {0, 4, 2});
    return tr(td(right, left, {0, 1}, {0, 1}), {3, 1, 2, 0});
  }

  // -2 <R1 R2|E|Theta> + <R1 R2|E|R1 R2> (:238-254)
  S delta(const Ten& E, const Ten& Theta, const Ten& R1, const Ten& R2) {
    const Ten ET = td(E, Theta, {0, 1}, {0, 1});
    const S a = trace(td(ET, cj(R2), {1, 3}, {0, 2}), cj(R1), {0, 1, 2}, {0, 2, 1});
    const S b = trace(R1, td(R2, td(E, td(cj(R1), cj(R2), {1}, {1}), {2, 3}, {0, 2}), {0, 2}, {1, 3}), {0, 1, 2},
                      {1, 0, 2});
    return S(-2.0) * a + b;
  }
  // R = N^+ W with N^+ the pseudo-inverse of the Hermitian normal matrix (:276-296)
  Ten solve(const Ten& N, const Ten& W) {
    Ten U, VT;
    std::vector<double> s;
    svd(N, {1, 3}, {0, 2}, U, s, VT);
    std::vector<double> si(s.size());
    for (size_t i = 0; i < s.size(); ++i) si[i] = s[i] / s[0] > p.inverse_precision ? 1.0 / s[i] : 0.0;
    const Ten Ninv = td(cj(bk.mulvec(U, si, 2)), cj(VT), {2}, {0});
    return td(Ninv, W, {0, 1}, {0, 2});
  }

  // Full_update_bond_horizontal (:85-389)
  Stats horizontal(const Ten& C1, const Ten& C2, const Ten& C3, const Ten& C4, const Ten& eT1, const Ten& eT2,
                   const Ten& eT3, const Ten& eT4, const Ten& eT5, const Ten& eT6, const Ten& Tn1, const Ten& Tn2,
                   const Ten& op12, Ten& Tn1_new, Ten& Tn2_new) {
    Stats st;
    const int64_t Dc = BK::shape(Tn1)[2];
    auto q1r1 = qr(Tn1, {0, 1, 3}, {2, 4});
    auto q2r2 = qr(Tn2, {1, 2, 3}, {0, 4});
    const Ten Q1 = q1r1.first, Q2 = q2r2.first;
    Ten R1 = q1r1.second, R2 = q2r2.second;
    const int64_t envR1 = BK::shape(R1)[0], envR2 = BK::shape(R2)[0];
    Ten Theta = td(td(R1, R2, {1}, {1}), op12, {1, 3}, {0, 1});
    Ten E = environment(C1, C2, C3, C4, eT1, eT2, eT3, eT4, eT5, eT6, Q1, tr(Q2, {3, 0, 1, 2}));
    {  // Hermitise
      Ten Et = cj(tr(E, {2, 3, 0, 1}));
      bk.axpy(Et, E, 1.0);
      bk.scale(Et, 0.5);
      E = Et;
    }
    std::vector<double> w;
    Ten Z;
    eigh(E, {0, 1}, {2, 3}, w, Z);
    const double wmax = std::fabs(w[static_cast<size_t>(envR1 * envR2 - 1)]);
    for (double& x : w) x = x / wmax > p.inverse_env_cut ? std::sqrt(x) : 0.0;
    Z = bk.mulvec(Z, w, 2);
    Ten LR1_inv, LR2_inv;
    if (p.gauge_fix) {
      const Ten LR1 = qr(Z, {2, 1}, {0}).second;
      const Ten LR2 = qr(Z, {2, 0}, {1}).second;
      Theta = td(LR1, td(LR2, Theta, {1}, {1}), {1}, {1});
      LR1_inv = pinv_t(LR1);
      LR2_inv = pinv_t(LR2);
      Z = td(td(Z, LR1_inv, {0}, {1}), LR2_inv, {0}, {1});
      E = td(Z, cj(Z), {0}, {0});
    } else {
      E = td(Z, cj(Z), {2}, {2});
    }
    // initial guess: SVD of Theta truncated to Dc, weights sqrt(s / |s|)
    Ten U, VT;
    std::vector<double> s;
    svd(Theta, {0, 2}, {1, 3}, U, s, VT);
    const int64_t k = static_cast<int64_t>(s.size());
    const int64_t kc = std::min<int64_t>(k, Dc);
    std::vector<double> lam(static_cast<size_t>(Dc), 0.0);
    double nrm = 0.0;
    for (int64_t i = 0; i < kc; ++i) {
      lam[static_cast<size_t>(i)] = s[static_cast<size_t>(i)];
      nrm += s[static_cast<size_t>(i)] * s[static_cast<size_t>(i)];
    }
    nrm = std::sqrt(nrm);
    for (double& x : lam) x = std::sqrt(x / nrm);
    U = bk.slice(U, 2, kc);
    VT = bk.slice(VT, 0, kc);
    U = bk.mulvec(U, std::vector<double>(lam.begin(), lam.begin() + kc), 2);
    VT = bk.mulvec(VT, std::vector<double>(lam.begin(), lam.begin() + kc), 0);
    R1 = tr(U, {0, 2, 1});   // (envR1, Dc, m1)
    R2 = tr(VT, {1, 0, 2});  // (envR2, Dc, m2)
    const S C_phi = trace(td(E, Theta, {0, 1}, {0, 1}), cj(Theta), {0, 1, 2, 3}, {0, 1, 2, 3});
    S old = delta(E, Theta, R1, R2);
    while (!st.converged && st.iterations < p.max_iteration) {
      Ten W = td(td(E, Theta, {0, 1}, {0, 1}), cj(R2), {1, 3}, {0, 2});
      Ten N = td(td(E, R2, {1}, {0}), cj(R2), {2, 4}, {0, 2});
      R1 = solve(N, W);
      W = td(td(E, Theta, {0, 1}, {0, 1}), cj(R1), {0, 2}, {0, 2});
      N = td(td(E, R1, {0}, {0}), cj(R1), {1, 4}, {0, 2});
      R2 = solve(N, W);
      const S d = delta(E, Theta, R1, R2);
      if (std::abs(old - d) / std::abs(C_phi) < p.convergence_epsilon) st.converged = true;
      old = d;
      ++st.iterations;
    }
    if (p.gauge_fix) {
      R1 = td(LR1_inv, R1, {0}, {0});
      R2 = td(LR2_inv, R2, {0}, {0});
    }
    // balancing and normalisation
    auto a = qr(R1, {0, 2}, {1});
    auto b = qr(R2, {0, 2}, {1});
    Ten u, vt;
    std::vector<double> sv;
    bk.svd_matrix(td(a.second, b.second, {1}, {1}), u, sv, vt);
    const int64_t nb = std::min<int64_t>(static_cast<int64_t>(sv.size()), Dc);
    double n2 = 0.0;
    for (int64_t i = 0; i < nb; ++i) n2 += sv[static_cast<size_t>(i)] * sv[static_cast<size_t>(i)];
    n2 = std::sqrt(n2);
    for (int64_t i = 0; i < nb; ++i) sv[static_cast<size_t>(i)] = std::sqrt(sv[static_cast<size_t>(i)] / n2);
    u = bk.mulvec(u, sv, 1);
    vt = bk.mulvec(vt, sv, 0);
    R1 = td(a.first, u, {2}, {0});
    R2 = td(b.first, vt, {2}, {1});
    Tn1_new = tr(td(Q1, R1, {3}, {0}), {0, 1, 4, 2, 3});
    Tn2_new = tr(td(Q2, R2, {3}, {0}), {4, 0, 1, 2, 3});
    (void)envR1;
    (void)envR2;
    return st;
  }

  // Full_update_bond (:391-455): the bond on leg connect1 of Tn1 rotated onto
  // the horizontal case and back
  Stats bond(const Ten& C1, const Ten& C2, const Ten& C3, const Ten& C4, const Ten& eT1, const Ten& eT2,
             const Ten& eT3, const Ten& eT4, const Ten& eT5, const Ten& eT6, const Ten& Tn1, const Ten& Tn2,
             const Ten& op12, int connect1, Ten& Tn1_new, Ten& Tn2_new) {
    static const Axes rot[4] = {{2, 3, 0, 1, 4}, {3, 0, 1, 2, 4}, {0, 1, 2, 3, 4}, {1, 2, 3, 0, 4}};
    static const Axes back[4] = {{2, 3, 0, 1, 4}, {1, 2, 3, 0, 4}, {0, 1, 2, 3, 4}, {3, 0, 1, 2, 4}};
    if (connect1 < 0 || connect1 > 3) fail(TG_E_INPUT, "full update: bond leg must be 0..3");
    Ten a, b;
    const Stats st = horizontal(C1, C2, C3, C4, eT1, eT2, eT3, eT4, eT5, eT6, tr(Tn1, rot[connect1]),
                                tr(Tn2, rot[connect1]), op12, a, b);
    Tn1_new = tr(a, back[connect1]);
    Tn2_new = tr(b, back[connect1]);
    return st;
  }
};

}  // namespace fu
}  // namespace tg
