// Reverse-mode differentiation of the CTMRG energy of real site tensors.
//
// The energy E = sum_t coeff_t <ops_t> / <1>_t is evaluated on the
// environment reached after a fixed number of CTMRG sweeps from the initial
// environment of the site tensors (full-SVD corner projectors), and dE/dTn is
// obtained by a hand-written reverse pass over a tape of the forward's
// primitives:
//
//   tensordot   adjoint: two tensordots with the incoming adjoint, permuted
//               back to the operands' leg order;
//   transpose   adjoint: the inverse permutation;
//   max-abs     c = a / max|a| (ctm.cpp:514-517, 550-551); adjoint
//   rescale     ga = gc / m - (gc . c) sign(a_*) e_* / m at the first maximum;
//   extend /    adjoint: slice / zero-pad back (environment initialisation,
//   slice       ctm.cpp:998-1012);
//   truncated   Uc = U_w diag(s^-1/2), VTc = diag(s^-1/2) VT_w (ctm.cpp:245-302);
//   SVD         adjoint of the thin SVD M = U S VT with Lorentzian-broadened
//               F_ij = (s_j^2 - s_i^2) / ((s_j^2 - s_i^2)^2 + eps (s_i^2 + s_j^2)^2)
//               (broadened relative to the pair's scale: an absolute eps
//               distorted every pair of small kept values once the matrix's
//               norm was small, e.g. the up/down projectors' M = R1 R2):
//               gM = U [diag(gs) + (F o (J - J^T)) S + S (F o (K - K^T))] VT
//                    + (1 - U U^T) gU S^-1 VT + U S^-1 gVT (1 - V V^T),
//               J = U^T gU, K = V^T gV.  U, S, V are the rank-r part of
//               the SVD (singular values above kRankTol s_0; the rest are
//               taken as exact zeros), so the last two terms carry the whole
//               null space and the result does not depend on how a solver
//               completes the singular vectors of vanishing values (the
//               zero-padded environments of the first sweeps have many).
//
// Memory: the sweeps are cut into segments of `checkpoint_every` sweeps; the
// forward keeps only the environment at each segment start, and the backward
// recomputes one segment at a time on a fresh tape, chaining the adjoint of
// the environment from segment to segment.  The live tape is one segment.
//
// Everything here is generic over a backend BK (tensor type and the
// primitives above): the library instantiates it with device tensors and
// sm_100a kernels (adjoint.cu); a host backend instantiates the same code for
// checks on the CPU.  No CUDA code in this header.
#pragma once

#include <algorithm>
#include <array>
#include <cstdint>
#include <map>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "common.hpp"
#include "lattice.hpp"

namespace tg {
namespace ad {

using Axes = std::vector<int>;

// One product term of the energy: <prod ops> on an nrow x ncol window whose
// source site sits at (source_row, source_col), row 0 on top (the geometry of
// tg_measure_window), divided by the same window without operators.
struct WindowTerm {
  int source = 0, nrow = 1, ncol = 1, source_row = 0, source_col = 0;
  std::vector<int> op_row, op_col;
  std::vector<std::vector<double>> ops;  // d x d each, row-major
  double coeff = 1.0;
};

struct Options {
  int chi = 0;
  double cutoff = 1e-12;   // Inverse_projector_cut
  double eps = 1e-12;      // Lorentzian broadening of the SVD adjoint
  int iterations = 0;      // CTMRG sweeps after the initialisation
  int checkpoint_every = 5;
  int prec_absorb = 0;     // product precision of the moves (0 FP64, 1 3xTF32)
  bool projector_corner = true;  // Calc_projector_left_block, else Calc_projector_updown_blocks
};

// Singular values at or below kRankTol times the largest count as zero in
// the SVD adjoint.  Dropping their F terms changes the result by O(s_j / s_i)
// against the kept values; in exchange the adjoint reads no singular vector
// whose direction a Jacobi solver fixes only to eps s_0 / s_j.
constexpr double kRankTol = 1e-10;

inline bool identity_perm(const Axes& p) {
  for (size_t i = 0; i < p.size(); ++i)
    if (p[i] != static_cast<int>(i)) return false;
  return true;
}
inline Axes inverse_perm(const Axes& p) {
  Axes q(p.size());
  for (size_t i = 0; i < p.size(); ++i) q[static_cast<size_t>(p[i])] = static_cast<int>(i);
  return q;
}
inline Axes free_legs(int rank, const Axes& contracted) {
  Axes f;
  for (int i = 0; i < rank; ++i)
    if (std::find(contracted.begin(), contracted.end(), i) == contracted.end()) f.push_back(i);
  return f;
}
inline int position_in(const Axes& v, int x) {
  return static_cast<int>(std::find(v.begin(), v.end(), x) - v.begin());
}
// legs pos..pos+cnt-1 moved to the end / back
inline Axes moved_to_end(int rank, int pos, int cnt) {
  Axes p;
  for (int i = 0; i < rank; ++i)
    if (i < pos || i >= pos + cnt) p.push_back(i);
  for (int i = 0; i < cnt; ++i) p.push_back(pos + i);
  return p;
}
inline Axes moved_from_end(int rank, int pos, int cnt) {
  Axes p;
  const int keep = rank - cnt;
  for (int i = 0; i < rank; ++i) {
    if (i < pos) p.push_back(i);
    else if (i < pos + cnt) p.push_back(keep + (i - pos));
    else p.push_back(i - cnt);
  }
  return p;
}

// Adjoint permutations of c = tensordot(a, b, x, y) (legs of c: free legs of
// a, then free legs of b).  ga = transpose(tensordot(gc, b, [nA..], freeB), perm_a)
// and gb = transpose(tensordot(a, gc, freeA, [0..nA)), perm_b).
struct TdAdjoint {
  Axes freeA, freeB;
  Axes gc_free_b, gc_free_a;  // positions of c's legs that meet b's / a's free legs
  Axes perm_a, perm_b;
};
inline TdAdjoint td_adjoint(int ra, int rb, const Axes& x, const Axes& y) {
  TdAdjoint r;
  r.freeA = free_legs(ra, x);
  r.freeB = free_legs(rb, y);
  const int nA = static_cast<int>(r.freeA.size()), nB = static_cast<int>(r.freeB.size());
  const int nx = static_cast<int>(x.size());
  for (int i = 0; i < nB; ++i) r.gc_free_b.push_back(nA + i);
  for (int i = 0; i < nA; ++i) r.gc_free_a.push_back(i);
  // tensordot(gc, b, gc_free_b, freeB): legs = freeA (of c) ++ b's contracted legs, ascending
  Axes remB = y;
  std::sort(remB.begin(), remB.end());
  r.perm_a.assign(static_cast<size_t>(ra), 0);
  for (int i = 0; i < nA; ++i) r.perm_a[static_cast<size_t>(r.freeA[i])] = i;
  for (int j = 0; j < nx; ++j) r.perm_a[static_cast<size_t>(x[j])] = nA + position_in(remB, y[j]);
  // tensordot(a, gc, freeA, gc_free_a): legs = a's contracted legs, ascending ++ freeB
  Axes remA = x;
  std::sort(remA.begin(), remA.end());
  r.perm_b.assign(static_cast<size_t>(rb), 0);
  for (int i = 0; i < nB; ++i) r.perm_b[static_cast<size_t>(r.freeB[i])] = nx + i;
  for (int j = 0; j < nx; ++j) r.perm_b[static_cast<size_t>(y[j])] = position_in(remA, x[j]);
  return r;
}

template <class BK>
class Tape {
 public:
  using Ten = typename BK::Ten;
  enum class Kind { Leaf, Const, Td, Tr, Reshape, Norm, Fit, Svd, SvdU, SvdVT };
  struct Node {
    Kind kind = Kind::Const;
    bool need = false;  // depends on a differentiable leaf
    Ten v, g;
    int a = -1, b = -1;
    Axes x, y;
    int prec = 0;
    int64_t d1 = 0, d2 = 0, rest = 0, chi = 0;     // Fit
    Ten U, s, VT, sinv, gUc, gVTc;                // Svd
    int64_t m = 0, n = 0, k = 0, w = 0;
  };

  BK& bk;
  double eps = 1e-12;
  std::vector<Node> nodes;

  explicit Tape(BK& b) : bk(b) {}

  const Ten& val(int i) const { return nodes[static_cast<size_t>(i)].v; }
  const Shape& shape(int i) const { return BK::shape(val(i)); }
  int rank(int i) const { return static_cast<int>(shape(i).size()); }
  int64_t dim(int i, int l) const { return shape(i)[static_cast<size_t>(l)]; }
  bool need(int i) const { return nodes[static_cast<size_t>(i)].need; }
  const Ten& grad(int i) const { return nodes[static_cast<size_t>(i)].g; }

  int leaf(const Ten& v, bool differentiable) {
    Node nd;
    nd.kind = differentiable ? Kind::Leaf : Kind::Const;
    nd.need = differentiable;
    nd.v = v;
    return push(std::move(nd));
  }
  int td(int a, int b, const Axes& x, const Axes& y, int prec = 0) {
    Node nd;
    nd.kind = Kind::Td;
    nd.a = a;
    nd.b = b;
    nd.x = x;
    nd.y = y;
    nd.prec = prec;
    nd.need = need(a) || need(b);
    nd.v = bk.td(val(a), val(b), x, y, prec);
    return push(std::move(nd));
  }
  int tr(int a, const Axes& p) {
    if (identity_perm(p)) return a;
    Node nd;
    nd.kind = Kind::Tr;
    nd.a = a;
    nd.x = p;
    nd.need = need(a);
    nd.v = bk.tr(val(a), p);
    return push(std::move(nd));
  }
  int reshape(int a, const Shape& s) {
    if (s == shape(a)) return a;
    Node nd;
    nd.kind = Kind::Reshape;
    nd.a = a;
    nd.need = need(a);
    nd.v = bk.reshape(val(a), s);
    return push(std::move(nd));
  }
  int normalize(int a) {
    Node nd;
    nd.kind = Kind::Norm;
    nd.a = a;
    nd.need = need(a);
    nd.v = bk.normalize(val(a));
    return push(std::move(nd));
  }
  // out(chi, chi, rest...) = zero-padded / sliced a viewed as (d1, d2, rest)
  int fit(int a, int64_t d1, int64_t d2, int64_t rest, const Shape& out) {
    Node nd;
    nd.kind = Kind::Fit;
    nd.a = a;
    nd.d1 = d1;
    nd.d2 = d2;
    nd.rest = rest;
    nd.chi = out[0];
    nd.need = need(a);
    nd.v = bk.fit(val(a), d1, d2, rest, out);
    return push(std::move(nd));
  }
  // truncated factors (Uc, VTc) of the m x n matrix M
  std::pair<int, int> svd(int M, int chi, double cutoff) {
    Node nd;
    nd.kind = Kind::Svd;
    nd.a = M;
    nd.need = need(M);
    nd.m = dim(M, 0);
    nd.n = dim(M, 1);
    nd.k = std::min(nd.m, nd.n);
    nd.w = std::min<int64_t>(nd.k, chi);
    Ten Uc, VTc;
    bk.svd_trunc(val(M), nd.m, nd.n, chi, cutoff, nd.U, nd.s, nd.VT, nd.sinv, Uc, VTc);
    const bool nd_need = nd.need;
    const int id = push(std::move(nd));
    Node u;
    u.kind = Kind::SvdU;
    u.a = id;
    u.need = nd_need;
    u.v = Uc;
    const int iu = push(std::move(u));
    Node vt;
    vt.kind = Kind::SvdVT;
    vt.a = id;
    vt.need = nd_need;
    vt.v = VTc;
    const int iv = push(std::move(vt));
    return {iu, iv};
  }

  // g_i += t
  void seed(int i, const Ten& t) { acc(i, t); }

  // Reverse pass over the whole tape.  Values and adjoints of interior nodes
  // are released as soon as they have been propagated; leaves keep theirs.
  void backward() {
    for (int i = static_cast<int>(nodes.size()) - 1; i >= 0; --i) {
      Node& nd = nodes[static_cast<size_t>(i)];
      if (nd.kind == Kind::Leaf || nd.kind == Kind::Const) continue;
      if (!nd.need) {
        release(nd);
        continue;
      }
      switch (nd.kind) {
        case Kind::Svd:
          if (!BK::empty(nd.gUc) || !BK::empty(nd.gVTc)) svd_backward(i);
          break;
        case Kind::Td:
          if (!BK::empty(nd.g)) td_backward(i);
          break;
        case Kind::Tr:
          if (!BK::empty(nd.g)) acc(nd.a, bk.tr(nd.g, inverse_perm(nd.x)));
          break;
        case Kind::Reshape:
          if (!BK::empty(nd.g)) acc(nd.a, bk.reshape(nd.g, shape(nd.a)));
          break;
        case Kind::Norm:
          if (!BK::empty(nd.g)) acc(nd.a, bk.normalize_bwd(val(nd.a), nd.v, nd.g));
          break;
        case Kind::Fit:
          if (!BK::empty(nd.g)) acc(nd.a, bk.unfit(nd.g, nd.d1, nd.d2, nd.rest, nd.chi, shape(nd.a)));
          break;
        case Kind::SvdU:
          if (!BK::empty(nd.g)) acc_into(nodes[static_cast<size_t>(nd.a)].gUc, nd.g);
          break;
        case Kind::SvdVT:
          if (!BK::empty(nd.g)) acc_into(nodes[static_cast<size_t>(nd.a)].gVTc, nd.g);
          break;
        default:
          break;
      }
      release(nodes[static_cast<size_t>(i)]);
    }
  }

 private:
  int push(Node&& nd) {
    nodes.push_back(std::move(nd));
    return static_cast<int>(nodes.size()) - 1;
  }
  void release(Node& nd) {
    nd.v = Ten();
    nd.g = Ten();
    nd.U = Ten();
    nd.s = Ten();
    nd.VT = Ten();
    nd.sinv = Ten();
    nd.gUc = Ten();
    nd.gVTc = Ten();
  }
  void acc_into(Ten& g, const Ten& t) {
    if (BK::empty(g)) g = t;
    else bk.axpy(g, t, 1.0);
  }
  void acc(int i, const Ten& t) {
    Node& nd = nodes[static_cast<size_t>(i)];
    if (!nd.need) return;
    if (BK::shape(t) != BK::shape(nd.v)) acc_into(nd.g, bk.reshape(t, BK::shape(nd.v)));
    else acc_into(nd.g, t);
  }
  void td_backward(int i) {
    const Node& nd = nodes[static_cast<size_t>(i)];
    const int a = nd.a, b = nd.b, prec = nd.prec;
    const TdAdjoint r = td_adjoint(rank(a), rank(b), nd.x, nd.y);
    const Ten gc = nd.g;
    if (need(a)) {
      Ten t = bk.td(gc, val(b), r.gc_free_b, r.freeB, prec);
      acc(a, identity_perm(r.perm_a) ? t : bk.tr(t, r.perm_a));
    }
    if (need(b)) {
      Ten t = bk.td(val(a), gc, r.freeA, r.gc_free_a, prec);
      acc(b, identity_perm(r.perm_b) ? t : bk.tr(t, r.perm_b));
    }
  }
  void svd_backward(int i) {
    const Node& nd = nodes[static_cast<size_t>(i)];
    const int64_t m = nd.m, n = nd.n, k = nd.k, w = nd.w;
    const Ten gUc = BK::empty(nd.gUc) ? bk.zeros({m, w}) : nd.gUc;
    const Ten gVTc = BK::empty(nd.gVTc) ? bk.zeros({w, n}) : nd.gVTc;
    Ten gU, gVT, gs;
    bk.svd_prep(gUc, gVTc, nd.U, nd.VT, nd.sinv, m, n, k, w, gU, gVT, gs);
    // rank-r factors: columns of U / rows of VT of vanishing values zeroed
    Ten U, VT;
    bk.svd_rank_mask(nd.U, nd.VT, nd.s, kRankTol, U, VT);
    const Ten J = bk.td(U, gU, {0}, {0}, 0);    // U^T gU  (k x k)
    const Ten K = bk.td(VT, gVT, {1}, {1}, 0);  // V^T gV  (k x k)
    const Ten core = bk.svd_core(J, K, nd.s, gs, k, eps);
    Ten gM = bk.td(bk.td(U, core, {1}, {0}, 0), VT, {1}, {0}, 0);
    // (1 - U U^T) gU S^-1 VT
    Ten P = bk.td(U, J, {1}, {0}, 0);
    bk.axpy(P, gU, -1.0);
    bk.scale_cols_sq(P, nd.sinv, w);
    bk.axpy(gM, bk.td(P, VT, {1}, {0}, 0), -1.0);
    // U S^-1 gVT (1 - V V^T)
    Ten Q = bk.td(bk.td(gVT, VT, {1}, {1}, 0), VT, {1}, {0}, 0);
    bk.axpy(Q, gVT, -1.0);
    bk.scale_rows_sq(Q, nd.sinv, w);
    bk.axpy(gM, bk.td(U, Q, {1}, {0}, 0), -1.0);
    acc(nd.a, gM);
  }
};

// The CTMRG forward of ctm.cpp on a tape: environment initialisation, the
// four moves with full-SVD corner or up/down projectors, and window
// contractions.
// Environment tensors are zero-padded to chi as in the library's environment.
template <class BK>
struct CtmTape {
  using TP = Tape<BK>;
  using Ten = typename BK::Ten;
  TP& t;
  const Lattice& lat;
  Options o;
  std::vector<int> Tn;                     // leaf ids
  std::vector<std::array<int, 3>> rotc;    // rotated site tensors (right, top, bottom)
  std::array<std::vector<int>, 4> C, E;    // C1..C4; eTt, eTr, eTb, eTl
  std::map<std::tuple<int, int, int, int>, int> et_memo;

  CtmTape(TP& tp, const Lattice& l, const Options& opt) : t(tp), lat(l), o(opt) {}

  void set_sites(const std::vector<Ten>& T, bool differentiable) {
    Tn.clear();
    for (const Ten& x : T) Tn.push_back(t.leaf(x, differentiable));
    rotc.assign(T.size(), {-1, -1, -1});
  }
  void set_env(const std::array<std::vector<Ten>, 4>& Cv, const std::array<std::vector<Ten>, 4>& Ev,
               bool differentiable) {
    for (int w = 0; w < 4; ++w) {
      C[w].clear();
      E[w].clear();
      for (const Ten& x : Cv[w]) C[w].push_back(t.leaf(x, differentiable));
      for (const Ten& x : Ev[w]) E[w].push_back(t.leaf(x, differentiable));
    }
  }

  // Tn rotated for the right / top / bottom moves (ctm.cpp:642, 707, 773)
  int rot(int site, int w) {
    static const Axes perms[3] = {{2, 3, 0, 1, 4}, {1, 2, 3, 0, 4}, {3, 0, 1, 2, 4}};
    int& r = rotc[static_cast<size_t>(site)][static_cast<size_t>(w)];
    if (r < 0) r = t.tr(Tn[static_cast<size_t>(site)], perms[w]);
    return r;
  }

  // ------------------------------------------------------ initialisation
  int fit_corner(int X) {
    const int64_t chi = o.chi;
    return t.fit(X, t.dim(X, 0) * t.dim(X, 1), t.dim(X, 2) * t.dim(X, 3), 1, {chi, chi});
  }
  int fit_edge(int X) {
    const int64_t chi = o.chi;
    return t.fit(X, t.dim(X, 0) * t.dim(X, 1), t.dim(X, 2) * t.dim(X, 3), t.dim(X, 4) * t.dim(X, 5),
                 {chi, chi, t.dim(X, 4), t.dim(X, 5)});
  }
  // ctm.cpp:984-1193 (real tensors: conj(Tn) = Tn)
  void init() {
    const int N = lat.N;
    for (int w = 0; w < 4; ++w) {
      C[w].assign(static_cast<size_t>(N), -1);
      E[w].assign(static_cast<size_t>(N), -1);
    }
    for (int i = 0; i < N; ++i) {
      int s = Tn[static_cast<size_t>(lat.top(lat.left(i)))];
      C[0][i] = fit_corner(t.tr(t.td(s, s, {0, 1, 4}, {0, 1, 4}), {1, 3, 0, 2}));
      s = Tn[static_cast<size_t>(lat.top(lat.right(i)))];
      C[1][i] = fit_corner(t.tr(t.td(s, s, {1, 2, 4}, {1, 2, 4}), {0, 2, 1, 3}));
      s = Tn[static_cast<size_t>(lat.bottom(lat.right(i)))];
      C[2][i] = fit_corner(t.tr(t.td(s, s, {2, 3, 4}, {2, 3, 4}), {1, 3, 0, 2}));
      s = Tn[static_cast<size_t>(lat.bottom(lat.left(i)))];
      C[3][i] = fit_corner(t.tr(t.td(s, s, {0, 3, 4}, {0, 3, 4}), {1, 3, 0, 2}));
      s = Tn[static_cast<size_t>(lat.top(i))];
      E[0][i] = fit_edge(t.tr(t.td(s, s, {1, 4}, {1, 4}), {0, 3, 1, 4, 2, 5}));
      s = Tn[static_cast<size_t>(lat.right(i))];
      E[1][i] = fit_edge(t.tr(t.td(s, s, {2, 4}, {2, 4}), {1, 4, 2, 5, 0, 3}));
      s = Tn[static_cast<size_t>(lat.bottom(i))];
      E[2][i] = fit_edge(t.tr(t.td(s, s, {3, 4}, {3, 4}), {2, 5, 0, 3, 1, 4}));
      s = Tn[static_cast<size_t>(lat.left(i))];
      E[3][i] = fit_edge(t.tr(t.td(s, s, {0, 4}, {0, 4}), {2, 5, 0, 3, 1, 4}));
    }
  }

  // ---------------------------------------------------------- CTM pieces
  int block_LT(int C1, int eT1, int eT8, int T1) {  // ctm.cpp:207-212
    const int p = o.prec_absorb;
    const int X = t.td(t.td(t.td(C1, eT1, {1}, {0}, p), eT8, {0}, {1}, p), T1, {2, 5}, {1, 0}, p);
    return t.td(T1, X, {0, 1, 4}, {3, 1, 6}, p);
  }
  int block_LB(int C4, int eT7, int eT6, int T4) {  // ctm.cpp:222-227
    const int p = o.prec_absorb;
    const int X = t.td(t.td(t.td(C4, eT7, {1}, {0}, p), eT6, {0}, {1}, p), T4, {2, 5}, {0, 3}, p);
    return t.td(T4, X, {0, 3, 4}, {1, 3, 6}, p);
  }
  // Calc_projector_left_block, full-SVD branch (ctm.cpp:174-318)
  void projector(int C1, int C4, int eT1, int eT6, int eT7, int eT8, int T1, int T4, int& PU, int& PL) {
    const int p = o.prec_absorb;
    const int64_t e12 = t.dim(eT1, 1), e56 = t.dim(eT6, 0), e78 = t.dim(eT8, 0);
    const int64_t t12 = t.dim(T1, 2), t41 = t.dim(T1, 3), t34 = t.dim(T4, 2);
    if (t41 == 1) {  // identity projector (ctm.cpp:303-317)
      PU = PL = t.leaf(t.bk.identity_projector(e78), false);
      return;
    }
    const int64_t nrow = t12 * e12 * t12, nmid = t41 * e78 * t41, ncol = t34 * e56 * t34;
    const int LTm = t.reshape(t.tr(block_LT(C1, eT1, eT8, T1), {0, 2, 4, 1, 3, 5}), {nrow, nmid});
    const int LBm = t.reshape(t.tr(block_LB(C4, eT7, eT6, T4), {0, 2, 4, 1, 3, 5}), {nmid, ncol});
    const int M = t.td(LTm, LBm, {1}, {0}, p);
    const std::pair<int, int> f = t.svd(M, o.chi, o.cutoff);
    const int64_t w = t.dim(f.first, 1);
    // PU = LB conj(VT_c)^T, PL = LT^T conj(U_c), legs (e78, t41, tc41, w) (ctm.cpp:263-266, 298-302)
    PU = t.tr(t.reshape(t.td(LBm, f.second, {1}, {1}, p), {t41, e78, t41, w}), {1, 0, 2, 3});
    PL = t.tr(t.reshape(t.td(LTm, f.first, {0}, {0}, p), {t41, e78, t41, w}), {1, 0, 2, 3});
  }
  // Calc_projector_updown_blocks, full-SVD branch (ctm.cpp:320-491): the
  // four corner blocks, R1 = RT LT and R2 = RB LB, the truncated SVD of
  // M = R1 R2 (its row legs are R1's first three, its column legs R2's),
  // PU = R2 conj(VT_c)^T and PL = R1 conj(U_c), legs (e78, t41, tc41, w)
  void projector_ud(int C1, int C2, int C3, int C4, int eT1, int eT2, int eT3, int eT4, int eT5, int eT6, int eT7,
                    int eT8, int T1, int T2, int T3, int T4, int& PU, int& PL) {
    const int p = o.prec_absorb;
    const int64_t e78 = t.dim(eT7, 1), t41 = t.dim(T4, 1);
    if (t41 == 1) {  // identity projector (ctm.cpp:479-490)
      PU = PL = t.leaf(t.bk.identity_projector(e78), false);
      return;
    }
    const int LT = block_LT(C1, eT1, eT8, T1);
    const int RT = t.td(T2, t.td(t.td(t.td(C2, eT3, {1}, {0}, p), eT2, {0}, {1}, p), T2, {2, 5}, {2, 1}, p),
                        {1, 2, 4}, {3, 1, 6}, p);
    const int RB = t.td(T3, t.td(t.td(t.td(C3, eT5, {1}, {0}, p), eT4, {0}, {1}, p), T3, {2, 5}, {3, 2}, p),
                        {2, 3, 4}, {3, 1, 6}, p);
    const int LB = block_LB(C4, eT7, eT6, T4);
    const int R1 = t.td(RT, LT, {0, 3, 4}, {0, 2, 4}, p);
    const int R2 = t.td(RB, LB, {0, 2, 4}, {1, 3, 5}, p);
    const int64_t nrow = t.dim(R1, 0) * t.dim(R1, 1) * t.dim(R1, 2);
    const int64_t ncol = t.dim(R2, 0) * t.dim(R2, 1) * t.dim(R2, 2);
    const int64_t a3 = t.dim(R1, 3), a4 = t.dim(R1, 4), a5 = t.dim(R1, 5);
    const int64_t b3 = t.dim(R2, 3), b4 = t.dim(R2, 4), b5 = t.dim(R2, 5);
    const int R1m = t.reshape(R1, {nrow, a3 * a4 * a5});
    const int R2m = t.reshape(R2, {ncol, b3 * b4 * b5});
    const int M = t.td(R1m, R2m, {1}, {1}, p);
    const std::pair<int, int> f = t.svd(M, o.chi, o.cutoff);
    const int64_t w = t.dim(f.first, 1);
    PU = t.tr(t.reshape(t.td(R2m, f.second, {0}, {1}, p), {b3, b4, b5, w}), {1, 0, 2, 3});
    PL = t.tr(t.reshape(t.td(R1m, f.first, {0}, {0}, p), {a3, a4, a5, w}), {1, 0, 2, 3});
  }
  // Calc_Next_CTM (ctm.cpp:493-518)
  std::pair<int, int> next_ctm(int C1, int C4, int eT1, int eT6, int PU, int PL) {
    const int p = o.prec_absorb;
    const int a = t.normalize(t.td(PU, t.td(C1, eT1, {1}, {0}, p), {0, 1, 2}, {0, 2, 3}, p));
    const int b = t.normalize(t.td(t.td(eT6, C4, {1}, {0}, p), PL, {3, 1, 2}, {0, 1, 2}, p));
    return {a, b};
  }
  // Calc_Next_eT (ctm.cpp:520-552); a job repeated with the same inputs
  // within a move (rows iy and iy-1 share one edge) is computed once
  int next_et(int eT8, int T1, int PU, int PL) {
    const auto key = std::make_tuple(eT8, T1, PU, PL);
    auto it = et_memo.find(key);
    if (it != et_memo.end()) return it->second;
    const int p = o.prec_absorb;
    int X = t.td(T1, t.td(eT8, PL, {1}, {0}, p), {0, 1}, {2, 4}, p);
    X = t.td(T1, X, {0, 1, 4}, {4, 5, 2}, p);
    const int r = t.normalize(t.tr(t.td(X, PU, {1, 3, 4}, {1, 2, 0}, p), {3, 2, 0, 1}));
    et_memo[key] = r;
    return r;
  }

  // ------------------------------------------------------------- moves
  // The index rules of Left_move / Right_move / Top_move / Bottom_move
  // (ctm.cpp:562-813): all projectors of the line from the current
  // environment, then the new tensors from a snapshot of it.
  void left_move(int ix) {
    const int L = lat.LY_noskew;
    std::vector<int> PU(L), PL(L);
    for (int iy = 0; iy < L; ++iy) {
      const int i = lat.index(ix, iy), j = lat.right(i), k = lat.bottom(j), l = lat.left(k);
      if (o.projector_corner)
        projector(C[0][i], C[3][l], E[0][i], E[2][l], E[3][l], E[3][i], Tn[i], Tn[l], PU[iy], PL[iy]);
      else
        projector_ud(C[0][i], C[1][j], C[2][k], C[3][l], E[0][i], E[0][j], E[1][j], E[1][k], E[2][k], E[2][l],
                     E[3][l], E[3][i], Tn[i], Tn[j], Tn[k], Tn[l], PU[iy], PL[iy]);
    }
    const auto C0 = C, E0 = E;
    et_memo.clear();
    for (int iy = 0; iy < L; ++iy) {
      const int i = lat.index(ix, iy), j = lat.right(i), k = lat.bottom(j), l = lat.left(k);
      const int up = (iy + 1) % L, dn = (iy - 1 + L) % L;
      const auto c = next_ctm(C0[0][i], C0[3][l], E0[0][i], E0[2][l], PU[up], PL[dn]);
      C[0][j] = c.first;
      C[3][k] = c.second;
      E[3][j] = next_et(E0[3][i], Tn[i], PU[iy], PL[up]);
      E[3][k] = next_et(E0[3][l], Tn[l], PU[dn], PL[iy]);
    }
  }
  void right_move(int ix) {
    const int L = lat.LY_noskew;
    std::vector<int> PU(L), PL(L);
    for (int iy = 0; iy < L; ++iy) {
      const int k = lat.index(ix, iy), l = lat.left(k), i = lat.top(l), j = lat.right(i);
      if (o.projector_corner)
        projector(C[2][k], C[1][j], E[2][k], E[0][j], E[1][j], E[1][k], rot(k, 0), rot(j, 0), PU[iy], PL[iy]);
      else
        projector_ud(C[2][k], C[3][l], C[0][i], C[1][j], E[2][k], E[2][l], E[3][l], E[3][i], E[0][i], E[0][j],
                     E[1][j], E[1][k], rot(k, 0), rot(l, 0), rot(i, 0), rot(j, 0), PU[iy], PL[iy]);
    }
    const auto C0 = C, E0 = E;
    et_memo.clear();
    for (int iy = 0; iy < L; ++iy) {
      const int k = lat.index(ix, iy), l = lat.left(k), i = lat.top(l), j = lat.right(i);
      const int up = (iy + 1) % L, dn = (iy - 1 + L) % L;
      const auto c = next_ctm(C0[2][k], C0[1][j], E0[2][k], E0[0][j], PU[dn], PL[up]);
      C[2][l] = c.first;
      C[1][i] = c.second;
      E[1][l] = next_et(E0[1][k], rot(k, 0), PU[iy], PL[dn]);
      E[1][i] = next_et(E0[1][j], rot(j, 0), PU[up], PL[iy]);
    }
  }
  void top_move(int iy) {
    const int L = lat.LX_noskew;
    std::vector<int> PU(L), PL(L);
    for (int ix = 0; ix < L; ++ix) {
      const int j = lat.index(ix, iy), k = lat.bottom(j), l = lat.left(k), i = lat.top(l);
      if (o.projector_corner)
        projector(C[1][j], C[0][i], E[1][j], E[3][i], E[0][i], E[0][j], rot(j, 1), rot(i, 1), PU[ix], PL[ix]);
      else
        projector_ud(C[1][j], C[2][k], C[3][l], C[0][i], E[1][j], E[1][k], E[2][k], E[2][l], E[3][l], E[3][i],
                     E[0][i], E[0][j], rot(j, 1), rot(k, 1), rot(l, 1), rot(i, 1), PU[ix], PL[ix]);
    }
    const auto C0 = C, E0 = E;
    et_memo.clear();
    for (int ix = 0; ix < L; ++ix) {
      const int j = lat.index(ix, iy), k = lat.bottom(j), l = lat.left(k), i = lat.top(l);
      const int rt = (ix + 1) % L, lf = (ix - 1 + L) % L;
      const auto c = next_ctm(C0[1][j], C0[0][i], E0[1][j], E0[3][i], PU[rt], PL[lf]);
      C[1][k] = c.first;
      C[0][l] = c.second;
      E[0][k] = next_et(E0[0][j], rot(j, 1), PU[ix], PL[rt]);
      E[0][l] = next_et(E0[0][i], rot(i, 1), PU[lf], PL[ix]);
    }
  }
  void bottom_move(int iy) {
    const int L = lat.LX_noskew;
    std::vector<int> PU(L), PL(L);
    for (int ix = 0; ix < L; ++ix) {
      const int l = lat.index(ix, iy), i = lat.top(l), j = lat.right(i), k = lat.bottom(j);
      if (o.projector_corner)
        projector(C[3][l], C[2][k], E[3][l], E[1][k], E[2][k], E[2][l], rot(l, 2), rot(k, 2), PU[ix], PL[ix]);
      else
        projector_ud(C[3][l], C[0][i], C[1][j], C[2][k], E[3][l], E[3][i], E[0][i], E[0][j], E[1][j], E[1][k],
                     E[2][k], E[2][l], rot(l, 2), rot(i, 2), rot(j, 2), rot(k, 2), PU[ix], PL[ix]);
    }
    const auto C0 = C, E0 = E;
    et_memo.clear();
    for (int ix = 0; ix < L; ++ix) {
      const int l = lat.index(ix, iy), i = lat.top(l), j = lat.right(i), k = lat.bottom(j);
      const int rt = (ix + 1) % L, lf = (ix - 1 + L) % L;
      const auto c = next_ctm(C0[3][l], C0[2][k], E0[3][l], E0[1][k], PU[lf], PL[rt]);
      C[3][i] = c.first;
      C[2][j] = c.second;
      E[2][i] = next_et(E0[2][l], rot(l, 2), PU[ix], PL[lf]);
      E[2][j] = next_et(E0[2][k], rot(k, 2), PU[rt], PL[ix]);
    }
  }
  // one CTMRG iteration, in the order of ctm.cpp:1205-1228
  void sweep() {
    const int LX = lat.LX_noskew, LY = lat.LY_noskew;
    for (int ix = 0; ix < LX; ++ix) left_move(ix);
    for (int ix = 0; ix > -LX; --ix) right_move((ix + 1 + LX) % LX);
    for (int iy = 0; iy > -LY; --iy) top_move((iy + 1 + LY) % LY);
    for (int iy = 0; iy < LY; ++iy) bottom_move(iy);
  }

  // ---------------------------------------------------- window <ops...>
  // Contract_RxC_iTPS_CTM (contract_itps_ctm/ctm.cpp:45-87) row by row
  // through a boundary tensor (a, k0, kb0, ..., r); ops[r*ncol + c] is the
  // id of that site's operator (-1: identity), applied as
  // sum_{p,q} Tn[..p] op[p,q] Tn[..q].
  int window(int source, int nrow, int ncol, int source_row, int source_col, const std::vector<int>& ops) {
    std::vector<std::vector<int>> idx(static_cast<size_t>(nrow), std::vector<int>(static_cast<size_t>(ncol)));
    for (int r = 0; r < nrow; ++r)
      for (int c = 0; c < ncol; ++c) idx[r][c] = lat.other(source, c - source_col, source_row - r);
    int B = C[0][idx[0][0]];
    for (int c = 0; c < ncol; ++c) {
      B = t.td(B, E[0][idx[0][c]], {t.rank(B) - 1}, {0});
      B = t.tr(B, moved_to_end(t.rank(B), t.rank(B) - 3, 1));
    }
    B = t.td(B, C[1][idx[0][ncol - 1]], {t.rank(B) - 1}, {0});
    for (int r = 0; r < nrow; ++r) {
      B = t.td(E[3][idx[r][0]], B, {1}, {0});
      for (int c = 0; c < ncol; ++c) {
        const int Tc = Tn[static_cast<size_t>(idx[r][c])];
        const int pos = 1 + 2 * c;
        B = t.tr(B, moved_to_end(t.rank(B), pos, 4));
        int n = t.rank(B);
        B = t.td(B, Tc, {n - 4, n - 2}, {0, 1});
        const int op = ops[static_cast<size_t>(r * ncol + c)];
        if (op >= 0) B = t.td(B, op, {t.rank(B) - 1}, {0});
        n = t.rank(B);
        B = t.td(B, Tc, {n - 5, n - 4, n - 1}, {0, 1, 4});
        n = t.rank(B);
        Axes p;
        for (int q = 0; q < n - 4; ++q) p.push_back(q);
        p.insert(p.end(), {n - 3, n - 1, n - 4, n - 2});
        B = t.tr(B, p);
        B = t.tr(B, moved_from_end(t.rank(B), pos, 4));
      }
      const int n = t.rank(B);
      B = t.td(B, E[1][idx[r][ncol - 1]], {n - 1, n - 3, n - 2}, {0, 2, 3});
    }
    int X = t.td(C[3][idx[nrow - 1][0]], B, {1}, {0});
    for (int c = 0; c < ncol; ++c) X = t.td(E[2][idx[nrow - 1][c]], X, {1, 2, 3}, {0, 1, 2});
    return t.td(X, C[2][idx[nrow - 1][ncol - 1]], {0, t.rank(X) - 1}, {1, 0});
  }

  // Energy nodes: the value window of every term and the shared norm windows
  // (one per window geometry, as twosite_obs.cpp:160-181 caches them).
  struct EnergyNodes {
    std::vector<int> val, nrm_of_term, nrm;
    std::vector<double> v, nv;
    double E = 0.0;
  };
  EnergyNodes energy(const std::vector<WindowTerm>& terms) {
    EnergyNodes en;
    std::map<std::tuple<int, int, int, int, int>, int> norm_ids;
    for (const WindowTerm& w : terms) {
      std::vector<int> ops(static_cast<size_t>(w.nrow * w.ncol), -1);
      for (size_t q = 0; q < w.ops.size(); ++q) {
        const int r = w.op_row[q], c = w.op_col[q];
        const int site = lat.other(w.source, c - w.source_col, w.source_row - r);
        const int64_t d = lat.pdim[static_cast<size_t>(site)];
        ops[static_cast<size_t>(r * w.ncol + c)] = t.leaf(t.bk.from_host({d, d}, w.ops[q].data()), false);
      }
      const auto key = std::make_tuple(w.source, w.nrow, w.ncol, w.source_row, w.source_col);
      auto it = norm_ids.find(key);
      if (it == norm_ids.end()) {
        const int nid = window(w.source, w.nrow, w.ncol, w.source_row, w.source_col,
                               std::vector<int>(static_cast<size_t>(w.nrow * w.ncol), -1));
        it = norm_ids.emplace(key, static_cast<int>(en.nrm.size())).first;
        en.nrm.push_back(nid);
      }
      en.val.push_back(window(w.source, w.nrow, w.ncol, w.source_row, w.source_col, ops));
      en.nrm_of_term.push_back(it->second);
    }
    for (int id : en.nrm) en.nv.push_back(t.bk.scalar(t.val(id)));
    for (size_t q = 0; q < terms.size(); ++q) {
      en.v.push_back(t.bk.scalar(t.val(en.val[q])));
      en.E += terms[q].coeff * en.v[q] / en.nv[static_cast<size_t>(en.nrm_of_term[q])];
    }
    return en;
  }
  // dE/d(value) and dE/d(norm) as seeds of the reverse pass
  void seed_energy(const std::vector<WindowTerm>& terms, const EnergyNodes& en) {
    std::vector<double> gn(en.nrm.size(), 0.0);
    for (size_t q = 0; q < terms.size(); ++q) {
      const double nv = en.nv[static_cast<size_t>(en.nrm_of_term[q])];
      const double gv = terms[q].coeff / nv;
      t.seed(en.val[q], t.bk.from_host({}, &gv));
      gn[static_cast<size_t>(en.nrm_of_term[q])] -= terms[q].coeff * en.v[q] / (nv * nv);
    }
    for (size_t q = 0; q < en.nrm.size(); ++q) t.seed(en.nrm[q], t.bk.from_host({}, &gn[q]));
  }
};

// E and (when grads != nullptr) dE/dTn for every site, by the segmented
// forward / recompute-and-reverse scheme described at the top of this file.
template <class BK>
double energy_grad(BK& bk, const Lattice& lat, const std::vector<typename BK::Ten>& Tn,
                   const std::vector<WindowTerm>& terms, const Options& o,
                   std::vector<typename BK::Ten>* grads) {
  using Ten = typename BK::Ten;
  if (o.iterations < 0) fail(TG_E_INPUT, "energy gradient: iterations must be >= 0");
  if (o.checkpoint_every < 1) fail(TG_E_INPUT, "energy gradient: checkpoint_every must be >= 1");
  if (terms.empty()) fail(TG_E_INPUT, "energy gradient: no energy terms");
  const int K = o.checkpoint_every;
  const int nseg = o.iterations == 0 ? 1 : (o.iterations + K - 1) / K;
  auto seg_sweeps = [&](int s) { return std::min(o.iterations, (s + 1) * K) - s * K; };
  struct EnvVals {
    std::array<std::vector<Ten>, 4> C, E;
  };
  std::vector<EnvVals> ck(static_cast<size_t>(nseg));
  auto values_of = [](Tape<BK>& tp, const std::array<std::vector<int>, 4>& ids) {
    std::array<std::vector<Ten>, 4> v;
    for (int w = 0; w < 4; ++w)
      for (int id : ids[w]) v[w].push_back(tp.val(id));
    return v;
  };

  // forward: keep the environment at every segment start
  double E = 0.0;
  for (int s = 0; s < nseg; ++s) {
    Tape<BK> tp(bk);
    CtmTape<BK> ct(tp, lat, o);
    ct.set_sites(Tn, false);
    if (s == 0) ct.init();
    else ct.set_env(ck[s].C, ck[s].E, false);
    for (int it = 0; it < seg_sweeps(s); ++it) ct.sweep();
    if (s + 1 < nseg) {
      ck[s + 1].C = values_of(tp, ct.C);
      ck[s + 1].E = values_of(tp, ct.E);
    } else {
      E = ct.energy(terms).E;
    }
  }
  if (!grads) return E;

  // reverse: recompute each segment on a fresh tape, last segment first
  grads->assign(Tn.size(), Ten());
  std::array<std::vector<Ten>, 4> gC, gE;
  for (int s = nseg - 1; s >= 0; --s) {
    Tape<BK> tp(bk);
    tp.eps = o.eps;
    CtmTape<BK> ct(tp, lat, o);
    ct.set_sites(Tn, true);
    std::array<std::vector<int>, 4> leafC, leafE;
    if (s == 0) {
      ct.init();
    } else {
      ct.set_env(ck[s].C, ck[s].E, true);
      leafC = ct.C;
      leafE = ct.E;
    }
    for (int it = 0; it < seg_sweeps(s); ++it) ct.sweep();
    if (s == nseg - 1) {
      const auto en = ct.energy(terms);
      ct.seed_energy(terms, en);
    } else {
      for (int w = 0; w < 4; ++w)
        for (size_t i = 0; i < ct.C[w].size(); ++i) {
          if (!BK::empty(gC[w][i])) tp.seed(ct.C[w][i], gC[w][i]);
          if (!BK::empty(gE[w][i])) tp.seed(ct.E[w][i], gE[w][i]);
        }
    }
    tp.backward();
    for (size_t i = 0; i < Tn.size(); ++i) {
      const Ten& g = tp.grad(ct.Tn[i]);
      if (BK::empty(g)) continue;
      if (BK::empty((*grads)[i])) (*grads)[i] = g;
      else bk.axpy((*grads)[i], g, 1.0);
    }
    if (s > 0) {
      for (int w = 0; w < 4; ++w) {
        gC[w].assign(leafC[w].size(), Ten());
        gE[w].assign(leafE[w].size(), Ten());
        for (size_t i = 0; i < leafC[w].size(); ++i) gC[w][i] = tp.grad(leafC[w][i]);
        for (size_t i = 0; i < leafE[w].size(); ++i) gE[w][i] = tp.grad(leafE[w][i]);
      }
    }
  }
  for (size_t i = 0; i < Tn.size(); ++i)
    if (BK::empty((*grads)[i])) (*grads)[i] = bk.zeros(BK::shape(Tn[i]));
  return E;
}

}  // namespace ad
}  // namespace tg
