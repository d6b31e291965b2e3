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
#include "host_tensor.hpp"


int main(int argc, char** argv) {
  bool updown = false;
  for (int a = 1; a < argc; ++a) {
    if (std::string(argv[a]) == "zero-null") g_zero_null = true;
    if (std::string(argv[a]) == "updown") updown = true;
  }
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
  o.projector_corner = !updown;
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
