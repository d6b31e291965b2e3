// Host instantiation of the full-update bond step (tenes_b200/csrc/full_update.hpp)
// for tests on the CPU.  Reads from stdin 13 tensors -- C1 C2 C3 C4, eT1..eT6,
// Tn1, Tn2, op12 -- each as "rank d0 ... values..." (row-major), then connect1;
// prints "S <iterations> <converged>" and the new tensors as "T <rank> <dims> <values>".
#include <cstdio>
#include <iostream>
#include <vector>

#include "full_update.hpp"
#include "host_tensor.hpp"

int main() {
  std::vector<HT> t;
  for (int q = 0; q < 13; ++q) {
    int rank;
    std::cin >> rank;
    tg::Shape s(static_cast<size_t>(rank));
    for (auto& d : s) std::cin >> d;
    HT x = make(s);
    for (int64_t i = 0; i < x.size(); ++i) std::cin >> x.p()[i];
    t.push_back(x);
  }
  int connect;
  std::cin >> connect;
  HostBackend bk;
  tg::fu::FullUpdate<HostBackend> fu{bk, tg::fu::Params{}};
  HT a, b;
  const tg::fu::Stats st =
      fu.bond(t[0], t[1], t[2], t[3], t[4], t[5], t[6], t[7], t[8], t[9], t[10], t[11], t[12], connect, a, b);
  std::printf("S %d %d\n", st.iterations, st.converged ? 1 : 0);
  for (const HT& x : {a, b}) {
    std::printf("T %zu", x.sh.size());
    for (auto d : x.sh) std::printf(" %lld", static_cast<long long>(d));
    for (int64_t i = 0; i < x.size(); ++i) std::printf(" %.17g", x.p()[i]);
    std::printf("\n");
  }
  return 0;
}
