// Host instantiation of the full-update bond step (tenes_b200/csrc/full_update.hpp)
// for tests on the CPU, real or complex.  Reads from stdin "real" or
// "complex", then 13 tensors -- C1 C2 C3 C4, eT1..eT6, Tn1, Tn2, op12 -- each
// as "rank d0 ... values..." (row-major; complex entries as "re im"), then
// connect1; prints "S <iterations> <converged>" and the new tensors as
// "T <rank> <dims> <values>" (complex: re im pairs).
#include <complex>
#include <cstdio>
#include <iostream>
#include <string>
#include <vector>

#include "full_update.hpp"
#include "host_tensor.hpp"
#include "host_tensor_c.hpp"

template <class BK, class Make, class Read, class Write>
int run(Make make_t, Read read_v, Write write_v) {
  using Ten = typename BK::Ten;
  std::vector<Ten> t;
  for (int q = 0; q < 13; ++q) {
    int rank;
    std::cin >> rank;
    tg::Shape s(static_cast<size_t>(rank));
    for (auto& d : s) std::cin >> d;
    Ten x = make_t(s);
    for (int64_t i = 0; i < x.size(); ++i) x.p()[i] = read_v();
    t.push_back(x);
  }
  int connect;
  std::cin >> connect;
  BK bk;
  tg::fu::FullUpdate<BK> fu{bk, tg::fu::Params{}};
  Ten a, b;
  const tg::fu::Stats st =
      fu.bond(t[0], t[1], t[2], t[3], t[4], t[5], t[6], t[7], t[8], t[9], t[10], t[11], t[12], connect, a, b);
  std::printf("S %d %d\n", st.iterations, st.converged ? 1 : 0);
  for (const Ten& x : {a, b}) {
    std::printf("T %zu", x.sh.size());
    for (auto d : x.sh) std::printf(" %lld", static_cast<long long>(d));
    for (int64_t i = 0; i < x.size(); ++i) write_v(x.p()[i]);
    std::printf("\n");
  }
  return 0;
}

int main() {
  std::string kind;
  std::cin >> kind;
  if (kind == "complex") {
    return run<HostBackendC>(
        [](const tg::Shape& s) { return makec(s); },
        [] {
          double re, im;
          std::cin >> re >> im;
          return std::complex<double>(re, im);
        },
        [](const std::complex<double>& v) { std::printf(" %.17g %.17g", v.real(), v.imag()); });
  }
  return run<HostBackend>(
      [](const tg::Shape& s) { return make(s); },
      [] {
        double v;
        std::cin >> v;
        return v;
      },
      [](double v) { std::printf(" %.17g", v); });
}
