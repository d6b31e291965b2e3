// Host instantiation of the simple update's local gauge fixing
// (tenes_b200/csrc/local_gauge.hpp) for tests on the CPU, real or complex.
// Reads from stdin "real" or "complex", N, then per site "parity n0 n1 n2 n3"
// (its neighbours over legs 0..3), then N site tensors as "rank d0 ... values"
// (row-major; complex entries as "re im"), then the 4N bond weights in site,
// leg order (each as its values, lengths from the tensor shapes), then
// "lambda_cut maxiter eps".  Prints "S <sweeps> <score>", the N tensors as
// "T <rank> <dims> <values>" and the 4N weights as "L <values>".
#include <array>
#include <complex>
#include <cstdio>
#include <iostream>
#include <string>
#include <vector>

#include "host_tensor.hpp"
#include "host_tensor_c.hpp"
#include "local_gauge.hpp"

template <class BK, class Make, class Read, class Write>
int run(Make make_t, Read read_v, Write write_v) {
  using Ten = typename BK::Ten;
  int N;
  std::cin >> N;
  std::vector<int> par(static_cast<size_t>(N));
  std::vector<std::array<int, 4>> nb(static_cast<size_t>(N));
  for (int i = 0; i < N; ++i) {
    std::cin >> par[static_cast<size_t>(i)];
    for (auto& x : nb[static_cast<size_t>(i)]) std::cin >> x;
  }
  std::vector<Ten> Tn;
  std::vector<std::array<int, 4>> vdim(static_cast<size_t>(N));
  for (int q = 0; q < N; ++q) {
    int rank;
    std::cin >> rank;
    tg::Shape s(static_cast<size_t>(rank));
    for (auto& d : s) std::cin >> d;
    Ten x = make_t(s);
    for (int64_t i = 0; i < x.size(); ++i) x.p()[i] = read_v();
    for (int l = 0; l < 4; ++l) vdim[static_cast<size_t>(q)][static_cast<size_t>(l)] = static_cast<int>(s[static_cast<size_t>(l)]);
    Tn.push_back(x);
  }
  std::vector<tg::gauge::Weights> lam(static_cast<size_t>(N));
  for (int q = 0; q < N; ++q)
    for (int l = 0; l < 4; ++l) {
      auto& v = lam[static_cast<size_t>(q)][static_cast<size_t>(l)];
      v.resize(static_cast<size_t>(vdim[static_cast<size_t>(q)][static_cast<size_t>(l)]));
      for (double& x : v) std::cin >> x;
    }
  double cut, eps;
  int maxiter;
  std::cin >> cut >> maxiter >> eps;
  BK bk;
  tg::gauge::LocalGauge<BK> g{bk, cut};
  double score = 0.0;
  const int sweeps = g.run(
      Tn, lam, vdim, [&](int s, int leg) { return nb[static_cast<size_t>(s)][static_cast<size_t>(leg)]; },
      [&](int s) { return par[static_cast<size_t>(s)]; }, maxiter, eps, &score);
  std::printf("S %d %.17g\n", sweeps, score);
  for (const Ten& x : Tn) {
    std::printf("T %zu", x.sh.size());
    for (auto d : x.sh) std::printf(" %lld", static_cast<long long>(d));
    for (int64_t i = 0; i < x.size(); ++i) write_v(x.p()[i]);
    std::printf("\n");
  }
  for (const auto& w : lam)
    for (const auto& v : w) {
      std::printf("L");
      for (double x : v) std::printf(" %.17g", x);
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
  return run<HostBackend>([](const tg::Shape& s) { return make(s); },
                          [] {
                            double v;
                            std::cin >> v;
                            return v;
                          },
                          [](double v) { std::printf(" %.17g", v); });
}
