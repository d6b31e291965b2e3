// Golden draws of std::mt19937 + std::uniform_real_distribution<double>(-1,1)
// from the C++ standard library, the generator pair iTPS::initialize_tensors
// uses (src/iTPS/tensors.cpp:83-86).  Test infrastructure: the oracle's Python
// restatement of the generator is checked against this program's output.
//   usage: mt19937_draws <seed> <count>
#include <cstdio>
#include <cstdlib>
#include <random>

int main(int argc, char** argv) {
  unsigned seed = argc > 1 ? static_cast<unsigned>(std::atoi(argv[1])) : 11u;
  int count = argc > 2 ? std::atoi(argv[2]) : 16;
  std::mt19937 gen(seed);
  std::uniform_real_distribution<double> dist(-1.0, 1.0);
  for (int i = 0; i < count; ++i) std::printf("%.17g\n", dist(gen));
  return 0;
}
