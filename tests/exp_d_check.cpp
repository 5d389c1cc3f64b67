// Accuracy harness for gpuga_b200/csrc/exp_d.cuh on the host (built and run by
// tests/test_exp_d_cpu.py): max and mean relative error against the exponential
// evaluated in long double, over the arguments of the Tersoff pair terms and the
// whole domain, plus the edge cases.
#include <cmath>
#include <cstdio>
#include <random>

#include "../gpuga_b200/csrc/exp_d.cuh"

int main(int argc, char** argv) {
  const long n = argc > 1 ? atol(argv[1]) : 2000000;
  std::mt19937_64 g(11);
  std::uniform_real_distribution<double> pair(-12.0, 6.0), wide(-708.0, 708.0);
  double mx = 0, sum = 0, mx10 = 0, mx9c = 0;
  long cnt = 0;
  for (long i = 0; i < n; ++i) {
    const double x = (i % 4 == 3) ? wide(g) : pair(g);
    const long double ref = std::exp((long double)x);
    const double e = (double)(std::fabs((long double)gpuga::exp_d(x) - ref) / ref);
    mx = std::max(mx, e);
    mx10 = std::max(mx10, (double)(std::fabs((long double)gpuga::exp_d<10>(x) - ref) / ref));
    mx9c = std::max(mx9c, (double)(std::fabs((long double)gpuga::exp_d_clamped<9>(x) - ref) / ref));
    sum += e;
    ++cnt;
  }
  int bad = 0;
  bad += gpuga::exp_d(0.0) != 1.0;
  bad += gpuga::exp_d(-800.0) != 0.0;
  bad += !std::isinf(gpuga::exp_d(800.0));
  bad += !std::isnan(gpuga::exp_d(NAN));
  bad += std::fabs(gpuga::exp_d(1.0) - 2.718281828459045) > 1e-15;
  bad += !std::isnan(gpuga::exp_d_clamped<9>(NAN));
  bad += !(gpuga::exp_d_clamped<9>(-800.0) < 1e-300);
  printf("%ld %.6e %.6e %d %.6e %.6e\n", cnt, mx, sum / cnt, bad, mx10, mx9c);
  return 0;
}
