// Accuracy harness for gpuga_b200/csrc/powf_dd.cuh on the host (built and run by
// tests/test_powf_dd_cpu.py): max and mean error in units in the last place
// against the FP64 power, over the argument ranges of the Tersoff bond order.
#include <cmath>
#include <cstdio>
#include <random>

#include "../gpuga_b200/csrc/powf_dd.cuh"

static double ulp_err(float r, double ref) {
  int e;
  std::frexp((float)ref, &e);
  return std::fabs((double)r - ref) / std::ldexp(1.0, e - 24);
}

int main(int argc, char** argv) {
  const long n = argc > 1 ? atol(argv[1]) : 2000000;
  std::mt19937_64 g(7);
  std::uniform_real_distribution<double> lx(-16 * std::log(10.0), 4 * std::log(10.0)), uy(-3.0, 3.0), u1(0, 1);
  double mx = 0, sum = 0;
  long cnt = 0;
  for (long i = 0; i < n; ++i) {
    float x, y;
    switch (i % 4) {
      case 0: x = (float)std::exp(lx(g)); y = (float)uy(g); break;                       // general
      case 1: x = (float)(1.0 + 1e-3 * (u1(g) - 0.5)); y = (float)uy(g); break;          // near 1
      case 2: x = (float)(1.0 + std::exp(lx(g))); y = (float)(-0.5 / (0.3 + 2.7 * u1(g))); break;  // (1+z)^(-1/2n)
      default: x = (float)std::exp(0.25 * lx(g)); y = (float)(0.3 + 2.7 * u1(g)); break;  // zeta^n
    }
    const double ref = std::pow((double)x, (double)y);
    if (!(ref > 1e-37 && ref < 1e37)) continue;
    const double e = ulp_err(gpuga::powf_dd(x, y), ref);
    mx = std::max(mx, e);
    sum += e;
    ++cnt;
  }
  // exact and out-of-domain cases
  int bad = 0;
  bad += gpuga::powf_dd(1.0f, 0.7f) != 1.0f;
  bad += gpuga::powf_dd(2.0f, 3.0f) != 8.0f;
  bad += gpuga::powf_dd(4.0f, -0.5f) != 0.5f;
  bad += !(gpuga::powf_dd(0.0f, 2.0f) == 0.0f);
  bad += !std::isnan(gpuga::powf_dd(NAN, 0.5f));
  bad += !(gpuga::powf_dd(INFINITY, 1.0f) == INFINITY);
  bad += !(gpuga::powf_dd(INFINITY, -1.0f) == 0.0f);
  bad += !(gpuga::powf_dd(3.0f, 200.0f) == INFINITY);
  bad += gpuga::powf_dd(1e-30f, 4.0f) != 0.0f;  // 1e-120 flushes to zero
  printf("%ld %.6f %.6f %d\n", cnt, mx, sum / cnt, bad);
  return 0;
}
