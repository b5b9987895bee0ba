// limiter_check.cu -- the one-division minmod / superbee limited gradient
// (limited_gradient_t, mhc_device.cuh) against the reference two-division
// formula (limited_gradient_ref) on random and adversarial slope pairs:
// ratios a few ulps around 1/2, 1, 2 and 4, signed zeros, subnormals,
// the largest finite values, infinities and NaN.  Both run on the host with
// the IEEE operations the device performs (built without contraction).
// Exit status 0 when every result is bit-identical.
#include <cstdio>
#include <cstring>
#include <cstdint>
#include <random>
#include <cmath>
#include "mhc_device.cuh"
using namespace mhc;
static bool same(double a, double b) { uint64_t x, y; memcpy(&x, &a, 8); memcpy(&y, &b, 8); return x == y; }
template <int L> long check(double gb, double gf, long& bad) {
  double a = limited_gradient_ref<L>(gb, gf), b = limited_gradient_t<L>(gb, gf);
  if (!same(a, b) && !(std::isnan(a) && std::isnan(b))) { if (bad < 10) printf("LIM %d gb=%.17g gf=%.17g ref=%.17g new=%.17g\n", L, gb, gf, a, b); ++bad; }
  return 1;
}
int main() {
  std::mt19937_64 rng(12345);
  std::uniform_real_distribution<double> u(-1, 1), e(-300, 300);
  long n = 0, bad = 0;
  auto test = [&](double gb, double gf) { n += check<0>(gb, gf, bad); n += check<1>(gb, gf, bad); n += check<0>(gf, gb, bad); n += check<1>(gf, gb, bad); };
  // random magnitudes over the whole range
  for (long i = 0; i < 2000000; ++i) test(u(rng) * std::pow(10., e(rng) * 0.1), u(rng) * std::pow(10., e(rng) * 0.1));
  // ratios straddling 1/2, 1, 2 by a few ulps, both signs and orders
  const double ks[] = {0.5, 1.0, 2.0, 4.0, 0.25};
  for (long i = 0; i < 500000; ++i) {
    double d = u(rng) * std::pow(10., e(rng) * 0.03);
    double k = ks[i % 5];
    double nn = d * k;
    for (int s = -3; s <= 3; ++s) {
      double x = nn;
      for (int t = 0; t < std::abs(s); ++t) x = std::nextafter(x, s > 0 ? INFINITY : -INFINITY);
      test(d, x);
    }
  }
  // specials
  const double sp[] = {0.0, -0.0, 1.0, -1.0, 2.0, 0.5, 4.9e-324, -4.9e-324, 2.2250738585072014e-308, 1.7976931348623157e308,
                       -1.7976931348623157e308, 1e-300, 1e300, INFINITY, -INFINITY, NAN, 3.0, 1.5, 0.75, 1e-160, 1e160};
  for (double a : sp) for (double b : sp) test(a, b);
  for (double a : sp) for (long i = 0; i < 1000; ++i) { double b = u(rng) * std::pow(10., e(rng)); test(a, b); }
  printf("checked %ld pairs x limiters, mismatches %ld\n", n, bad);
  return bad != 0;
}
