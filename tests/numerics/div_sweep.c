/* Division through a shared reciprocal, checked against IEEE division.
 *
 * For a denominator b with y = RN(1/b), one Markstein correction step
 * (P. Markstein, IBM J. Res. Dev. 34(1), 1990):
 *     q  = RN(a * y)
 *     r  = fma(-q, b, a)      (exact)
 *     q' = fma(r, y, q)
 * should equal RN(a / b) away from underflow and overflow.  This program
 * counts the numerators a for which q' differs from a / b, over random
 * numerators with exponents -40..40 and the denominators listed in main plus
 * random ones.  Usage: div_sweep <quotients per fixed denominator>
 * <random denominators> <quotients per random denominator>; prints
 * "<quotients> <mismatches>". */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static uint64_t state = 0x9E3779B97F4A7C15ull;
static uint64_t next(void) { state ^= state << 13; state ^= state >> 7; state ^= state << 17; return state; }

static double random_double(int emin, int emax) {
  const uint64_t mant = next() & ((1ull << 52) - 1);
  const int e = emin + (int)(next() % (uint64_t)(emax - emin + 1));
  const uint64_t bits = ((uint64_t)(e + 1023) << 52) | mant;
  double d;
  memcpy(&d, &bits, sizeof d);
  return (next() & 1) ? -d : d;
}

static long long mismatches(double b, long long n) {
  const double y = 1.0 / b;
  long long bad = 0;
  for (long long i = 0; i < n; ++i) {
    const double a = random_double(-40, 40);
    const double q = a * y;
    const double r = fma(-q, b, a);
    if (fma(r, y, q) != a / b) ++bad;
  }
  return bad;
}

int main(int argc, char** argv) {
  const long long per_fixed = argc > 1 ? atoll(argv[1]) : 1000000;
  const int n_random = argc > 2 ? atoi(argv[2]) : 100;
  const long long per_random = argc > 3 ? atoll(argv[3]) : 100000;
  /* gamma - 1 for gamma = 1.4 and 5/3, and a few others */
  const double fixed[] = {0.4, 2.0 / 3.0, 0.4000000000000001, 1.0 / 3.0, 0.1, 3.0};
  long long total = 0, bad = 0;
  for (size_t k = 0; k < sizeof fixed / sizeof fixed[0]; ++k) {
    bad += mismatches(fixed[k], per_fixed);
    total += per_fixed;
  }
  for (int k = 0; k < n_random; ++k) {
    bad += mismatches(random_double(-20, 20), per_random);
    total += per_random;
  }
  printf("%lld %lld\n", total, bad);
  return 0;
}
