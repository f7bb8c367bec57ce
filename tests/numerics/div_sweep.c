/* Division through a reciprocal fixed for the launch, checked against IEEE
 * division bit for bit.
 *
 * div_by mirrors the FP64 device routine of the same name: for a divisor b
 * with y = RN(1/b) (y = 0 where b lies outside 2^-120 <= |b| < 2^121) and a
 * numerator a with 2^-900 <= |a| < 2^900, one Markstein correction step
 * (P. Markstein, IBM J. Res. Dev. 34(1), 1990)
 *     q  = RN(a * y)
 *     r  = fma(-q, b, a)      (exact)
 *     q' = fma(r, y, q)
 * gives RN(a / b); every other numerator (zero, subnormal, huge, Inf, NaN)
 * takes IEEE division.  This program counts the quotients for which div_by
 * differs from a / b in any bit (NaN: in NaN-ness), over
 *   - random numerators (exponents -40..40) by the fixed denominators listed
 *     in main and by random ones,
 *   - quotients within t * 2^-106 (|t| <= 3) of a rounding midpoint -- the
 *     cases where a wrong last correction would show -- with a/b below and
 *     above 1 and random power-of-two scalings of a and b,
 *   - the numerators at and around the ends of the range (signed zeros,
 *     subnormals, 2^-900, 2^900, DBL_MAX, Inf, NaN) by every fixed denominator.
 * Usage: div_sweep <quotients per fixed denominator> <random denominators>
 * <quotients per random denominator> [<near-midpoint quotients>]; prints
 * "<quotients> <mismatches>". */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

static uint64_t state = 0x9E3779B97F4A7C15ull;
static uint64_t next(void) { state ^= state << 13; state ^= state >> 7; state ^= state << 17; return state; }

static double shared_reciprocal(double b) {
  const double m = fabs(b);
  return (m >= 0x1p-120 && m < 0x1p121) ? 1.0 / b : 0.0;
}

static double div_by(double a, double b, double y) {
  uint64_t bits;
  memcpy(&bits, &a, sizeof bits);
  const unsigned e = (unsigned)(bits >> 52) & 0x7ffu;
  if (y != 0.0 && e - 123u < 1800u) {
    const double q = a * y;
    const double r = fma(-q, b, a);
    return fma(r, y, q);
  }
  return a / b;
}

static int differs(double got, double want) {
  if (isnan(got) || isnan(want)) return !(isnan(got) && isnan(want));
  return memcmp(&got, &want, sizeof got) != 0;
}

static double random_double(int emin, int emax) {
  const uint64_t mant = next() & ((1ull << 52) - 1);
  const int e = emin + (int)(next() % (uint64_t)(emax - emin + 1));
  const uint64_t bits = ((uint64_t)(e + 1023) << 52) | mant;
  double d;
  memcpy(&d, &bits, sizeof d);
  return (next() & 1) ? -d : d;
}

static long long mismatches(double b, long long n) {
  const double y = shared_reciprocal(b);
  long long bad = 0;
  for (long long i = 0; i < n; ++i) {
    const double a = random_double(-40, 40);
    bad += differs(div_by(a, b, y), a / b);
  }
  return bad;
}

/* a/b = m - t 2^-k / b for a midpoint m: B = b 2^52 odd in (2^52, 2^53), M odd
 * (the midpoint's significand one bit longer than a double's) and A = a's
 * significand with A 2^S - B M = t exactly. */
static long long near_midpoint(long long n, long long* made) {
  long long bad = 0;
  for (long long it = 0; it < n; ++it) {
    const uint64_t B = (1ull << 52) | (next() & ((1ull << 52) - 1)) | 1ull;
    long t = (long)(next() % 7) - 3;
    if ((t & 1) == 0) t += 1;
    const int below = (int)(next() & 1);       /* a/b in [1/2, 1) or in [1, 2) */
    const int S = below ? 54 : 53;             /* m = M 2^-S */
    const uint64_t mask = (S == 64) ? ~0ull : ((1ull << S) - 1);
    uint64_t Binv = B;                          /* B^-1 mod 2^64 (Newton) */
    for (int i = 0; i < 6; ++i) Binv *= 2 - B * Binv;
    const uint64_t M = ((uint64_t)(-(int64_t)t) * Binv) & mask;
    if (M < (1ull << (S - 1))) continue;       /* m in [1/2, 1) or [1, 2) */
    const u128 num = (u128)B * M + (u128)(int64_t)t;
    const uint64_t A = (uint64_t)(num >> S);
    if (A < (1ull << 52) || A >= (1ull << 53)) continue;
    double a = ldexp((double)A, -52), b = ldexp((double)B, -52);
    if (below ? !(a < b) : !(a >= b)) continue;
    /* power-of-two scalings keep the quotient's significand */
    const int ea = (int)(next() % 1601) - 800, eb = (int)(next() % 201) - 100;
    a = ldexp(a, ea);
    b = ldexp(b, eb);
    if (next() & 1) a = -a;
    if (next() & 1) b = -b;
    ++*made;
    bad += differs(div_by(a, b, shared_reciprocal(b)), a / b);
  }
  return bad;
}

int main(int argc, char** argv) {
  const long long per_fixed = argc > 1 ? atoll(argv[1]) : 1000000;
  const int n_random = argc > 2 ? atoi(argv[2]) : 100;
  const long long per_random = argc > 3 ? atoll(argv[3]) : 100000;
  const long long n_mid = argc > 4 ? atoll(argv[4]) : 4000000;
  /* gamma - 1 for gamma = 1.4 and 5/3, cell volumes, and a few others */
  const double fixed[] = {0.4, 2.0 / 3.0, 0.4000000000000001, 1.0 / 3.0, 0.1, 3.0,
                          1.0 / 1048576.0, 9.5367431640625e-07 * 2.0, 2.3841857910156250e-07 * 1.5,
                          0x1p-120, 0x1.fffffffffffffp120, 0x1p121, 1e-300};
  const int n_fixed = (int)(sizeof fixed / sizeof fixed[0]);
  long long total = 0, bad = 0;
  for (int k = 0; k < n_fixed; ++k) {
    bad += mismatches(fixed[k], per_fixed);
    total += per_fixed;
  }
  for (int k = 0; k < n_random; ++k) {
    bad += mismatches(random_double(-20, 20), per_random);
    total += per_random;
  }
  long long made = 0;
  bad += near_midpoint(n_mid, &made);
  total += made;
  const double edges[] = {0.0, -0.0, 0x1p-1074, -0x1p-1074, 0x1p-1022, 0x1.fffffffffffffp-901, 0x1p-900,
                          -0x1p-900, 0x1.0000000000001p-900, 0x1.fffffffffffffp899, -0x1.fffffffffffffp899,
                          0x1p900, 1.7976931348623157e308, INFINITY, -INFINITY, NAN, 1.0, -2.5};
  for (int k = 0; k < n_fixed; ++k) {
    for (size_t i = 0; i < sizeof edges / sizeof edges[0]; ++i) {
      bad += differs(div_by(edges[i], fixed[k], shared_reciprocal(fixed[k])), edges[i] / fixed[k]);
      ++total;
    }
  }
  printf("%lld %lld\n", total, bad);
  return 0;
}
