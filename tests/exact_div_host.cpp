// Host build of volcano-ash3d_b200/csrc/exact_div.cuh (test infrastructure).
//
// The device code refines a hardware reciprocal estimate and certifies the
// quotient with an exact residual before returning it; anything it cannot
// certify goes to the IEEE division operator.  Soundness of that
// certification does not depend on how good the estimate is, so this harness
// replaces the estimate by 1/b times (1 + d), d uniform in [-rel, rel], from
// exact (rel = 0) to useless (rel = 0.2), and checks div_rn and div_rn_rcp
// against the host's IEEE division bit for bit on several operand families.
//
// usage: exact_div_host <pairs per case> <seed>
// prints one line per case: "<func> <family> <rel> pairs <n> mismatches <m> fallbacks <f>"
// (fallbacks: quotients left to the IEEE operator, uncertified or out of range)
#include <math.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>

#define __device__
#define __forceinline__ inline
#define __noinline__ __attribute__((noinline))
static inline int __double2hiint(double x) {
  uint64_t u;
  std::memcpy(&u, &x, 8);
  return (int)(uint32_t)(u >> 32);
}
static inline long long __double_as_longlong(double x) {
  long long u;
  std::memcpy(&u, &x, 8);
  return u;
}
static inline double __longlong_as_double(long long u) {
  double x;
  std::memcpy(&x, &u, 8);
  return x;
}
#define A3G_HOST_TEST
#include "../volcano-ash3d_b200/csrc/exact_div.cuh"

static double g_rel = 0.0;
static std::mt19937_64 g_est(7);

double a3g::host_rcp_estimate(double b) {
  const double y = 1.0 / b;
  if (g_rel == 0.0) return y;
  std::uniform_real_distribution<double> u(-g_rel, g_rel);
  return y * (1.0 + u(g_est));
}

long &a3g::host_fallback_count() {
  static long n = 0;
  return n;
}

static double make(std::mt19937_64 &r, int emin, int emax) {
  const uint64_t m = r() & 0x000fffffffffffffULL;
  const int e = emin + (int)(r() % (uint64_t)(emax - emin + 1));
  uint64_t u = ((uint64_t)(e + 1023) << 52) | m;
  if (r() & 1) u |= 0x8000000000000000ULL;
  double x;
  std::memcpy(&x, &u, 8);
  return x;
}

static bool same(double x, double y) {
  if (isnan(x) && isnan(y)) return true;
  return std::memcmp(&x, &y, 8) == 0;
}

static void pair_of(int fam, std::mt19937_64 &r, double &a, double &b) {
  switch (fam) {
    case 0:  // exponents across and beyond the fast ranges (dividends to 2^+-1000, divisors to 2^+-230)
      a = make(r, -1000, 1000);
      b = make(r, -230, 230);
      break;
    case 1: {  // quotients within a few ulps of a power of two or of an integer
      b = make(r, -40, 40);
      const double q = (r() & 1) ? std::ldexp(1.0, (int)(r() % 60) - 30) : (double)(1 + r() % 1000);
      a = q * b;
      long long u = __double_as_longlong(a) + (long long)(r() % 7) - 3;
      a = __longlong_as_double(u);
      break;
    }
    case 2: {  // limiter-like ratios: differences of nearby concentrations
      const double c = make(r, -12, 12);
      a = c * (1.0 + std::ldexp((double)(r() % 4096) - 2048.0, -20)) - c;
      b = c * (1.0 + std::ldexp((double)(r() % 4096) - 2048.0, -18)) - c;
      if (b == 0.0) b = c;
      break;
    }
    case 3: {  // tails of a diffused cloud: tiny dividends (down to subnormal) over pivots in [1, 4)
      const int e = -1080 + (int)(r() % 931);  // -1080 .. -150
      a = make(r, 0, 0);
      a = std::ldexp(a, e);  // rounds into the subnormal range below 2^-1022
      b = make(r, 0, 1);
      break;
    }
    default: {  // specials: zeros, infinities, NaN, subnormals, equal operands
      static const double sp[] = {0.0, -0.0, INFINITY, -INFINITY, NAN, 4.9e-324, -2.2e-308, 1.0, -1.0,
                                  1.0e300, 1.0e-300, 3.0};
      const int n = (int)(sizeof(sp) / sizeof(sp[0]));
      a = (r() % 3) ? sp[r() % n] : make(r, -100, 100);
      b = (r() % 3) ? sp[r() % n] : make(r, -100, 100);
      if (r() % 8 == 0) b = a;
      break;
    }
  }
}

int main(int argc, char **argv) {
  const long n = argc > 1 ? std::atol(argv[1]) : 200000;
  const uint64_t seed = argc > 2 ? std::strtoull(argv[2], nullptr, 10) : 1;
  const double rels[] = {0.0, 1.2e-7, 6.0e-5, 4.0e-3, 0.2};
  const char *fams[] = {"wide", "near_exact", "limiter", "tails", "special"};
  int bad_total = 0;
  for (int f = 0; f < 2; f++) {
    for (int fam = 0; fam < 5; fam++) {
      for (double rel : rels) {
        g_rel = rel;
        std::mt19937_64 r(seed * 1000 + fam);
        long bad = 0;
        a3g::host_fallback_count() = 0;
        for (long t = 0; t < n; t++) {
          double a, b;
          pair_of(fam, r, a, b);
          double q;
          if (f == 0) {
            q = a3g::div_rn(a, b);
          } else {
            const double y = a3g::host_rcp_estimate(b);  // RN(1/b) when rel = 0
            q = a3g::div_rn_rcp(a, b, y);
          }
          const double ref = a / b;
          if (!same(q, ref)) {
            if (bad < 5)
              std::printf("MISMATCH %s %s rel=%g a=%a b=%a got=%a want=%a\n", f ? "div_rn_rcp" : "div_rn",
                          fams[fam], rel, a, b, q, ref);
            bad++;
          }
        }
        std::printf("%s %s %g pairs %ld mismatches %ld fallbacks %ld\n", f ? "div_rn_rcp" : "div_rn", fams[fam],
                    rel, n, bad, a3g::host_fallback_count());
        bad_total += bad != 0;
      }
    }
  }
  return bad_total ? 1 : 0;
}
