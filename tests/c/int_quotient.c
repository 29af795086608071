/* Exhaustive check behind the integer time-axis evaluation: for every integer
 * pair 0 <= a <= b <= n, with y = RN(1/b), one Markstein correction
 *   q0 = RN(a*y),  q1 = RN(q0 + RN(a - b*q0)*y)   (both steps as FMAs)
 * equals the IEEE quotient RN(a/b) bit for bit.  Prints the mismatch counts of
 * q1 and, for contrast, of the bare product q0.  Build with FMA contraction
 * off so the compiler adds no fusions of its own. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

int main(int argc, char** argv) {
  long n = argc > 1 ? atol(argv[1]) : 65536;
  unsigned long long bad0 = 0, bad1 = 0, pairs = 0;
  for (long b = 1; b <= n; ++b) {
    const double bd = (double)b, y = 1.0 / bd;
    for (long a = 0; a <= b; ++a) {
      const double ad = (double)a, q = ad / bd;
      const double q0 = ad * y;
      const double q1 = fma(fma(-q0, bd, ad), y, q0);
      bad0 += memcmp(&q0, &q, sizeof q) != 0;
      bad1 += memcmp(&q1, &q, sizeof q) != 0;
      ++pairs;
    }
  }
  printf("%ld %llu %llu %llu\n", n, pairs, bad1, bad0);
  return 0;
}
