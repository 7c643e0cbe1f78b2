/* CPU check of the reciprocal-and-FMA division used by the kernels
 * (fsmeld_b200/csrc/rcpdiv.h) against IEEE division: every accepted case must
 * give the bits of a / b.  Build: gcc -O2 -ffp-contract=off rcpdiv_check.c -lm
 * Usage: rcpdiv_check <cases per family> <seed>; prints "mismatches N tested M". */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../fsmeld_b200/csrc/rcpdiv.h"

static uint64_t s_state;
static uint64_t rnd(void) { /* splitmix64 */
    uint64_t z = (s_state += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
static double mk(uint64_t sign, int exp, uint64_t mant) {
    const uint64_t bits = (sign << 63) | ((uint64_t)(exp + 1023) << 52) | (mant & ((1ull << 52) - 1));
    double d;
    memcpy(&d, &bits, 8);
    return d;
}
static uint64_t bits_of(double d) {
    uint64_t u;
    memcpy(&u, &d, 8);
    return u;
}

static long long tested, bad;
static void check(double a, double b) {
    const double qe = a * (1.0 / b);
    if (rcp_div_in_range_bits(qe) && !rcp_div_in_range(qe)) {  /* the integer test is the narrower one */
        if (bad < 10) printf("range tests disagree at %a\n", qe);
        ++bad;
    }
    if (!rcp_div_in_range(b)) return;
    const double y = 1.0 / b;
    const double q0 = rcp_div_estimate(a, y);
    if (!rcp_div_in_range(q0)) return;
    const double q = rcp_div_finish(a, b, y, q0);
    const double ref = a / b;
    ++tested;
    if (bits_of(q) != bits_of(ref)) {
        if (bad < 10) printf("mismatch a=%a b=%a got %a want %a\n", a, b, q, ref);
        ++bad;
    }
}

int main(int argc, char** argv) {
    const long long n = argc > 1 ? atoll(argv[1]) : 1000000;
    s_state = argc > 2 ? strtoull(argv[2], 0, 10) : 1;
    const uint64_t ones = (1ull << 52) - 1;
    for (long long i = 0; i < n; ++i) {
        const uint64_t r1 = rnd(), r2 = rnd(), r3 = rnd();
        const int ea = (int)(r3 % 161) - 80, eb = (int)((r3 >> 8) % 161) - 80;
        /* random significands and exponents */
        check(mk(r3 >> 63, ea, r1), mk((r3 >> 62) & 1, eb, r2));
        /* all-ones and minimal divisor significands */
        check(mk(0, ea, r1), mk(0, eb, ones));
        check(mk(0, ea, r1), mk(0, eb, 1));
        check(mk(0, ea, r1), mk(0, eb, ones - (r2 & 0xff)));
        /* dividends with all-ones significands */
        check(mk(1, ea, ones - (r1 & 0xff)), mk(0, eb, r2));
        /* powers of two */
        check(mk(0, ea, r1), mk(0, eb, 0));
        check(mk(0, ea, 0), mk(0, eb, r2));
        /* quotients close to a rounding boundary: a = RN(b * (q +- half ulp)) */
        {
            const double b = mk(0, eb, r2), q = mk(0, ea, r1);
            const double h = mk(0, ea - 53, 0);
            check(b * (q + h), b);
            check(b * (q - h), b);
            check(fma(b, q, b * h), b);
            check(fma(b, q, -b * h), b);
        }
        /* z-normalisation-like operands: small differences of nearby values */
        {
            const double t = mk(r3 & 1, (int)(r3 % 8) - 4, r1);
            const double mu = t + mk(r2 & 1, (int)((r2 >> 3) % 40) - 45, r2 >> 12);
            const double sg = mk(0, (int)((r1 >> 5) % 30) - 20, r2 >> 7);
            check(t - mu, sg);
        }
    }
    printf("mismatches %lld tested %lld\n", bad, tested);
    return bad != 0;
}
