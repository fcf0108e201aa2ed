/* fx_split_check.c -- compiled and run by tests/test_fixed_point_scheme.py.
 *
 * Restates, in host C, the device's split of a J/K contribution v into the
 * two fixed-point words it adds (csrc/pfk_device.cuh, fx_add):
 *   a = fma(v, 2^24, 1.5 2^52);  h = a - 1.5 2^52;  r = fma(v, 2^24, -h);
 *   b = fma(r, 2^36, 1.5 2^52);
 *   hi = bits(a) - bits(1.5 2^52) (added only when h != 0),
 *   lo = bits(b) - bits(1.5 2^52),
 * and checks, for seeded random v of every binade from 2^-80 to 2^27 plus
 * edge cases (ties, powers of two, the range limits), that
 * hi 2^36 + lo == rint(v 2^60) exactly, |lo| <= 2^35, and that the value
 * rule hi_sum 2^-24 + lo_sum 2^-60 of a shuffled sum equals the exact sum
 * rounded once.  Prints "ok <count>" or the first failure; exit status 0 on
 * success. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

static int64_t bits(double x)
{
    int64_t b;
    memcpy(&b, &x, sizeof b);
    return b;
}

static const double M = 6755399441055744.0; /* 1.5 2^52 */

static void split(double v, int64_t *hi, int64_t *lo)
{
    const double a = fma(v, 16777216.0, M);
    const double h = a - M;
    const double r = fma(v, 16777216.0, -h);
    const double b = fma(r, 68719476736.0, M);
    *hi = h != 0.0 ? bits(a) - bits(M) : 0;
    *lo = bits(b) - bits(M);
}

/* xorshift64*: a seeded uniform in (-1, 1) */
static uint64_t s = 0x9E3779B97F4A7C15ull;
static double urand(void)
{
    s ^= s >> 12;
    s ^= s << 25;
    s ^= s >> 27;
    const uint64_t x = s * 2685821657736338717ull;
    return ((double)(x >> 11) / 9007199254740992.0) * 2.0 - 1.0;
}

static int check(double v)
{
    int64_t hi, lo;
    split(v, &hi, &lo);
    const long double X = rintl((long double)v * 1152921504606846976.0L); /* exact: v 2^60 has 53 bits */
    const __int128 want = (__int128)X;
    const __int128 got = (__int128)hi * ((__int128)1 << 36) + lo;
    if (got != want || lo > (1ll << 35) || lo < -(1ll << 35)) {
        printf("FAIL v=%a hi=%lld lo=%lld\n", v, (long long)hi, (long long)lo);
        return 1;
    }
    return 0;
}

int main(void)
{
    long n = 0;
    for (int e = -80; e <= 26; ++e)
        for (int k = 0; k < 20000; ++k, ++n)
            if (check(ldexp(urand(), e + 1))) return 1;
    const double edge[] = {0.0, -0.0, 1.0, -1.0, 0.5, ldexp(1.0, -24), ldexp(1.5, -24), ldexp(2.5, -24),
                           ldexp(-2.5, -24), ldexp(1.0, -61), ldexp(3.0, -61), ldexp(5.0, -61),
                           ldexp(1.0, -60), ldexp(1.0, -25), ldexp(1.0, -26), ldexp(0.999999999, 27),
                           -ldexp(0.999999999, 27), 1e-300, -1e-300, 123.456, -98765.4321};
    for (size_t i = 0; i < sizeof edge / sizeof edge[0]; ++i, ++n)
        if (check(edge[i])) return 1;
    /* order independence of the accumulated value: the same 4096 adds in two
     * orders give the same words, and the value rule rounds the exact sum */
    enum { N = 4096 };
    static double v[N];
    for (int i = 0; i < N; ++i) v[i] = ldexp(urand(), -(i % 40));
    uint64_t h1 = 0, l1 = 0, h2 = 0, l2 = 0;
    long double exact = 0.0L;
    for (int i = 0; i < N; ++i) {
        int64_t hi, lo;
        split(v[i], &hi, &lo);
        h1 += (uint64_t)hi;
        l1 += (uint64_t)lo;
        exact += rintl((long double)v[i] * 1152921504606846976.0L);
    }
    for (int i = N - 1; i >= 0; --i) {
        int64_t hi, lo;
        split(v[(i * 7919) % N], &hi, &lo);
        h2 += (uint64_t)hi;
        l2 += (uint64_t)lo;
    }
    if (h1 != h2 || l1 != l2) {
        printf("FAIL order dependence\n");
        return 1;
    }
    /* value rule (pfk_device.cuh fx_value): lo's multiples of 2^36 move into hi */
    const int64_t lo_s = (int64_t)l1, rem = lo_s & ((1ll << 36) - 1), carry = (lo_s - rem) / (1ll << 36);
    const double value = (double)((int64_t)h1 + carry) * ldexp(1.0, -24) + (double)rem * ldexp(1.0, -60);
    const double want = (double)(exact * ldexpl(1.0L, -60));
    if (fabs(value - want) > 2.0 * fabs(want) * 1.2e-16) {
        printf("FAIL value rule %a vs %a\n", value, want);
        return 1;
    }
    printf("ok %ld\n", n);
    return 0;
}
