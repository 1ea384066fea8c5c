/* Host restatement of the FP64 modular arithmetic of fp64mod.cuh (the FP64
 * three-prime form), checked against 128-bit integer arithmetic:
 *   dmul_tw:  y w mod p, |r| <= 0.75 p, |y| < 2^51, 0 <= w < p, wp = fl(w / p);
 *             |r| <= p with wp = fl(w fl(1 / p)) (the FP64 form's companion)
 *   dmul_mod: a b mod p, |r| <= 0.75 p, |a b| < 2^51 p
 *   dreduce:  s mod p,   |r| <= p / 2 + 1, |s| < 2^56
 * Built with -ffp-contract=off so that every multiply, add and fma rounds
 * exactly once, as the device intrinsics do.  Usage: fp64mod_check COUNT;
 * prints "bad=N maxr=X" and exits nonzero on any failure. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

static const double C = 6755399441055744.0; /* 1.5 * 2^52 */

static double dmul_tw(double y, double w, double wp, double p)
{
    double q = fma(y, wp, C) - C;
    double h = y * w;
    double l = fma(y, w, -h);
    return fma(-q, p, h) + l;
}

static double dmul_mod(double a, double b, double p, double pinv)
{
    double h = a * b;
    double l = fma(a, b, -h);
    double q = fma(h, pinv, C) - C;
    return fma(-q, p, h) + l;
}

static double dreduce(double s, double p, double pinv)
{
    double q = fma(s, pinv, C) - C;
    return fma(-q, p, s);
}

static uint64_t st = 88172645463325252ull;
static uint64_t rnd(void)
{
    st ^= st << 13;
    st ^= st >> 7;
    st ^= st << 17;
    return st;
}

static int check(double r, __int128 want, double p, double bound, double* maxr)
{
    __int128 m = (__int128)(int64_t)r % (__int128)(int64_t)p;
    if (m < 0) m += (int64_t)p;
    if (fabs(r) / p > *maxr) *maxr = fabs(r) / p;
    return r == floor(r) && m == want && fabs(r) <= bound;
}

int main(int argc, char** argv)
{
    const long count = argc > 1 ? atol(argv[1]) : 1000000;
    const uint64_t primes[3] = {140496970186753ull, 140458315481089ull, 140449725546497ull};
    long bad = 0;
    double maxr = 0;
    for (int pi = 0; pi < 3; pi++) {
        const uint64_t p = primes[pi];
        const double pd = (double)p, pinv = 1.0 / pd;
        for (long it = 0; it < count; it++) {
            /* y up to 12 p (the largest forward value of a radix-16 round) */
            const int64_t lim = (int64_t)(12 * p);
            int64_t y;
            uint64_t w = rnd() % p;
            switch (it & 3) {
            case 0: y = (int64_t)(rnd() % (2 * (uint64_t)lim + 1)) - lim; break;
            case 1: y = lim - (int64_t)(rnd() % 64); break;
            case 2: y = -lim + (int64_t)(rnd() % 64); break;
            default: y = (int64_t)(rnd() % p); w = p - 1 - rnd() % 4; break;
            }
            __int128 want = ((__int128)y * (int64_t)w) % (__int128)p;
            if (want < 0) want += p;
            const double wd = (double)w;
            if (!check(dmul_tw((double)y, wd, wd / pd, pd), want, pd, 0.75 * pd, &maxr)) bad++;
            /* the companion formed in the butterfly, fl(w fl(1/p)): |r| <= p
               for |y| up to 16 p (the largest forward value of a radix-16
               round and the CRT's largest input) */
            {
                const int64_t lim16 = (int64_t)(16 * p) - 1;
                int64_t y16 = (it & 1) ? (int64_t)(rnd() % (2 * (uint64_t)lim16 + 1)) - lim16
                                       : ((it & 2) ? lim16 - (int64_t)(rnd() % 64) : -lim16 + (int64_t)(rnd() % 64));
                __int128 w16 = ((__int128)y16 * (int64_t)w) % (__int128)p;
                if (w16 < 0) w16 += p;
                double maxr16 = 0;
                if (!check(dmul_tw((double)y16, wd, wd * pinv, pd), w16, pd, pd, &maxr16)) bad++;
            }
            /* two residues below 0.75 p */
            const int64_t a = (int64_t)(rnd() % (p + p / 2)) - (int64_t)(3 * p / 4);
            const int64_t b = (int64_t)(rnd() % (p + p / 2)) - (int64_t)(3 * p / 4);
            want = ((__int128)a * b) % (__int128)p;
            if (want < 0) want += p;
            if (!check(dmul_mod((double)a, (double)b, pd, pinv), want, pd, 0.75 * pd, &maxr)) bad++;
            /* reduction of a value below 12 p */
            const int64_t sv = (int64_t)(rnd() % (2 * (uint64_t)lim + 1)) - lim;
            want = (__int128)sv % (__int128)p;
            if (want < 0) want += p;
            if (!check(dreduce((double)sv, pd, pinv), want, pd, 0.5 * pd + 1, &maxr)) bad++;
        }
    }
    printf("bad=%ld maxr=%.6f\n", bad, maxr);
    return bad != 0;
}
