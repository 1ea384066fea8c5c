/* Headless driver around the reference's own decimal output,
 * BigFloat::to_string_dec (BigFloat.cpp:83-94), compiled with the unmodified
 * reference sources by oracle/Makefile into oracle/_ref/picref_dec.  Test
 * infrastructure only (the golden fixtures of the decimal conversion).
 *
 *   picref_dec words <file> <digits> <out>   the number stored in <file>
 *       (int32 sign, int64 exp, uint64 L, then L uint32 words, little-endian)
 *   picref_dec pi <digits> <threads> <out>   Pi()'s final number: the
 *       reference's Pi_BSR, combination, division, inverse square root and
 *       final product in Pi()'s order (PI.h:141-199); Pi() itself prints it
 *       in hex
 *
 * writes to_string_dec(digits) into the file <out> (stdout carries the
 * reference's own progress lines, PI.h:114-135). */
#define private public
#include "BigFloat.h"
#undef private
#include "PI.h"
#include <cstdlib>
#include <vector>

int main(int argc, char** argv)
{
    if (argc < 5) {
        fprintf(stderr, "usage: %s words <file> <digits> <out> | pi <digits> <threads> <out>\n", argv[0]);
        return 2;
    }
    const std::string mode = argv[1];
    BigFloat P;
    size_t digits = 0;
    if (mode == "words") {
        FILE* f = fopen(argv[2], "rb");
        if (!f) return 3;
        int32_t sign;
        int64_t exp;
        uint64_t L;
        if (fread(&sign, 4, 1, f) != 1 || fread(&exp, 8, 1, f) != 1 || fread(&L, 8, 1, f) != 1) return 4;
        P.sign = sign != 0;
        P.exp = exp;
        P.L = (size_t)L;
        P.T = std::unique_ptr<uint32_t[]>(new uint32_t[L ? L : 1]);
        if (L && fread(P.T.get(), 4, L, f) != L) return 5;
        fclose(f);
        digits = (size_t)strtoull(argv[3], nullptr, 10);
    } else if (mode == "pi") {
        digits = (size_t)strtoull(argv[2], nullptr, 10);
        const size_t threads = (size_t)strtoull(argv[3], nullptr, 10);
        const size_t hex_digits = digits * log(10) / log(16);
        const size_t p = (hex_digits + 9) / 9;
        const size_t p_dec = (digits + 9) / 9;
        const size_t terms = (size_t)(p_dec * 0.6346230241342037371474889163921741077188431452678) + 1;
        fft_ensure_table(26);  // PI.h:145-146: the tables are built before the threads start
        ntt_ensure_table(29);
        steps = terms - 1;
        time_init = wall_clock();
        BigFloat Q, R;
        int h;
        Pi_BSR(P, Q, R, 0, (uint32_t)terms, p, h, (int)threads);
        P = Q.mul(13591409).add(P, p);
        Q = Q.mul(4270934400);
        P = Q.div(P, p, threads);
        Q = invsqrt(10005, p, threads);
        P = P.mul(Q, p, threads);
    } else {
        return 2;
    }
    const std::string s = P.to_string_dec(digits);
    FILE* out = fopen(argv[4], "wb");
    if (!out) return 6;
    const bool ok = fwrite(s.data(), 1, s.size(), out) == s.size();
    fclose(out);
    return ok ? 0 : 7;
}
