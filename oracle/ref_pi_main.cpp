/* Headless driver around the reference's own Pi() (PI.h:138-212), compiled
 * with the unmodified reference sources by oracle/Makefile into
 * oracle/_ref/picref_pi.  Test infrastructure and CPU baseline only.
 *
 * usage: picref_pi <decimal_digits> <threads>
 * Writes pi.txt into the current directory exactly as the reference does
 * (PI.h:210) and prints one JSON line on stderr with wall-clock seconds for
 * the table build (PI.h:145-146, done up front so Pi() finds them ready) and
 * for Pi() itself. */
#include "PI.h"
#include <cstdlib>

int main(int argc, char** argv)
{
    if (argc < 3) {
        fprintf(stderr, "usage: %s <decimal_digits> <threads>\n", argv[0]);
        return 2;
    }
    size_t digits = (size_t)strtoull(argv[1], nullptr, 10);
    size_t threads = (size_t)strtoull(argv[2], nullptr, 10);
    double t0 = wall_clock();
    fft_ensure_table(26);
    ntt_ensure_table(29);
    double t1 = wall_clock();
    try {
        Pi(digits, threads);
    } catch (const char* e) {
        fprintf(stderr, "reference threw: %s\n", e);
        return 1;
    }
    double t2 = wall_clock();
    fprintf(stderr, "{\"digits\": %zu, \"threads\": %zu, \"tables_s\": %.6f, \"pi_s\": %.6f}\n",
            digits, threads, t1 - t0, t2 - t1);
    return 0;
}
