/* The reference's own Pi() driver (PI.h:138-212), compiled unmodified from
 * the reference checkout, running on this library's pic::BigFloat instead of
 * the reference's BigFloat.cpp (oracle/Makefile target `dropin` ->
 * oracle/_ref/picdropin_pi).  It proves the C++ drop-in: the only changes are
 * the three headers in oracle/dropin_shim/ and pic_init() before the first
 * BigFloat.  The reference's std::thread fork of Pi_BSR (PI.h:93-108) runs as
 * written, so two host threads drive the library at once.
 *
 * usage: picdropin_pi <decimal_digits> <threads>
 * Writes pi.txt into the current directory (PI.h:210) and one JSON line on
 * stderr with the wall-clock seconds of Pi(). */
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
    if (pic_init(0) != PIC_OK) {
        fprintf(stderr, "pic_init failed: %s\n", pic_last_error());
        return 1;
    }
    double t0 = wall_clock();
    try {
        Pi(digits, threads);
    } catch (const char* e) {
        fprintf(stderr, "threw: %s\n", e);
        return 1;
    } catch (const std::exception& e) {
        fprintf(stderr, "threw: %s\n", e.what());
        return 1;
    }
    double t1 = wall_clock();
    fprintf(stderr, "{\"digits\": %zu, \"threads\": %zu, \"pi_s\": %.6f}\n", digits, threads, t1 - t0);
    pic_shutdown();
    return 0;
}
