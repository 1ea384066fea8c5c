/* Drop-in check: the reference's FFT.h (FFT.h:4-9) as seen by its PI.h.
 * Pi() only calls fft_ensure_table (PI.h:145); it forwards to the library's
 * table build (the products themselves go through pic::BigFloat::mul). */
#pragma once
#include "piculator_b200.h"

inline void fft_ensure_table(int k)
{
    if (pic_fft_ensure_table(k) != PIC_OK) throw pic_last_error();
}
