/* Drop-in check: the reference's NTT.h (NTT.h:4-9) as seen by its PI.h.
 * Pi() only calls ntt_ensure_table (PI.h:146); it forwards to the library's
 * table build for the reference's prime of that length. */
#pragma once
#include "piculator_b200.h"

inline void ntt_ensure_table(int k)
{
    if (pic_ntt_ensure_table(k) != PIC_OK) throw pic_last_error();
}
