#pragma once
#include <stdint.h>

#include "bigfloat.hpp"

namespace pic {

void pi_sizes(uint64_t decimal_digits, uint64_t* hex_digits, uint64_t* p_words, uint64_t* terms);
void bsr_recursive(BigFloat& P, BigFloat& Q, BigFloat& R, uint32_t a, uint32_t b, size_t p);
// The final P of Pi() (before to_string_hex); fills *st when non-null.
BigFloat pi_compute(uint64_t decimal_digits, int mode, pic_pi_stats* st);

}  // namespace pic
