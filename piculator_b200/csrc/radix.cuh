// Decimal output (BigFloat::to_string_dec, BigFloat.cpp:83-94); see radix.cu.
#pragma once
#include <stddef.h>

#include <string>

#include "bigfloat.hpp"

namespace pic {

// The 9 * groups decimal digits of the fraction held below x's top word
// (what the reference's to_string_dec prints after the '.'), as text into
// d_out (device, 9 * groups bytes, not terminated).
void dec_digits(const BigFloat& x, size_t groups, char* d_out);
// The reference's to_string_dec(digits) text.
std::string to_string_dec_fast(const BigFloat& x, size_t digits);

}  // namespace pic
