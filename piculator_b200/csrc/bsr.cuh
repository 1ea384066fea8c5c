// Chudnovsky binary splitting (PI.h:64-136), batched form.
#pragma once
#include <stdint.h>

#include "bigfloat.hpp"

namespace pic {

// Same P, Q, R as Pi_BSR(P, Q, R, a, b, p) word for word.  need_root_R =
// false skips the root's R = R0 R1, which Pi() never reads (PI.h:176-181);
// R is then left empty.
void bsr_chosen(BigFloat& P, BigFloat& Q, BigFloat& R, uint32_t a, uint32_t b, size_t p,
                bool need_root_R = true);
void bsr_set_school_threshold(uint32_t words);
uint32_t bsr_school_threshold();
// Wrapped products in the NTT merges (main transform at the smaller power of
// two plus a short tail product); on by default.
void bsr_set_wrap(bool on);
// CTA schoolbook merges take one Karatsuba level for products whose operands
// both have at least this many words (0: plain schoolbook).
void bsr_set_karatsuba(uint32_t min_words);
uint32_t bsr_karatsuba();
bool bsr_wrap();
// Kernels for the short schoolbook levels: 0 one CTA per parent, 1 also one
// warp per parent (nodes <= 64 words), 2 also one thread per parent (nodes
// <= 28 words, the default).
void bsr_set_small_merge(int mode);
// P of the batched NTT merges formed in the transform domain (one inverse
// transform and one conversion instead of two; on by default).
void bsr_set_combine(bool on);
bool bsr_combine();
int bsr_small_merge();

}  // namespace pic
