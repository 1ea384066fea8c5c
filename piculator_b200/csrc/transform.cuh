// Transform-domain operands: the intent of the reference's Transform.h:5-33
// (never included by the reference itself).  An operand's forward three-prime
// NTT is kept with its BigFloat metadata so a factor used by several products
// is transformed once; mulNTT (Transform.h:13-18) becomes a pointwise product
// that also combines sign, exponent and length.
#pragma once
#include <memory>

#include "bigfloat.hpp"

namespace pic {

struct TransformOperand {
    std::shared_ptr<DevBuf<uint64_t>> data;  // 3 x 2^k residues, bit-reversed order
    int k = 0;
    bool sign = true;
    int64_t exp = 0;
    size_t L = 0;
    int depth = 0;  // pointwise Montgomery products folded in (each adds R^-1)
};

// Truncates x to its top p + 2 words when p > 0 (as BigFloat::mul does,
// BigFloat.cpp:337-366) and transforms it at length 2^k (k = 0: long enough
// for the product with an operand of equal length).
TransformOperand transform_create(const BigFloat& x, size_t p, int k);
void transform_mul(TransformOperand& t1, const TransformOperand& t2);
BigFloat transform_to_bigfloat(const TransformOperand& t);

}  // namespace pic
