// Transform-domain operands (see transform.cuh).
#include "mul.cuh"
#include "transform.cuh"

namespace pic {

TransformOperand transform_create(const BigFloat& x, size_t p, int k)
{
    TransformOperand t;
    size_t L = x.get_precision();
    int64_t exp = x.get_exponent();
    const uint32_t* T = x.device_words();
    if (p != 0 && L > p + 2) {
        const size_t chop = L - (p + 2);
        T += chop;
        exp += (int64_t)chop;
        L = p + 2;
    }
    const size_t pieces = (L + 1) / 2;
    if (k == 0) {
        while (((size_t)1 << k) < 2 * pieces) k++;
        if (k < 1) k = 1;
    }
    PIC_REQUIRE(k >= 1 && k <= 30, PIC_ERR_INVALID, "transform length out of range");
    PIC_REQUIRE(((size_t)1 << k) >= pieces, PIC_ERR_LENGTH, "FFT length is too small.");
    t.k = k;
    t.sign = x.get_sign();
    t.exp = exp;
    t.L = L;
    t.depth = 0;
    t.data = std::make_shared<DevBuf<uint64_t>>((size_t)3 << k, ctx().stream);
    ntt3_forward_operand(t.data->get(), k, T, L, ctx().stream);
    return t;
}

void transform_mul(TransformOperand& t1, const TransformOperand& t2)
{
    PIC_REQUIRE(t1.k == t2.k, PIC_ERR_INVALID, "transforms of different lengths");
    PIC_REQUIRE(((size_t)1 << t1.k) >= (t1.L + 1) / 2 + (t2.L + 1) / 2 - 1, PIC_ERR_LENGTH,
                "FFT length is too small.");
    ntt3_pointwise(t1.data->get(), t2.data->get(), t1.k, ctx().stream);
    t1.sign = t1.sign == t2.sign;  // Transform.h:15-17
    t1.exp += t2.exp;
    t1.L += t2.L;
    t1.depth += t2.depth + 1;
}

BigFloat transform_to_bigfloat(const TransformOperand& t)
{
    if (t.L == 0) return BigFloat();
    DevBuf<uint64_t> work((size_t)3 << t.k, ctx().stream);
    PIC_CUDA(cudaMemcpyAsync(work.get(), t.data->get(), sizeof(uint64_t) * ((size_t)3 << t.k),
                             cudaMemcpyDeviceToDevice, ctx().stream));
    auto st = alloc_words(t.L);
    ntt3_inverse_to_words(work.get(), t.k, (t.L + 1) / 2, t.depth, st->base, t.L, ctx().stream);
    size_t L = t.L;
    if (t.depth > 0) {
        uint32_t top;
        read_words(&top, st->base + L - 1, 1, ctx().stream);
        if (top == 0) L--;  // BigFloat.cpp:411-412
    }
    return BigFloat::from_device(t.sign, t.exp, st, st->base, L);
}

}  // namespace pic
