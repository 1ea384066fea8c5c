// pic::BigFloat -- drop-in for the reference's class BigFloat (BigFloat.h:8-46)
// with the words resident in B200 HBM.
//
// Same public API and the same semantics word for word: sign / exp / L / T
// with exp in 32-bit words, precision p in words plus two guard words
// (YCL_BIGFLOAT_EXTRA_PRECISION, BigFloat.h:6), p == 0 meaning exact.  The
// `threads` arguments are accepted for source compatibility; parallelism comes
// from the GPU.  Words are immutable once written, so copies share storage and
// operand truncation (BigFloat.cpp:355-366) is a pointer offset, not a copy.
#pragma once
#include <stdint.h>

#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

namespace pic {

// Device words shared between BigFloat values (a truncated operand is a view).
struct WordStore {
    uint32_t* base = nullptr;
    size_t bytes = 0;
    ~WordStore();
};

// Multiply form used by BigFloat::mul (PIC_MUL_*), per thread.
void set_mul_mode(int mode);
int get_mul_mode();

class BigFloat {
public:
    BigFloat(BigFloat&& x) noexcept;
    BigFloat(const BigFloat& x);
    BigFloat& operator=(BigFloat&& x) noexcept;
    BigFloat& operator=(const BigFloat& x);

    BigFloat();
    BigFloat(uint32_t x, bool sign = true);

    std::string to_string_dec(size_t digits = 0) const;
    std::string to_string_hex(size_t digits = 0) const;
    size_t get_precision() const { return L; }
    int64_t get_exponent() const { return exp; }
    uint32_t word_at(int64_t mag) const;

    void negate();
    BigFloat mul(uint32_t x) const;
    BigFloat add(const BigFloat& x, size_t p = 0) const;
    BigFloat sub(const BigFloat& x, size_t p = 0) const;
    BigFloat mul(const BigFloat& x, size_t p = 0, int threads = 1) const;
    BigFloat rcp(size_t p, int threads = 1) const;
    BigFloat div(const BigFloat& x, size_t p, int threads = 1) const;

    // ---- extensions beyond the reference API ----
    static BigFloat from_host(bool sign, int64_t exp, const uint32_t* words, size_t L);
    // Adopts device words [ptr, ptr + L) owned by `store`.
    static BigFloat from_device(bool sign, int64_t exp, std::shared_ptr<WordStore> store, const uint32_t* ptr,
                                size_t L);
    void to_host(uint32_t* words) const;
    std::vector<uint32_t> words() const;
    bool get_sign() const { return sign; }
    const uint32_t* device_words() const { return T; }
    void set_exponent(int64_t e) { exp = e; }
    // Writes to_string_hex into a host buffer without building a std::string.
    size_t hex_into(size_t digits, char* out, size_t cap) const;
    int ucmp(const BigFloat& x) const;

private:
    bool sign;      // true = positive or zero
    int64_t exp;    // exponent, in words
    size_t L;       // length, in words
    const uint32_t* T = nullptr;
    std::shared_ptr<WordStore> store;

    BigFloat uadd(const BigFloat& x, size_t p) const;
    BigFloat usub(const BigFloat& x, size_t p) const;

    friend BigFloat invsqrt(uint32_t x, size_t p, int threads);
};

BigFloat invsqrt(uint32_t x, size_t p, int threads = 1);

// Allocates L words of device memory on the library stream.
std::shared_ptr<WordStore> alloc_words(size_t L);

}  // namespace pic
