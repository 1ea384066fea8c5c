// Checkpoint / resume of a pi computation at its phase boundaries (see
// checkpoint.cu for the file format).
#pragma once
#include <stdint.h>

#include <vector>

#include "bigfloat.hpp"

namespace pic {

struct CkptNumber {
    bool sign;
    int64_t exp;
    std::vector<uint32_t> words;
};

// dir == nullptr disables; flags: PIC_CKPT_WRITE | PIC_CKPT_RESUME.
void checkpoint_configure(const char* dir, int flags);
// Test hook: after writing the checkpoint of `phase`, stop the computation
// with PIC_ERR_STOPPED (0 = never).
void checkpoint_debug_stop_after(int phase);
// The phase a resumed computation starts after (0: none), P and Q loaded.
int checkpoint_resume(uint64_t digits, uint64_t p_words, BigFloat* P, BigFloat* Q);
// Writes the state at the end of `phase` (Q may be null).
void checkpoint_save(int phase, uint64_t digits, uint64_t p_words, uint64_t terms, const BigFloat* P,
                     const BigFloat* Q);
// Reads a checkpoint file's header (and with verify, every number and its
// hash).  Returns -1 if the file cannot be opened; throws PIC_ERR_IO if it is
// not a valid checkpoint.
int checkpoint_inspect_file(const char* path, uint64_t* digits, uint64_t* p_words, uint32_t* phase, bool verify,
                            std::vector<CkptNumber>* numbers);
uint64_t ckpt_hash(const uint32_t* w, size_t n);

}  // namespace pic
