// Batched binary splitting.
#include "bsr.cuh"
#include "pi.cuh"

namespace pic {

void bsr_chosen(BigFloat& P, BigFloat& Q, BigFloat& R, uint32_t a, uint32_t b, size_t p)
{
    bsr_recursive(P, Q, R, a, b, p);
}

}  // namespace pic
