// H_eff matvec with all scratch in a static device array (no device allocation).
#pragma once

#include "common.cuh"

// bytes of the static scratch array; must equal the value the public header states
#define NOALLOC_SCRATCH_BYTES (64ull << 20)

namespace dmrg2 {

// scratch bytes heff_noalloc needs for these shapes (WWt + X + Y, each 256-byte aligned)
size_t heff_noalloc_scratch_bytes(int cL, int cR, int d, int Dl, int Dr, size_t scalar_bytes);

// out = H_eff theta with every operand already on the current device; enqueued on s,
// no synchronisation, no allocation. Throws std::invalid_argument when the shapes
// need more than NOALLOC_SCRATCH_BYTES of scratch.
template <typename T>
void heff_noalloc(int cL, int cR, int d, int Dl, int Dm, int Dr, const T* L, const T* R, const T* WL,
                  const T* WR, const T* theta, T* out, cudaStream_t s);

}  // namespace dmrg2
