// Pointwise Montgomery product launcher (pointwise.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace nttb {
// c = a (.) b per limb modulus q[limb], over `polys` polynomials of `limbs`
// limbs of 2^logN words (logN >= 2), polynomial p at + p * stride words;
// 16-byte aligned.
cudaError_t launch_pointwise(uint32_t* c, const uint32_t* a, const uint32_t* b,
                             const uint32_t* q, int limbs, int logN, size_t polys,
                             size_t stride, cudaStream_t s);
}  // namespace nttb
