// Pointwise Montgomery product of two spectra (ntt_pointwise_mul).
//
// c[i] = a[i] * b[i] * 2^-32 mod q_limb for NTT-domain operands: forward
// outputs are x * 2^32 (Montgomery domain), so the product of two of them is
// again a Montgomery-domain spectrum, ready for the inverse transform.  The
// reference has no such kernel; it is the middle step of the unfused
// negacyclic multiply (forward, forward, pointwise, inverse), which the batch
// kernel's multiply tiles do in one pass.  HBM-bound: 12 bytes per word.
#include <cuda_runtime.h>

#include "arith.cuh"
#include "pdl.cuh"
#include "pointwise.h"

namespace nttb {

__global__ void __launch_bounds__(256) pointwise_kernel(uint32_t* c, const uint32_t* a,
                                                        const uint32_t* b, const uint32_t* q,
                                                        uint32_t limbs, uint32_t logn,
                                                        uint32_t rows, unsigned long long stride) {
    pdl_enter();
    const uint32_t vecs = (1u << logn) >> 2;
    for (uint32_t row = blockIdx.y; row < rows; row += gridDim.y) {
        const uint32_t poly = row / limbs, limb = row - poly * limbs;
        const uint32_t m = __ldg(q + limb);
        // -m^{-1} mod 2^32 by Newton's iteration (m odd: m is its own inverse mod 8)
        uint32_t x = m;
        for (int i = 0; i < 4; ++i) x *= 2u - m * x;
        const uint32_t nqinv = 0u - x;
        const size_t base = (size_t)poly * stride + ((size_t)limb << logn);
        const uint4* av = reinterpret_cast<const uint4*>(a + base);
        const uint4* bv = reinterpret_cast<const uint4*>(b + base);
        uint4* cv = reinterpret_cast<uint4*>(c + base);
        for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < vecs;
             v += gridDim.x * blockDim.x) {
            const uint4 s = __ldcs(av + v), t = __ldcs(bv + v);
            __stcs(cv + v, make_uint4(mont_mul(s.x, t.x, m, nqinv), mont_mul(s.y, t.y, m, nqinv),
                                      mont_mul(s.z, t.z, m, nqinv), mont_mul(s.w, t.w, m, nqinv)));
        }
    }
}

cudaError_t launch_pointwise(uint32_t* c, const uint32_t* a, const uint32_t* b,
                             const uint32_t* q, int limbs, int logN, size_t polys,
                             size_t stride, cudaStream_t s) {
    const size_t rows = polys * (size_t)limbs;
    if (rows == 0) return cudaSuccess;
    const uint32_t vecs = (1u << logN) >> 2;
    const uint32_t bx = (vecs + 255) / 256 < 16 ? (vecs + 255) / 256 : 16;
    const uint32_t by = rows < 65535 ? (uint32_t)rows : 65535u;
    return launch_pdl(pointwise_kernel, dim3(bx, by), dim3(256), 0, s, c, a, b, q,
                      (uint32_t)limbs, (uint32_t)logN, (uint32_t)rows, stride);
}

}  // namespace nttb
