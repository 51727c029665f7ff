// Twiddle-table construction on the device (see twiddle.cu for the layout).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "arith.cuh"

namespace nttb {

// Per-limb inputs of the generation kernel (all normal-domain values).
struct TwGenLimb {
    uint32_t q;
    uint32_t nqinv;  // -q^{-1} mod 2^32
    uint32_t r_mod;  // 2^32 mod q
    uint32_t r2;     // 2^64 mod q
    uint32_t base;   // psi (forward) or psi^{-1} (inverse)
    uint32_t fold0;  // entry 0
    uint32_t fold1;  // entry 1
};

cudaError_t launch_twiddle_gen(TwPair* out, const TwGenLimb* limbs_dev, int limbs, int logN,
                               cudaStream_t s);
// Compressed tables (arith.cuh, tw_comp_*): tw_comp_entries(logN) pairs per
// limb, logN >= kTwCompMinLogN.
cudaError_t launch_twiddle_gen_comp(TwPair* out, const TwGenLimb* limbs_dev, int limbs, int logN,
                                    cudaStream_t s);
cudaError_t launch_twiddle_import(TwPair* out, const uint32_t* tw_mont, const uint32_t* moduli,
                                  const uint32_t* nqinv, const uint32_t* aux, int limbs,
                                  int logN, int inverse, cudaStream_t s);
// shadow: limbs * N + 3 * limbs + 2 words, zeroed before the first (forced)
// call.
cudaError_t launch_shim_refresh(TwPair* out, uint32_t* shadow, const uint32_t* tw_mont,
                                const uint32_t* moduli, const uint32_t* nqinv,
                                const uint32_t* aux, int limbs, int logN, int inverse,
                                int force, cudaStream_t s);

}  // namespace nttb
