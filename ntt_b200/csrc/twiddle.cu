// Device-side twiddle generation and import (sm_100a).
//
// Table layout (per limb, N entries of (w, w') uint32 pairs, w' the Shoup
// companion floor(w * 2^32 / q)):
//   forward  entry i >= 2: psi^bitrev(i)      (the reference's
//            make_twiddle_table, src/v04_montgomery.cu:720-727, kept in the
//            normal domain because Shoup products need no Montgomery form)
//            entry 0: R mod q            (R = 2^32; folded normal->Montgomery
//                                         conversion of the input, v04:229-232)
//            entry 1: psi^bitrev(1) * R  (limb stage 0's only twiddle, with R)
//   inverse  entry i >= 2: psi^-bitrev(i)
//            entry 0: c = N^-1 * R^-1    (the reference's NormalizeKernel,
//                                         v04:567-580, folded into the last
//                                         stage: N^-1 and from_mont)
//            entry 1: psi^-bitrev(1) * c
// Entry i is stored at slot tw_slot(i, logN) (arith.cuh): the last four
// stages' blocks are interleaved for coalesced loads.
#include <cuda_runtime.h>
#include <cstdint>
#include "arith.cuh"
#include "twiddle.h"

namespace nttb {

__device__ __forceinline__ uint32_t dev_redc(uint64_t t, uint32_t q, uint32_t nqinv) {
    uint32_t m = (uint32_t)t * nqinv;
    uint64_t u = (t + (uint64_t)m * q) >> 32;
    return (uint32_t)(u >= q ? u - q : u);
}

__device__ __forceinline__ uint32_t dev_brev(uint32_t v, int width) {
    return __brev(v) >> (32 - width);
}

// base^e mod q by Montgomery square-and-multiply (q < 2^31), normal domain.
__device__ uint32_t gen_pow(const TwGenLimb& L, uint32_t e) {
    uint32_t x = dev_redc((uint64_t)L.base * L.r2, L.q, L.nqinv);  // base * R
    uint32_t acc = L.r_mod;                                          // 1 * R
    while (e) {
        if (e & 1u) acc = dev_redc((uint64_t)acc * x, L.q, L.nqinv);
        x = dev_redc((uint64_t)x * x, L.q, L.nqinv);
        e >>= 1;
    }
    return dev_redc(acc, L.q, L.nqinv);  // leave the Montgomery domain
}

// One thread per table entry; blockIdx.y = limb.
__global__ void twiddle_gen_kernel(TwPair* out, const TwGenLimb* limbs, int logN) {
    const uint32_t N = 1u << logN;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const TwGenLimb L = limbs[blockIdx.y];
    const uint32_t w = i == 0 ? L.fold0 : i == 1 ? L.fold1 : gen_pow(L, dev_brev(i, logN));
    out[(size_t)blockIdx.y * N + tw_slot(i, logN)] =
        TwPair{w, (uint32_t)(((uint64_t)w << 32) / L.q)};
}

// Compressed tables (arith.cuh, tw_comp_*): one thread per slot of
// tw_comp_entries(logN) per limb.  Slots below N/16 hold entries 0 .. N/16-1
// (the folded 0 and 1 included), then four base blocks of N/32 entries
// (stages logN-4 .. logN-1: entry H + m F), then the 16 unit-step factors
// base^bitrev(c), factor 0 = 1, never folded.
__global__ void twiddle_gen_comp_kernel(TwPair* out, const TwGenLimb* limbs, int logN) {
    const uint32_t N = 1u << logN, S = N >> 5, E = tw_comp_entries(logN);
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= E) return;
    const TwGenLimb L = limbs[blockIdx.y];
    uint32_t w;
    if (k >= 6 * S) {
        w = gen_pow(L, dev_brev(k - 6 * S, logN));
    } else {
        uint32_t i = k;
        if (k >= 2 * S) {
            const uint32_t b = (k - 2 * S) / S, m = (k - 2 * S) % S;  // block b: p = 3 - b
            i = (N >> (4 - b)) + m * (2u << b);
        }
        w = i == 0 ? L.fold0 : i == 1 ? L.fold1 : gen_pow(L, dev_brev(i, logN));
    }
    out[(size_t)blockIdx.y * E + k] = TwPair{w, (uint32_t)(((uint64_t)w << 32) / L.q)};
}

// Import the reference's Montgomery-form tables (tw_mont[i] = to_mont(w_i)).
// Forward: fold0 = R = redc(r2), fold1 = tw_mont[1] itself (= w_1 * R).
// Inverse: fold0 = c = redc(redc(degree_inv_mont)), fold1 = w_1 * c.
__device__ __forceinline__ uint32_t import_entry(const uint32_t* t, uint32_t i, uint32_t q,
                                                 uint32_t qi, uint32_t aux, int inverse) {
    if (!inverse) {
        if (i == 0) return dev_redc(aux, q, qi);
        if (i == 1) return t[1] % q;
        return dev_redc(t[i], q, qi);
    }
    const uint32_t c = dev_redc(dev_redc(aux, q, qi), q, qi);
    if (i == 0) return c;
    if (i == 1) return (uint32_t)(((uint64_t)dev_redc(t[1], q, qi) * c) % q);
    return dev_redc(t[i], q, qi);
}

__global__ void twiddle_import_kernel(TwPair* out, const uint32_t* tw_mont,
                                      const uint32_t* moduli, const uint32_t* nqinv,
                                      const uint32_t* aux, int logN, int inverse) {
    const uint32_t N = 1u << logN;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const uint32_t l = blockIdx.y;
    const uint32_t q = moduli[l];
    const uint32_t w = import_entry(tw_mont + (size_t)l * N, i, q, nqinv[l], aux[l], inverse);
    out[(size_t)l * N + tw_slot(i, logN)] = TwPair{w, (uint32_t)(((uint64_t)w << 32) / q)};
}

// Stream-ordered refresh of a converted table against the caller's
// Montgomery-form table, once per drop-in call: entry i of limb l is
// re-derived when its source word, or the limb's modulus, -q^{-1} or
// auxiliary constant, differs from the shadow copy it was derived from.
// `force` re-derives every entry (the first call).
// Shadow layout: limbs * N source words, then (q, qinv, aux) per limb, then
// a block counter and a status word.  Every block compares the limb
// parameters against their shadows; the last block to finish (the counter)
// stores the new parameters, so no block can see half-updated shadows.  A
// modulus that is even or not below 2^31 sets status bit 0 (the converted
// entries would be meaningless; ntt_shim_check reports it).
__global__ void shim_refresh_kernel(TwPair* out, uint32_t* shadow, const uint32_t* tw_mont,
                                    const uint32_t* moduli, const uint32_t* nqinv,
                                    const uint32_t* aux, int limbs, int logN, int inverse,
                                    int force) {
    const uint32_t N = 1u << logN;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t l = blockIdx.y;
    uint32_t* params = shadow + (size_t)limbs * N;
    uint32_t* counter = params + 3 * (size_t)limbs;
    uint32_t* status = counter + 1;
    const uint32_t q = moduli[l], qi = nqinv[l], ax = aux[l];
    const bool changed = force || q != params[3 * l] || qi != params[3 * l + 1] || ax != params[3 * l + 2];
    if (i < N) {
        const uint32_t* t = tw_mont + (size_t)l * N;
        const uint32_t src = t[i];
        uint32_t* sh = shadow + (size_t)l * N + i;
        if (changed || src != *sh) {
            if ((q & 1u) && q < (1u << 31)) {
                const uint32_t w = import_entry(t, i, q, qi, ax, inverse);
                out[(size_t)l * N + tw_slot(i, logN)] =
                    TwPair{w, (uint32_t)(((uint64_t)w << 32) / q)};
            } else if (i == 0) {
                atomicOr(status, 1u);
            }
            *sh = src;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t blocks = gridDim.x * gridDim.y;
        if (atomicAdd(counter, 1u) == blocks - 1) {
            __threadfence();
            for (int k = 0; k < limbs; ++k) {
                params[3 * k] = moduli[k];
                params[3 * k + 1] = nqinv[k];
                params[3 * k + 2] = aux[k];
            }
            *counter = 0;
        }
    }
}

cudaError_t launch_twiddle_gen(TwPair* out, const TwGenLimb* limbs_dev, int limbs, int logN,
                               cudaStream_t s) {
    const uint32_t N = 1u << logN;
    dim3 block(N < 256 ? N : 256), grid((N + block.x - 1) / block.x, limbs);
    twiddle_gen_kernel<<<grid, block, 0, s>>>(out, limbs_dev, logN);
    return cudaGetLastError();
}

cudaError_t launch_twiddle_gen_comp(TwPair* out, const TwGenLimb* limbs_dev, int limbs, int logN,
                                    cudaStream_t s) {
    const uint32_t E = tw_comp_entries(logN);
    dim3 block(256), grid((E + 255) / 256, limbs);
    twiddle_gen_comp_kernel<<<grid, block, 0, s>>>(out, limbs_dev, logN);
    return cudaGetLastError();
}

cudaError_t launch_twiddle_import(TwPair* out, const uint32_t* tw_mont, const uint32_t* moduli,
                                  const uint32_t* nqinv, const uint32_t* aux, int limbs,
                                  int logN, int inverse, cudaStream_t s) {
    const uint32_t N = 1u << logN;
    dim3 block(N < 256 ? N : 256), grid((N + block.x - 1) / block.x, limbs);
    twiddle_import_kernel<<<grid, block, 0, s>>>(out, tw_mont, moduli, nqinv, aux, logN,
                                                 inverse);
    return cudaGetLastError();
}

cudaError_t launch_shim_refresh(TwPair* out, uint32_t* shadow, const uint32_t* tw_mont,
                                const uint32_t* moduli, const uint32_t* nqinv,
                                const uint32_t* aux, int limbs, int logN, int inverse,
                                int force, cudaStream_t s) {
    const uint32_t N = 1u << logN;
    dim3 block(N < 256 ? N : 256), grid((N + block.x - 1) / block.x, limbs);
    shim_refresh_kernel<<<grid, block, 0, s>>>(out, shadow, tw_mont, moduli, nqinv, aux, limbs,
                                               logN, inverse, force);
    return cudaGetLastError();
}

}  // namespace nttb
