/*
 * ntt_b200 64-bit word variant (C ABI): RNS negacyclic NTT / INTT over
 * uint64 limbs with primes below 2^62.
 *
 * The reference's v04 path works on 32-bit words only; its Cheddar handler
 * is also instantiated for 64-bit words (src/NTT_cheddar.cu:1313,
 * `template class NTTHandler<uint64_t>`), whose source is not part of the
 * reference checkout.  This variant gives the 64-bit word width the same
 * contract as the 32-bit plans (include/ntt_b200.h), with R = 2^64:
 *   forward: normal-domain input in [0, q) -> Montgomery-domain output
 *            (x * 2^64 mod q), bit-reversed order, canonical [0, q);
 *   inverse: Montgomery-domain bit-reversed input in [0, q) -> normal-domain
 *            output in natural order, N^{-1} applied, canonical;
 *   layout:  limb-major, A[poly * poly_stride + limb * N + i], in place;
 *   psi = root^((q - 1) / 2N), table tw[i] = psi^bitrev(i, logN).
 * Arithmetic: 64-bit Shoup products with Harvey's lazy [0, 4q) ranges
 * (hence q < 2^62).  Kernels: logN <= 12 in one launch (a CTA per limb);
 * larger sizes in two launches per direction (the column stages, then the
 * row stages), each CTA holding <= 2^12 words of a few adjacent columns /
 * rows in shared memory and running their stages as register passes of up
 * to four stages (16 words per thread) with one barrier per pass.  No
 * reference counterpart for the kernels themselves.
 */
#ifndef NTT_B200_U64_H
#define NTT_B200_U64_H
#include "ntt_b200.h"
#ifdef __cplusplus
extern "C" {
#endif

#define NTT64_MIN_LOGN 1
#define NTT64_MAX_LOGN 17

typedef struct ModulusConfig64 {
    uint64_t qi;             /* prime, q == 1 (mod 2N), q < 2^62              */
    uint64_t primitive_root; /* g with g^((q-1)/2) == -1 (mod q): then
                                psi = g^((q-1)/2N) is a primitive 2N-th root  */
} ModulusConfig64;

typedef struct ntt64_plan ntt64_plan_t;

/* The first `count` primes q >= lower_bound with q == 1 (mod 2N) and
 * q < 2^62, ascending, each with its smallest quadratic non-residue as root
 * (deterministic Miller-Rabin for 64-bit integers). */
NTT_API ntt_status_t ntt64_find_moduli(int logN, int count, uint64_t lower_bound,
                                       ModulusConfig64* out);
/* Validates every modulus (prime, q == 1 mod 2N, q < 2^62, psi^N == -1,
 * NTT_ERR_MODULUS / _ROOT / _MODULUS_RANGE otherwise) and uploads the
 * limbs' forward and inverse Shoup tables to the current device. */
NTT_API ntt_status_t ntt64_plan_create(int logN, const ModulusConfig64* moduli, int limbs,
                                       ntt64_plan_t** out);
NTT_API ntt_status_t ntt64_plan_destroy(ntt64_plan_t* plan);
/* `polys` polynomials of limbs * N uint64 words, poly_stride words apart
 * (0 = packed, else >= limbs * N); 16-byte aligned.  One (logN <= 12) or two
 * launches on `stream`. */
NTT_API ntt_status_t ntt64_forward_many(const ntt64_plan_t* plan, uint64_t* a_dev, size_t polys,
                                        size_t poly_stride, ntt_stream_t stream);
NTT_API ntt_status_t ntt64_inverse_many(const ntt64_plan_t* plan, uint64_t* a_dev, size_t polys,
                                        size_t poly_stride, ntt_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif
