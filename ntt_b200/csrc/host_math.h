// Host-side number theory for plan construction (C++17, no CUDA).
//
// Same formulas as the reference's host precompute (src/v04_montgomery.cu:
// pow_mod 660-670, bit_reverse 672-679, mont_q_inv 125-131, mont_r2 138-141,
// to_mont 133-136, make_modulus_runtime 681-718), so that every derived
// constant -- and therefore every twiddle -- is the value the reference uses.
// Inverses are taken with Fermat's exponent q-2 exactly as the reference
// does.  The modulus search (primality, smallest generator) has no
// reference counterpart.
#pragma once
#include <cstdint>
#include <vector>

namespace nttb {
namespace hm {

inline uint32_t mulmod(uint32_t a, uint32_t b, uint32_t q) {
    return (uint32_t)(((uint64_t)a * b) % q);
}

inline uint32_t powmod(uint32_t base, uint64_t e, uint32_t q) {
    uint64_t r = 1 % q, x = base % q;
    while (e) {
        if (e & 1) r = (r * x) % q;
        x = (x * x) % q;
        e >>= 1;
    }
    return (uint32_t)r;
}

inline uint32_t bitrev(uint32_t v, int width) {
    uint32_t r = 0;
    for (int i = 0; i < width; ++i) {
        r = (r << 1) | (v & 1u);
        v >>= 1;
    }
    return r;
}

// -q^{-1} mod 2^32 (Newton iteration on the 2-adic inverse).
inline uint32_t neg_qinv(uint32_t q) {
    uint32_t inv = 1;
    for (int i = 0; i < 5; ++i) inv *= 2u - q * inv;
    return 0u - inv;
}

inline uint32_t r_mod(uint32_t q) { return (uint32_t)((uint64_t{1} << 32) % q); }
inline uint32_t r2_mod(uint32_t q) {
    uint64_t r = r_mod(q);
    return (uint32_t)((r * r) % q);
}
inline uint32_t to_mont(uint32_t x, uint32_t q) { return mulmod(x, r_mod(q), q); }

// Deterministic Miller-Rabin for n < 2^32 (bases 2, 7, 61).
inline bool is_prime(uint32_t n) {
    if (n < 2) return false;
    static const uint32_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (uint32_t p : small)
        if (n % p == 0) return n == p;
    uint32_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) {
        d >>= 1;
        ++s;
    }
    for (uint32_t a : {2u, 7u, 61u}) {
        uint32_t x = powmod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool comp = true;
        for (int i = 1; i < s; ++i) {
            x = mulmod(x, x, n);
            if (x == n - 1) {
                comp = false;
                break;
            }
        }
        if (comp) return false;
    }
    return true;
}

inline uint32_t smallest_generator(uint32_t q) {
    std::vector<uint32_t> f;
    uint32_t n = q - 1;
    for (uint32_t p = 2; (uint64_t)p * p <= n; p += (p == 2 ? 1 : 2)) {
        if (n % p == 0) {
            f.push_back(p);
            while (n % p == 0) n /= p;
        }
    }
    if (n > 1) f.push_back(n);
    for (uint32_t g = 2; g < q; ++g) {
        bool ok = true;
        for (uint32_t p : f)
            if (powmod(g, (q - 1) / p, q) == 1) {
                ok = false;
                break;
            }
        if (ok) return g;
    }
    return 0;
}

}  // namespace hm
}  // namespace nttb
