/*
 * CPU oracle for the RNS negacyclic NTT / INTT path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: only tests/, the smoke
 * check in __graft_entry__.py and the cpu_baseline leg of bench.py may load it.
 * The product library (ntt_b200/) never links, loads or calls it.
 *
 * It restates, in plain C, the host-side algorithm of the reference
 * (vnny27/NTT, src/v04_montgomery.cu, "v04" below):
 *   - scalar modular helpers           v04:93-146, v04:660-679
 *   - per-limb modulus precompute      v04:681-718   (make_modulus_runtime)
 *   - bit-reversed twiddle tables      v04:720-727   (make_twiddle_table)
 *   - textbook CT NTT / GS INTT        v04:742-784   (cpu_ntt_butterfly,
 *                                                     cpu_intt_butterfly)
 *   - seeded input generator           v04:786-797   (fill_random: std::mt19937
 *     seeded per limb, std::uniform_int_distribution<uint32_t>(0, q-1) as
 *     implemented by libstdc++ 13 -- Lemire's nearly divisionless method)
 * plus independent checks the reference does not have: an O(N^2) direct
 * evaluation of the same bit-reversed negacyclic transform and a schoolbook
 * negacyclic product.
 *
 * Errors are returned as codes instead of the reference's std::exit.
 * The pinning of this restatement against the reference's own compiled CPU
 * functions lives in tests/test_oracle.py (golden fixtures in tests/golden/).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define ORACLE_OK 0
#define ORACLE_ERR_MODULUS 1 /* q != 1 mod 2N (v04:685-689)                    */
#define ORACLE_ERR_ROOT 2    /* psi is not a primitive 2N-th root (v04:703-707) */
#define ORACLE_ERR_ARG 3

typedef struct {
    uint32_t qi;
    uint32_t primitive_root;
    uint32_t q_inv; /* -q^{-1} mod 2^32 */
    uint32_t r2;    /* R^2 mod q, R = 2^32 */
    uint32_t psi;
    uint32_t psi_inv;
    uint32_t omega;
    uint32_t degree_inv;
} oracle_modulus_runtime_t; /* field order of ModulusRuntime, v04:17-26 */

/* ---- scalar helpers ------------------------------------------------------ */

/* v04:93-97 */
uint32_t oracle_add_mod(uint32_t a, uint32_t b, uint32_t q) {
    uint64_t s = (uint64_t)a + b;
    if (s >= q) s -= q;
    return (uint32_t)s;
}

/* v04:99-102 */
uint32_t oracle_sub_mod(uint32_t a, uint32_t b, uint32_t q) {
    if (a >= b) return a - b;
    return (uint32_t)((uint64_t)a + q - b);
}

/* v04:104-108 */
uint32_t oracle_mul_mod(uint32_t a, uint32_t b, uint32_t q) {
    return (uint32_t)(((uint64_t)a * b) % q);
}

/* v04:660-670: square-and-multiply with % reduction */
uint32_t oracle_pow_mod(uint32_t base, uint64_t exp, uint32_t mod) {
    uint64_t result = 1, x = base;
    while (exp > 0) {
        if (exp & 1) result = (result * x) % mod;
        x = (x * x) % mod;
        exp >>= 1;
    }
    return (uint32_t)result;
}

/* v04:672-679 */
uint32_t oracle_bit_reverse(uint32_t value, int width) {
    uint32_t r = 0;
    for (int i = 0; i < width; ++i) {
        r = (r << 1) | (value & 1u);
        value >>= 1;
    }
    return r;
}

/* v04:125-131: Newton iteration for q^{-1} mod 2^32, returned negated */
uint32_t oracle_mont_q_inv(uint32_t q) {
    uint32_t inv = 1;
    for (int i = 0; i < 5; ++i) inv *= 2u - q * inv;
    return 0u - inv;
}

/* v04:138-141 */
uint32_t oracle_mont_r2(uint32_t q) {
    uint64_t r = ((uint64_t)1 << 32) % q;
    return (uint32_t)((r * r) % q);
}

/* v04:133-136 */
uint32_t oracle_to_mont(uint32_t x, uint32_t q) {
    uint64_t r = ((uint64_t)1 << 32) % q;
    return (uint32_t)(((uint64_t)x * r) % q);
}

/* v04:110-118 (REDC with q_inv = -q^{-1} mod 2^32; requires q < 2^31) */
uint32_t oracle_mont_reduce(uint64_t t, uint32_t q, uint32_t q_inv) {
    uint32_t m = (uint32_t)t * q_inv;
    uint64_t u = (t + (uint64_t)m * q) >> 32;
    if (u >= q) u -= q;
    return (uint32_t)u;
}

/* v04:120-123 */
uint32_t oracle_mont_mul(uint32_t a, uint32_t b, uint32_t q, uint32_t q_inv) {
    return oracle_mont_reduce((uint64_t)a * b, q, q_inv);
}

/* v04:143-146 */
uint32_t oracle_from_mont(uint32_t x, uint32_t q, uint32_t q_inv) {
    return oracle_mont_mul(x, 1u, q, q_inv);
}

/* ---- per-limb precompute ------------------------------------------------- */

/* v04:681-718.  Same formulas (Fermat inverses, psi = g^((q-1)/2N)), same two
 * validity checks, but a status code instead of std::exit. */
int oracle_modulus_runtime(int logN, uint32_t qi, uint32_t g,
                           oracle_modulus_runtime_t* out) {
    if (logN < 1 || logN > 30 || qi < 3 || !out) return ORACLE_ERR_ARG;
    uint64_t N = (uint64_t)1 << logN;
    uint64_t order = 2 * N;
    if (((uint64_t)qi - 1) % order != 0) return ORACLE_ERR_MODULUS;
    uint32_t psi = oracle_pow_mod(g, ((uint64_t)qi - 1) / order, qi);
    uint32_t psi_inv = oracle_pow_mod(psi, qi - 2, qi);
    uint32_t omega = (uint32_t)(((uint64_t)psi * psi) % qi);
    uint32_t degree_inv = oracle_pow_mod((uint32_t)N, qi - 2, qi);
    if (oracle_pow_mod(psi, order, qi) != 1 || oracle_pow_mod(psi, N, qi) != qi - 1)
        return ORACLE_ERR_ROOT;
    out->qi = qi;
    out->primitive_root = g;
    out->q_inv = oracle_mont_q_inv(qi);
    out->r2 = oracle_mont_r2(qi);
    out->psi = psi;
    out->psi_inv = psi_inv;
    out->omega = omega;
    out->degree_inv = degree_inv;
    return ORACLE_OK;
}

/* v04:720-727: tw[i] = psi^bitrev(i, logN) mod q, tw[0] = 1 (unused). */
void oracle_twiddle_table(int logN, uint32_t q, uint32_t psi, uint32_t* out) {
    size_t N = (size_t)1 << logN;
    for (size_t i = 0; i < N; ++i)
        out[i] = oracle_pow_mod(psi, oracle_bit_reverse((uint32_t)i, logN), q);
}

/* ---- transforms ---------------------------------------------------------- */

/* v04:742-759: in-place Cooley-Tukey, natural order in, bit-reversed out,
 * twiddle psi[m + j] for butterfly group j of stage m. */
void oracle_ntt(uint32_t* a, int logN, uint32_t q, const uint32_t* psi) {
    size_t N = (size_t)1 << logN, t = N >> 1;
    for (size_t m = 1; m < N; m *= 2) {
        for (size_t j = 0; j < m; ++j) {
            for (size_t k = j * 2 * t; k < j * 2 * t + t; ++k) {
                uint32_t u = a[k];
                uint32_t v = (uint32_t)(((uint64_t)a[k + t] * psi[m + j]) % q);
                a[k] = oracle_add_mod(u, v, q);
                a[k + t] = oracle_sub_mod(u, v, q);
            }
        }
        t >>= 1;
    }
}

/* v04:761-784: in-place Gentleman-Sande, bit-reversed in, natural out, then
 * multiply every coefficient by N^{-1}. */
void oracle_intt(uint32_t* a, int logN, uint32_t q, const uint32_t* inv_psi,
                 uint32_t degree_inv) {
    size_t N = (size_t)1 << logN, t = 1;
    for (size_t m = N >> 1; m >= 1; m >>= 1) {
        for (size_t j = 0; j < m; ++j) {
            for (size_t k = j * 2 * t; k < j * 2 * t + t; ++k) {
                uint32_t u = a[k], v = a[k + t];
                a[k] = oracle_add_mod(u, v, q);
                a[k + t] = oracle_mul_mod(oracle_sub_mod(u, v, q), inv_psi[m + j], q);
            }
        }
        t <<= 1;
        if (m == 1) break;
    }
    for (size_t i = 0; i < N; ++i) a[i] = oracle_mul_mod(a[i], degree_inv, q);
}

/* Independent O(N^2) evaluation of the same map: the CT loop above computes
 * out[j] = sum_i a[i] * psi^((2*bitrev(j, logN) + 1) * i)  (mod q).
 * Not in the reference's call path; used as a known-answer check. */
void oracle_ntt_direct(const uint32_t* a, uint32_t* out, int logN, uint32_t q,
                       uint32_t psi) {
    size_t N = (size_t)1 << logN;
    for (size_t j = 0; j < N; ++j) {
        uint64_t e = 2ull * oracle_bit_reverse((uint32_t)j, logN) + 1;
        uint32_t step = oracle_pow_mod(psi, e, q), w = 1;
        uint64_t acc = 0;
        for (size_t i = 0; i < N; ++i) {
            acc = (acc + (uint64_t)a[i] * w) % q;
            w = (uint32_t)(((uint64_t)w * step) % q);
        }
        out[j] = (uint32_t)acc;
    }
}

/* Coefficient k of the negacyclic product a*b mod (X^N + 1, q), O(N). */
uint32_t oracle_negacyclic_coeff(const uint32_t* a, const uint32_t* b, int logN,
                                 uint32_t q, size_t k) {
    size_t N = (size_t)1 << logN;
    uint64_t pos = 0, neg = 0;
    for (size_t i = 0; i < N; ++i) {
        uint64_t p = ((uint64_t)(a[i] % q) * (b[(k + N - i) % N] % q)) % q;
        if (i <= k) pos += p; else neg += p;
        pos %= q; neg %= q;
    }
    return (uint32_t)((pos + q - neg) % q);
}

/* ---- seeded input generator (v04:786-797) ---------------------------------
 * std::mt19937 (Matsumoto & Nishimura 1998, 32-bit MT with the standard
 * tempering and init_genrand seeding), consumed by libstdc++ 13's
 * uniform_int_distribution<uint32_t>: because mt19937's range is exactly
 * 32 bits, it uses Lemire's nearly divisionless rejection method
 * (ACM TOMACS 29(1), 2019) with a 64-bit product. */
typedef struct { uint32_t mt[624]; int idx; } mt19937_t;

static void mt_seed(mt19937_t* s, uint32_t seed) {
    s->mt[0] = seed;
    for (int i = 1; i < 624; ++i)
        s->mt[i] = 1812433253u * (s->mt[i - 1] ^ (s->mt[i - 1] >> 30)) + (uint32_t)i;
    s->idx = 624;
}

static uint32_t mt_next(mt19937_t* s) {
    if (s->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            uint32_t y = (s->mt[i] & 0x80000000u) | (s->mt[(i + 1) % 624] & 0x7fffffffu);
            s->mt[i] = s->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        s->idx = 0;
    }
    uint32_t y = s->mt[s->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

static uint32_t lemire_bounded(mt19937_t* s, uint32_t range) {
    uint64_t product = (uint64_t)mt_next(s) * range;
    uint32_t low = (uint32_t)product;
    if (low < range) {
        uint32_t threshold = (0u - range) % range;
        while (low < threshold) {
            product = (uint64_t)mt_next(s) * range;
            low = (uint32_t)product;
        }
    }
    return (uint32_t)(product >> 32);
}

/* fill_random(arr, size, q) with the generator seeded by `seed` (the
 * reference re-seeds with SEED = 1234 for every limb, v04:786-797, v04:932-934). */
int oracle_fill_random(uint32_t* arr, size_t size, uint32_t q, uint32_t seed) {
    if (q <= 1) return ORACLE_ERR_ARG;
    mt19937_t s;
    mt_seed(&s, seed);
    for (size_t i = 0; i < size; ++i) arr[i] = lemire_bounded(&s, q);
    return ORACLE_OK;
}

/* ---- multi-limb drivers (threads split limbs, as the CPU baseline does) -- */

typedef struct {
    uint32_t* a;
    int logN;
    const uint32_t* q;
    const uint32_t* tables; /* limbs * N: psi (forward) or psi^-1 (inverse) table */
    const uint32_t* degree_inv; /* NULL for forward */
    int limb_begin, limb_end;
} oracle_job_t;

static void* oracle_worker(void* arg) {
    oracle_job_t* j = (oracle_job_t*)arg;
    size_t N = (size_t)1 << j->logN;
    for (int l = j->limb_begin; l < j->limb_end; ++l) {
        if (j->degree_inv)
            oracle_intt(j->a + (size_t)l * N, j->logN, j->q[l], j->tables + (size_t)l * N,
                        j->degree_inv[l]);
        else
            oracle_ntt(j->a + (size_t)l * N, j->logN, j->q[l], j->tables + (size_t)l * N);
    }
    return NULL;
}

/* Transform `limbs` limbs of a[limb*N + i] in place with `threads` threads.
 * degree_inv == NULL selects the forward transform. */
int oracle_transform_limbs(uint32_t* a, int logN, int limbs, const uint32_t* q,
                           const uint32_t* tables, const uint32_t* degree_inv,
                           int threads) {
    if (threads < 1) threads = 1;
    if (threads > limbs) threads = limbs;
    if (threads > 256) threads = 256;
    pthread_t tid[256];
    oracle_job_t jobs[256];
    int per = limbs / threads, extra = limbs % threads, start = 0;
    for (int t = 0; t < threads; ++t) {
        int cnt = per + (t < extra ? 1 : 0);
        jobs[t] = (oracle_job_t){a, logN, q, tables, degree_inv, start, start + cnt};
        start += cnt;
    }
    for (int t = 1; t < threads; ++t) pthread_create(&tid[t], NULL, oracle_worker, &jobs[t]);
    if (threads > 0) oracle_worker(&jobs[0]);
    for (int t = 1; t < threads; ++t) pthread_join(tid[t], NULL);
    return ORACLE_OK;
}

/* ---- 64-bit words (the 64-bit variant, include/ntt_b200_u64.h) -------------
 * The same textbook CT NTT / GS INTT as oracle_ntt / oracle_intt (v04:742-784)
 * with 64-bit words and 128-bit products, and the same O(N^2) definition.
 * The reference has no 64-bit CPU path in its checkout; these restate the
 * 32-bit algorithm for q < 2^62 and are pinned by the direct evaluation. */
typedef unsigned __int128 oracle_u128;

uint64_t oracle_mul_mod64(uint64_t a, uint64_t b, uint64_t q) {
    return (uint64_t)((oracle_u128)a * b % q);
}

uint64_t oracle_pow_mod64(uint64_t base, uint64_t exp, uint64_t q) {
    uint64_t r = 1 % q;
    base %= q;
    while (exp) {
        if (exp & 1) r = oracle_mul_mod64(r, base, q);
        base = oracle_mul_mod64(base, base, q);
        exp >>= 1;
    }
    return r;
}

/* psi = g^((q-1)/2N) and the bit-reversed tables of psi and psi^{-1}. */
void oracle_tables64(int logN, uint64_t q, uint64_t g, uint64_t* psi_tab, uint64_t* inv_tab,
                     uint64_t* degree_inv) {
    size_t N = (size_t)1 << logN;
    uint64_t psi = oracle_pow_mod64(g, (q - 1) / (2 * N), q);
    uint64_t psi_inv = oracle_pow_mod64(psi, q - 2, q);
    for (size_t i = 0; i < N; ++i) {
        uint32_t e = oracle_bit_reverse((uint32_t)i, logN);
        psi_tab[i] = oracle_pow_mod64(psi, e, q);
        inv_tab[i] = oracle_pow_mod64(psi_inv, e, q);
    }
    *degree_inv = oracle_pow_mod64(N % q, q - 2, q);
}

void oracle_ntt64(uint64_t* a, int logN, uint64_t q, const uint64_t* psi) {
    size_t N = (size_t)1 << logN, t = N >> 1;
    for (size_t m = 1; m < N; m *= 2) {
        for (size_t j = 0; j < m; ++j)
            for (size_t k = j * 2 * t; k < j * 2 * t + t; ++k) {
                uint64_t u = a[k], v = oracle_mul_mod64(a[k + t], psi[m + j], q);
                a[k] = u + v >= q ? u + v - q : u + v;
                a[k + t] = u >= v ? u - v : u + q - v;
            }
        t >>= 1;
    }
}

void oracle_intt64(uint64_t* a, int logN, uint64_t q, const uint64_t* inv_psi,
                   uint64_t degree_inv) {
    size_t N = (size_t)1 << logN, t = 1;
    for (size_t m = N >> 1; m >= 1; m >>= 1) {
        for (size_t j = 0; j < m; ++j)
            for (size_t k = j * 2 * t; k < j * 2 * t + t; ++k) {
                uint64_t u = a[k], v = a[k + t];
                a[k] = u + v >= q ? u + v - q : u + v;
                a[k + t] = oracle_mul_mod64(u >= v ? u - v : u + q - v, inv_psi[m + j], q);
            }
        t <<= 1;
        if (m == 1) break;
    }
    for (size_t i = 0; i < N; ++i) a[i] = oracle_mul_mod64(a[i], degree_inv, q);
}

/* out[j] = sum_i a[i] psi^((2 bitrev(j) + 1) i) mod q. */
void oracle_ntt_direct64(const uint64_t* a, uint64_t* out, int logN, uint64_t q, uint64_t psi) {
    size_t N = (size_t)1 << logN;
    for (size_t j = 0; j < N; ++j) {
        uint64_t step = oracle_pow_mod64(psi, 2ull * oracle_bit_reverse((uint32_t)j, logN) + 1, q);
        uint64_t w = 1, acc = 0;
        for (size_t i = 0; i < N; ++i) {
            acc = (acc + oracle_mul_mod64(a[i], w, q)) % q;
            w = oracle_mul_mod64(w, step, q);
        }
        out[j] = acc;
    }
}
