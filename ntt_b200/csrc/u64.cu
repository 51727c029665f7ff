// 64-bit word variant of the RNS negacyclic NTT / INTT (include/ntt_b200_u64.h).
//
// Same algorithm and table conventions as the 32-bit path (reference:
// cpu_ntt_butterfly / cpu_intt_butterfly and the two-phase kernels of
// src/v04_montgomery.cu:196-580, 742-784) with 64-bit words: Shoup products
// w*a - umulhi(w', a)*q (w' = floor(w * 2^64 / q)) and Harvey's lazy ranges,
// so q < 2^62.  The Montgomery factor R = 2^64 and N^{-1} ride on the
// stage-0 twiddle pair (table entries 0 and 1), as in the 32-bit tables.
//
// Kernel: one stage-range kernel per launch shape.  A CTA loads G
// sub-transforms of 2^k words of a limb into shared memory (G adjacent
// columns of the 2^k x 2^(n-k) limb matrix for the column stages, or G
// adjacent rows for the row stages; both loads coalesced), runs the
// launch's radix-2 stages there, and
// writes the words back in place.  logN <= 12: one launch with all stages on
// whole limbs; larger: the column stages, then the row stages.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "../../include/ntt_b200_u64.h"
#include "pdl.cuh"
#include "runtime.h"

using namespace nttb;

namespace {

typedef unsigned __int128 u128;

struct TwPair64 {
    unsigned long long w, wp;
};

// ---- host arithmetic -------------------------------------------------------
uint64_t mulmod64(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)((u128)a * b % q); }
uint64_t powmod64(uint64_t a, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    a %= q;
    for (; e; e >>= 1, a = mulmod64(a, a, q))
        if (e & 1) r = mulmod64(r, a, q);
    return r;
}
// Deterministic Miller-Rabin for n < 2^64 (the first 12 primes as bases).
bool is_prime64(uint64_t n) {
    if (n < 2) return false;
    static const uint64_t bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (uint64_t p : bases)
        if (n % p == 0) return n == p;
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) {
        d >>= 1;
        ++s;
    }
    for (uint64_t a : bases) {
        uint64_t x = powmod64(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool comp = true;
        for (int r = 1; r < s && comp; ++r) {
            x = mulmod64(x, x, n);
            if (x == n - 1) comp = false;
        }
        if (comp) return false;
    }
    return true;
}
uint32_t bitrev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}
TwPair64 pair_of(uint64_t w, uint64_t q) { return TwPair64{w, (uint64_t)(((u128)w << 64) / q)}; }

// ---- device arithmetic (lazy ranges as Lazy4 in arith.cuh) ------------------
__device__ __forceinline__ uint64_t csub64(uint64_t x, uint64_t m) {
    const uint64_t y = x - m;
    return y < x ? y : x;  // x >= m: x - m; else the subtraction wrapped
}
__device__ __forceinline__ uint64_t shoup64(uint64_t a, TwPair64 w, uint64_t q) {
    return a * w.w - __umul64hi(a, w.wp) * q;  // in [0, 2q)
}

struct U64Args {
    unsigned long long* data;
    const TwPair64* tw;  // [limbs][N]
    const unsigned long long* q;
    unsigned long long stride;  // words between polynomials
    uint32_t limbs, groups;     // sub-transform groups per limb
    int n;                      // logN
};

constexpr int kU64Threads = 256;

// Geometry of one stage-range launch: a CTA holds 2^GL sub-transforms of 2^K
// words, G adjacent columns of the 2^K x 2^(n-K) limb matrix (COL) or G
// adjacent rows, in shared memory at si(g, u).  Compile-time, so that the
// index arithmetic of the passes is shifts and masks.  Rows keep each
// sub-transform contiguous with bits 0..3 of the word index XORed with bits
// 4..7 (a bijection on the 2^K words): the passes over low bits would
// otherwise put 4 to 8 threads of a half-warp on one 8-byte bank; swizzled,
// every pass of K <= 12 has at most 2 (measured before it: 8.5 M bank
// conflicts per row launch at 2^16 x 16 limbs x 16 polynomials).
template <int K_, int GL_, bool COL_>
struct U64Geo {
    static constexpr int K = K_, GL = GL_;
    static constexpr bool COL = COL_;
    static constexpr uint32_t KW = 1u << K, G = 1u << GL, TOTAL = KW << GL;
    static constexpr bool kWholeOrCol = COL || GL == 0;  // GL == 0 only for whole limbs
    static_assert(TOTAL <= 4096, "32 KB of shared memory per CTA");
    __device__ static __forceinline__ uint32_t si(uint32_t g, uint32_t u) {
        return COL ? (u << GL) + g : (g << K) + (u ^ ((u >> 4) & 15u));
    }
    // global word offset (within the limb) of local word u of sub-transform c
    __device__ static __forceinline__ uint32_t off(int n, uint32_t c, uint32_t u) {
        return COL ? c + (u << (n - K)) : (c << K) + u;
    }
};

// One register pass over local bits [BMIN, BMIN + RP) of every sub-transform
// the CTA holds: a thread takes 2^RP words whose local indices differ only in
// those bits, runs the RP stages on them in registers (forward: from the
// highest bit down; inverse: from the lowest up) and writes them back.
template <class Gm, int RP, int BMIN, bool Fwd>
__device__ __forceinline__ void u64_pass(int n, unsigned long long* s, uint32_t c0,
                                         const TwPair64* tw, uint64_t q) {
    constexpr int W = 1 << RP;
    constexpr uint32_t rest = Gm::KW >> RP;  // local indices per group outside the pass's bits
    constexpr uint32_t groups = Gm::G * rest;
    const uint64_t q2 = 2 * q;
#pragma unroll 1
    for (uint32_t grp = threadIdx.x; grp < groups; grp += kU64Threads) {
        // consecutive threads: consecutive shared-memory words where possible
        const uint32_t g = Gm::COL ? grp % Gm::G : grp / rest;
        const uint32_t ur = Gm::COL ? grp / Gm::G : grp % rest;
        const uint32_t ubase = ((ur >> BMIN) << (BMIN + RP)) | (ur & ((1u << BMIN) - 1u));
        uint64_t v[W];
#pragma unroll
        for (int j = 0; j < W; ++j) v[j] = s[Gm::si(g, ubase | ((uint32_t)j << BMIN))];
#pragma unroll
        for (int t = 0; t < RP; ++t) {
            const int rb = Fwd ? RP - 1 - t : t;  // pass bit of this stage
            const int b = BMIN + rb;              // local bit
            // global stage: compile-time for the columns and for whole limbs
            // (K = logN); row launches (logN >= 13) never hold stage 0
            const int sg = Gm::kWholeOrCol ? Gm::K - 1 - b : n - 1 - b;
            // the pair (j, j | 2^rb) sits at global distance 2^(n-1-sg), so its
            // twiddle depends only on the pass bits above rb: block h of
            // 2^rb pairs shares one, fetched with one 16-byte load just
            // before its pairs (one live twiddle at a time)
#pragma unroll
            for (int h = 0; h < (W >> (rb + 1)); ++h) {
                TwPair64 wh{0, 0};
                if (!Gm::kWholeOrCol || sg != 0) {
                    const uint32_t gi =
                        Gm::off(n, c0 + g, ubase | ((uint32_t)(h << (rb + 1)) << BMIN));
                    const ulonglong2 p = __ldg(
                        reinterpret_cast<const ulonglong2*>(tw + (1u << sg) + (gi >> (n - sg))));
                    wh = TwPair64{p.x, p.y};
                }
#pragma unroll
                for (int lo = 0; lo < (1 << rb); ++lo) {
                    const int j = (h << (rb + 1)) | lo;
                    uint64_t X = v[j], Y = v[j | (1 << rb)];
                    if (Gm::kWholeOrCol && sg == 0) {
                        const TwPair64 f = tw[0], fw = tw[1];
                        if (Fwd) {
                            const uint64_t A = shoup64(X, f, q), T = shoup64(Y, fw, q);
                            X = A + T;
                            Y = A - T + q2;
                        } else {
                            const uint64_t S = X + Y, D = X - Y + q2;
                            X = csub64(shoup64(S, f, q), q);
                            Y = csub64(shoup64(D, fw, q), q);
                        }
                    } else if (Fwd) {
                        const uint64_t A = csub64(X, q2), T = shoup64(Y, wh, q);
                        X = A + T;
                        Y = A - T + q2;
                    } else {
                        const uint64_t S = X + Y, D = X - Y + q2;
                        X = csub64(S, q2);
                        Y = shoup64(D, wh, q);
                    }
                    v[j] = X;
                    v[j | (1 << rb)] = Y;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < W; ++j) s[Gm::si(g, ubase | ((uint32_t)j << BMIN))] = v[j];
    }
}

// Stages per register pass (8 words per thread at 3).  Measured on B200 at
// 2^16 x 16 limbs x 16 polynomials, forward / inverse per launch pair:
// four-stage passes 0.66 / 0.71 ms (124 registers, 2 CTAs per SM), three-stage
// ones 0.50 / 0.45 ms, 0.435 / 0.453 ms with the 4-CTA launch bound below
// (64 registers), 0.371 / 0.357 ms with the launch shape compile-time,
// 0.336 / 0.331 ms with the row swizzle and the compile-time stage index,
// and 0.331 / 0.326 ms with programmatic dependent launch.
constexpr int kU64PassStages = 3;

// The passes after the first DONE local bits: forward from the highest bit
// down, inverse from the lowest up, kU64PassStages bits at a time, one
// barrier after each.
template <class Gm, bool Fwd, int DONE>
__device__ __forceinline__ void u64_passes(int n, unsigned long long* s, uint32_t c0,
                                           const TwPair64* tw, uint64_t q) {
    if constexpr (DONE < Gm::K) {
        constexpr int RP = Gm::K - DONE < kU64PassStages ? Gm::K - DONE : kU64PassStages;
        constexpr int BMIN = Fwd ? Gm::K - DONE - RP : DONE;
        u64_pass<Gm, RP, BMIN, Fwd>(n, s, c0, tw, q);
        __syncthreads();
        u64_passes<Gm, Fwd, DONE + RP>(n, s, c0, tw, q);
    }
}

// Every local stage of the CTA's sub-transforms (the launches of run64 give
// each CTA whole column or row sub-transforms).  LAST: the launch holds the
// limb's last stages (the forward then stores canonical words).
template <class Gm, bool Fwd, bool LAST>
__global__ void __launch_bounds__(kU64Threads, 4) u64_stage_kernel(U64Args a) {
    pdl_enter();  // launched with programmatic dependent launch (run64)
    extern __shared__ unsigned long long s[];
    const uint32_t group = blockIdx.x % a.groups;
    const uint32_t lp = blockIdx.x / a.groups;  // limb-major: limb * polys + poly
    const uint32_t polys = gridDim.x / (a.groups * a.limbs);
    const uint32_t limb = lp / polys, poly = lp - limb * polys;
    const int n = a.n;
    unsigned long long* x = a.data + poly * a.stride + ((size_t)limb << n);
    const TwPair64* tw = a.tw + ((size_t)limb << n);
    const uint64_t q = a.q[limb], q2 = 2 * q;
    const uint32_t c0 = group << Gm::GL;
    // load: consecutive indices are consecutive words in global memory
    for (uint32_t i = threadIdx.x; i < Gm::TOTAL; i += kU64Threads) {
        const uint32_t g = Gm::COL ? i % Gm::G : i >> Gm::K;
        const uint32_t u = Gm::COL ? i >> Gm::GL : i % Gm::KW;
        s[Gm::si(g, u)] = x[Gm::off(n, c0 + g, u)];
    }
    __syncthreads();
    u64_passes<Gm, Fwd, 0>(n, s, c0, tw, q);
    for (uint32_t i = threadIdx.x; i < Gm::TOTAL; i += kU64Threads) {
        const uint32_t g = Gm::COL ? i % Gm::G : i >> Gm::K;
        const uint32_t u = Gm::COL ? i >> Gm::GL : i % Gm::KW;
        uint64_t v = s[Gm::si(g, u)];
        if (Fwd && LAST) v = csub64(csub64(v, q2), q);  // canonical words
        x[Gm::off(n, c0 + g, u)] = v;
    }
}

using U64Kernel = void (*)(U64Args);

// The compiled launch shapes: logN <= 12, one launch of whole limbs
// (K = logN, one per CTA); logN 13..17, the column stages on K1 = logN / 2
// bits, then the row stages on K2 = logN - K1 bits, 4096 words per CTA.
template <bool Fwd>
U64Kernel u64_whole_kernel(int k) {
    switch (k) {
#define NTTB_U64_WHOLE(K) \
    case K: return u64_stage_kernel<U64Geo<K, 0, false>, Fwd, true>;
        NTTB_U64_WHOLE(1) NTTB_U64_WHOLE(2) NTTB_U64_WHOLE(3) NTTB_U64_WHOLE(4)
        NTTB_U64_WHOLE(5) NTTB_U64_WHOLE(6) NTTB_U64_WHOLE(7) NTTB_U64_WHOLE(8)
        NTTB_U64_WHOLE(9) NTTB_U64_WHOLE(10) NTTB_U64_WHOLE(11) NTTB_U64_WHOLE(12)
#undef NTTB_U64_WHOLE
    }
    return nullptr;
}
template <bool Fwd>
U64Kernel u64_col_kernel(int k) {  // the first stages: forward launch 1
    switch (k) {
        case 6: return u64_stage_kernel<U64Geo<6, 6, true>, Fwd, !Fwd>;
        case 7: return u64_stage_kernel<U64Geo<7, 5, true>, Fwd, !Fwd>;
        case 8: return u64_stage_kernel<U64Geo<8, 4, true>, Fwd, !Fwd>;
    }
    return nullptr;
}
template <bool Fwd>
U64Kernel u64_row_kernel(int k) {  // the last stages: forward launch 2
    switch (k) {
        case 7: return u64_stage_kernel<U64Geo<7, 5, false>, Fwd, Fwd>;
        case 8: return u64_stage_kernel<U64Geo<8, 4, false>, Fwd, Fwd>;
        case 9: return u64_stage_kernel<U64Geo<9, 3, false>, Fwd, Fwd>;
    }
    return nullptr;
}

}  // namespace

struct ntt64_plan {
    int logN = 0, limbs = 0, device = 0;
    TwPair64* fwd = nullptr;  // [limbs][N] device, then inv, then q
    TwPair64* inv = nullptr;
    unsigned long long* q = nullptr;
    void* block = nullptr;
};

namespace {

ntt_status_t validate64(int logN, ModulusConfig64 m, uint64_t* psi) {
    const uint64_t N = uint64_t{1} << logN, q = m.qi;
    if (q < 3 || (q - 1) % (2 * N) != 0)
        return fail(NTT_ERR_MODULUS, "q must satisfy q == 1 mod 2N (q=%llu, logN=%d)",
                    (unsigned long long)q, logN);
    if (q >> 62) return fail(NTT_ERR_MODULUS_RANGE, "modulus %llu must be below 2^62", (unsigned long long)q);
    if (!is_prime64(q)) return fail(NTT_ERR_MODULUS_RANGE, "modulus %llu is not prime", (unsigned long long)q);
    const uint64_t p = powmod64(m.primitive_root, (q - 1) / (2 * N), q);
    if (powmod64(p, N, q) != q - 1)
        return fail(NTT_ERR_ROOT, "root %llu does not give a primitive 2N-th root mod %llu",
                    (unsigned long long)m.primitive_root, (unsigned long long)q);
    *psi = p;
    return NTT_OK;
}

// Forward and inverse tables of one limb: tw[i] = psi^bitrev(i) with Shoup
// companions; entries 0 and 1 carry R (forward stage 0) and N^{-1} R^{-1}
// (inverse last stage), R = 2^64 mod q.
void limb_tables(int logN, uint64_t q, uint64_t psi, TwPair64* f, TwPair64* iv) {
    const uint32_t N = 1u << logN;
    const uint64_t psi_inv = powmod64(psi, q - 2, q);
    std::vector<uint64_t> pw(N), pwi(N);
    pw[0] = pwi[0] = 1;
    for (uint32_t k = 1; k < N; ++k) {
        pw[k] = mulmod64(pw[k - 1], psi, q);
        pwi[k] = mulmod64(pwi[k - 1], psi_inv, q);
    }
    for (uint32_t i = 0; i < N; ++i) {
        f[i] = pair_of(pw[bitrev(i, logN)], q);
        iv[i] = pair_of(pwi[bitrev(i, logN)], q);
    }
    const uint64_t R = (uint64_t)(((u128)1 << 64) % q);
    const uint64_t c = mulmod64(powmod64(N % q, q - 2, q), powmod64(R, q - 2, q), q);
    f[0] = pair_of(R, q);
    if (N > 1) f[1] = pair_of(mulmod64(pw[bitrev(1, logN)], R, q), q);
    iv[0] = pair_of(c, q);
    if (N > 1) iv[1] = pair_of(mulmod64(pwi[bitrev(1, logN)], c, q), q);
}

ntt_status_t run64(const ntt64_plan* p, uint64_t* a, size_t polys, size_t stride, bool fwd,
                   cudaStream_t s) {
    if (!p || !a) return fail(NTT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (polys == 0) return NTT_OK;
    const int n = p->logN;
    if (stride == 0) stride = (size_t)p->limbs << n;
    if (polys > 1 && stride < ((size_t)p->limbs << n))
        return fail(NTT_ERR_INVALID_ARGUMENT, "poly_stride smaller than limbs * N");
    if (((uintptr_t)a & 15u) || (polys > 1 && (stride & 1u)))
        return fail(NTT_ERR_MISALIGNED, "data must be 16-byte aligned (stride even)");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return cuda_fail(cudaGetLastError(), "cudaGetDevice");
    if (dev != p->device)
        return fail(NTT_ERR_INVALID_ARGUMENT, "plan was created on device %d, current is %d",
                    p->device, dev);
    const U64Args base{(unsigned long long*)a, fwd ? p->fwd : p->inv, p->q,
                       (unsigned long long)stride, (uint32_t)p->limbs, 1, n};
    struct Launch {
        U64Kernel k;
        uint32_t groups, words;  // CTAs per limb, words per CTA
    };
    Launch launches[2];
    int count = 0;
    if (n <= 12) {
        launches[count++] = {fwd ? u64_whole_kernel<true>(n) : u64_whole_kernel<false>(n), 1,
                             1u << n};
    } else {
        const int k1 = n / 2, k2 = n - k1;  // column bits, row bits
        const Launch c{fwd ? u64_col_kernel<true>(k1) : u64_col_kernel<false>(k1),
                       1u << (n - 12), 4096};
        const Launch r{fwd ? u64_row_kernel<true>(k2) : u64_row_kernel<false>(k2),
                       1u << (n - 12), 4096};
        launches[count++] = fwd ? c : r;
        launches[count++] = fwd ? r : c;
    }
    for (int i = 0; i < count; ++i) {
        const Launch& L = launches[i];
        if (!L.k) return fail(NTT_ERR_UNSUPPORTED, "no 64-bit kernel for logN %d", n);
        const size_t blocks = (size_t)L.groups * p->limbs * polys;
        if (blocks > (size_t)INT_MAX) return fail(NTT_ERR_INVALID_ARGUMENT, "too many limbs");
        U64Args args = base;
        args.groups = L.groups;
        // programmatic dependent launch: the row launch (and the next call's
        // first launch) is scheduled while its predecessor drains
        if (cudaError_t e = launch_pdl(L.k, dim3((unsigned)blocks), dim3(kU64Threads),
                                       (size_t)L.words * 8, s, args);
            e != cudaSuccess)
            return cuda_fail(e, "64-bit NTT launch");
    }
    return NTT_OK;
}

}  // namespace

extern "C" {

ntt_status_t ntt64_find_moduli(int logN, int count, uint64_t lower_bound, ModulusConfig64* out) {
    if (logN < NTT64_MIN_LOGN || logN > NTT64_MAX_LOGN)
        return fail(NTT_ERR_UNSUPPORTED, "logN %d outside [%d, %d]", logN, NTT64_MIN_LOGN, NTT64_MAX_LOGN);
    if (count < 0 || (count > 0 && !out)) return fail(NTT_ERR_INVALID_ARGUMENT, "bad output array");
    const uint64_t step = uint64_t{2} << logN;
    uint64_t q = lower_bound <= 1 ? 1 : ((lower_bound - 2) / step + 1) * step + 1;
    for (int found = 0; found < count; q += step) {
        if (q >> 62) return fail(NTT_ERR_MODULUS_RANGE, "no more primes below 2^62");
        if (!is_prime64(q)) continue;
        uint64_t g = 2;
        while (powmod64(g, (q - 1) / 2, q) != q - 1) ++g;
        out[found++] = ModulusConfig64{q, g};
    }
    return NTT_OK;
}

ntt_status_t ntt64_plan_create(int logN, const ModulusConfig64* moduli, int limbs,
                               ntt64_plan_t** out) {
    if (!out) return fail(NTT_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (logN < NTT64_MIN_LOGN || logN > NTT64_MAX_LOGN)
        return fail(NTT_ERR_UNSUPPORTED, "logN %d outside [%d, %d]", logN, NTT64_MIN_LOGN, NTT64_MAX_LOGN);
    if (limbs < 1 || !moduli) return fail(NTT_ERR_INVALID_ARGUMENT, "need at least one modulus");
    const size_t N = size_t{1} << logN;
    std::vector<TwPair64> f(N * limbs), iv(N * limbs);
    std::vector<unsigned long long> q(limbs);
    for (int l = 0; l < limbs; ++l) {
        uint64_t psi = 0;
        if (ntt_status_t st = validate64(logN, moduli[l], &psi)) return st;
        limb_tables(logN, moduli[l].qi, psi, f.data() + l * N, iv.data() + l * N);
        q[l] = moduli[l].qi;
    }
    auto* p = new ntt64_plan;
    p->logN = logN;
    p->limbs = limbs;
    cudaGetDevice(&p->device);
    const size_t tb = N * limbs * sizeof(TwPair64);
    cudaError_t e = cudaMalloc(&p->block, 2 * tb + limbs * 8);
    if (e == cudaSuccess) {
        p->fwd = (TwPair64*)p->block;
        p->inv = (TwPair64*)((char*)p->block + tb);
        p->q = (unsigned long long*)((char*)p->block + 2 * tb);
        e = cudaMemcpy(p->fwd, f.data(), tb, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(p->inv, iv.data(), tb, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(p->q, q.data(), limbs * 8, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        if (p->block) cudaFree(p->block);
        delete p;
        return cuda_fail(e, "64-bit plan tables");
    }
    *out = p;
    return NTT_OK;
}

ntt_status_t ntt64_plan_destroy(ntt64_plan_t* p) {
    if (!p) return NTT_OK;
    if (p->block) cudaFree(p->block);
    delete p;
    return NTT_OK;
}

ntt_status_t ntt64_forward_many(const ntt64_plan_t* p, uint64_t* a, size_t polys, size_t stride,
                                ntt_stream_t s) {
    return run64(p, a, polys, stride, true, (cudaStream_t)s);
}

ntt_status_t ntt64_inverse_many(const ntt64_plan_t* p, uint64_t* a, size_t polys, size_t stride,
                                ntt_stream_t s) {
    return run64(p, a, polys, stride, false, (cudaStream_t)s);
}

}  // extern "C"
