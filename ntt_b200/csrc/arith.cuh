// Exact 32-bit modular arithmetic for the NTT kernels (host + device).
//
// The reference (src/v04_montgomery.cu:93-146) keeps every value canonical in
// [0, q) and multiplies with 32-bit Montgomery REDC (4 multiplies + 2
// conditional corrections per product).  On sm_100a the transform is bound by
// integer issue, so the kernels here use Shoup's precomputed-quotient product
// (3 multiplies) with Harvey's lazy reduction ranges instead:
//
//   shoup(a, w, w') = a*w - umulhi(a, w')*q   (mod 2^32),  w' = floor(w*2^32/q)
//   -> a*w mod q  + {0, q}  for any a < 2^32, 0 <= w < q < 2^31.
//
// Two range disciplines ("kinds"), chosen per limb from its modulus:
//   Lazy4 (q < 2^30): CT butterflies keep values in [0, 4q), GS in [0, 2q);
//                     7 integer instructions per butterfly.
//   Lazy2 (q < 2^31): CT in [0, 2q), GS in [0, q); 9 instructions.
// Every transform ends with a canonicalisation to [0, q), so outputs are the
// unique residues and therefore bit-identical to the reference's.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define NTT_HD __host__ __device__ __forceinline__
#else
#define NTT_HD inline
#endif

namespace nttb {

NTT_HD uint32_t mulhi32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

NTT_HD uint32_t umin32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    return min(a, b);
#else
    return a < b ? a : b;
#endif
}

// x in [0, 2m) -> [0, m).  Unsigned wrap makes x - m huge when x < m.
NTT_HD uint32_t csub(uint32_t x, uint32_t m) { return umin32(x, x - m); }

// Shoup product: result congruent to a*w (mod q), in [0, 2q).
NTT_HD uint32_t shoup_mul(uint32_t a, uint32_t w, uint32_t wp, uint32_t q) {
    uint32_t h = mulhi32(a, wp);
    return a * w - h * q;
}

// A twiddle as stored on the device: value and Shoup companion.
struct TwPair {
    uint32_t w;
    uint32_t wp;
};

// ModDown's output word: y - e * s (mod q), canonical; y and s in [0, q),
// e with its Shoup companion.
NTT_HD uint32_t sub_scaled(uint32_t y, uint32_t s, TwPair e, uint32_t q) {
    const uint32_t u = csub(shoup_mul(s, e.w, e.wp, q), q);
    return y - u + (y < u ? q : 0u);
}

// Device twiddle-table layout of one limb (N = 2^logN entries).  In the last
// stages every thread of the transform kernels owns a run of consecutive
// entries (16, 8, 4, 2 of them in the last four stages with the usual 5-word
// runs of a 4-stage register pass), so in the natural order the 32 lanes of a
// warp would read 32 scattered cache lines per load.  The blocks of the last
// four stages are therefore stored interleaved, which makes the lanes' loads
// consecutive: for p = 0..3, stage logN-1-p's block starts at H = N / 2^(p+1)
// and its entry H + j sits at slot
//   H + (j % F) * (N/32) + j / F,   F = 16 / 2^p,
// for logN >= kTwPermMinLogN (the sizes of the cluster and batch kernels,
// whose last four stages are all in their second phase); every other entry,
// and every entry of smaller tables, sits at its index.
constexpr int kTwPermMinLogN = 10;
constexpr int kTwPermStages = 4;
NTT_HD constexpr uint32_t tw_slot(uint32_t i, int logN) {
    if (logN < kTwPermMinLogN) return i;
    const uint32_t s32 = 1u << (logN - 5);
    for (int p = 0; p < kTwPermStages; ++p) {
        const uint32_t h = 1u << (logN - 1 - p);
        if (i >= h) {
            const int lf = 4 - p;  // log2 F
            return h + ((i - h) & ((1u << lf) - 1u)) * s32 + ((i - h) >> lf);
        }
    }
    return i;
}

// Compressed tables (plans created with NTT_PLAN_COMPRESSED_TWIDDLES, logN >=
// kTwCompMinLogN): per limb 3N/16 + 16 pairs instead of N.
//   slots [0, N/16):  entries 0 .. N/16 - 1, as in the full table (stages
//                     0 .. logN-5, folded entries 0 and 1 included);
//   for p = 3, 2, 1, 0, at tw_comp_base(logN, p): the base block of stage
//                     logN-1-p (H = N/2^(p+1), F = 16/2^p), B_p[m] =
//                     tw[H + m F] for m < N/32;
//   at tw_comp_lsb(logN): L[c] = psi^bitrev(c) (inverse psi^-bitrev(c)) for
//                     c < 16, L[0] = 1 (never folded).
// With j = m F + c, c < F, the bits of H + m F and of c are disjoint, so
// bitrev(H + j) = bitrev(H + m F) + bitrev(c) and tw[H + j] = B_p[m] L[c]:
// a butterfly of those stages multiplies by the two factors in turn (two
// Shoup products, one when c = 0).  The base blocks are the c = 0 slots of
// the full table's interleaved blocks, so a warp's loads stay as coalesced;
// the factors L are the same 16 pairs for every thread (broadcast loads).
constexpr int kTwCompMinLogN = 15;
NTT_HD constexpr uint32_t tw_comp_base(int logN, int p) {
    return (1u << (logN - 4)) + (uint32_t)(3 - p) * (1u << (logN - 5));
}
NTT_HD constexpr uint32_t tw_comp_lsb(int logN) { return 3u << (logN - 4); }
NTT_HD constexpr uint32_t tw_comp_entries(int logN) { return tw_comp_lsb(logN) + 16u; }

// ---- butterflies ----------------------------------------------------------

struct Lazy4 {  // q < 2^30
    static constexpr bool kLazy4 = true;
    // Cooley-Tukey: (X, Y) -> (X + wY, X - wY); in/out ranges [0, 4q).
    NTT_HD static void ct(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wp, uint32_t q,
                          uint32_t q2) {
        uint32_t a = csub(x, q2);
        uint32_t t = shoup_mul(y, w, wp, q);
        x = a + t;
        y = a - t + q2;
    }
    // First forward stage with the normal->Montgomery factor R folded in:
    // (X, Y) -> (R X + (wR) Y, R X - (wR) Y); any 32-bit input.
    NTT_HD static void ct_first(uint32_t& x, uint32_t& y, TwPair r, TwPair wr, uint32_t q,
                                uint32_t q2) {
        uint32_t a = shoup_mul(x, r.w, r.wp, q);
        uint32_t t = shoup_mul(y, wr.w, wr.wp, q);
        x = a + t;
        y = a - t + q2;
    }
    // Forward output range [0, 4q) -> canonical.
    NTT_HD static uint32_t fwd_final(uint32_t v, uint32_t q, uint32_t q2) {
        return csub(csub(v, q2), q);
    }
    // Gentleman-Sande: (X, Y) -> (X + Y, (X - Y) w); in/out ranges [0, 2q).
    NTT_HD static void gs(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wp, uint32_t q,
                          uint32_t q2) {
        uint32_t s = x + y;
        uint32_t d = x - y + q2;
        x = csub(s, q2);
        y = shoup_mul(d, w, wp, q);
    }
    // Last inverse stage with c = N^{-1} R^{-1} folded in, canonical output:
    // (X, Y) -> ((X + Y) c, (X - Y) (w c)).
    NTT_HD static void gs_last(uint32_t& x, uint32_t& y, TwPair c, TwPair wc, uint32_t q,
                               uint32_t q2) {
        uint32_t s = x + y;
        uint32_t d = x - y + q2;
        x = csub(shoup_mul(s, c.w, c.wp, q), q);
        y = csub(shoup_mul(d, wc.w, wc.wp, q), q);
    }
    // The same butterflies with the twiddle given as two factors a * b
    // (compressed tables); Shoup products accept any 32-bit input, so the
    // ranges are those of ct / gs.
    NTT_HD static void ct2(uint32_t& x, uint32_t& y, TwPair a, TwPair b, uint32_t q,
                           uint32_t q2) {
        y = shoup_mul(y, b.w, b.wp, q);
        ct(x, y, a.w, a.wp, q, q2);
    }
    NTT_HD static void gs2(uint32_t& x, uint32_t& y, TwPair a, TwPair b, uint32_t q,
                           uint32_t q2) {
        gs(x, y, a.w, a.wp, q, q2);
        y = shoup_mul(y, b.w, b.wp, q);
    }
};

struct Lazy2 {  // q < 2^31
    static constexpr bool kLazy4 = false;
    // ranges [0, 2q)
    NTT_HD static void ct(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wp, uint32_t q,
                          uint32_t) {
        uint32_t a = csub(x, q);
        uint32_t t = csub(shoup_mul(y, w, wp, q), q);
        x = a + t;
        y = a - t + q;
    }
    NTT_HD static void ct_first(uint32_t& x, uint32_t& y, TwPair r, TwPair wr, uint32_t q,
                                uint32_t) {
        uint32_t a = csub(shoup_mul(x, r.w, r.wp, q), q);
        uint32_t t = csub(shoup_mul(y, wr.w, wr.wp, q), q);
        x = a + t;
        y = a - t + q;
    }
    NTT_HD static uint32_t fwd_final(uint32_t v, uint32_t q, uint32_t) { return csub(v, q); }
    // ranges [0, q)
    NTT_HD static void gs(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wp, uint32_t q,
                          uint32_t) {
        uint32_t s = x + y;
        uint32_t d = x - y + q;
        x = csub(s, q);
        y = csub(shoup_mul(d, w, wp, q), q);
    }
    NTT_HD static void gs_last(uint32_t& x, uint32_t& y, TwPair c, TwPair wc, uint32_t q,
                               uint32_t) {
        uint32_t s = x + y;
        uint32_t d = x - y + q;
        x = csub(shoup_mul(s, c.w, c.wp, q), q);
        y = csub(shoup_mul(d, wc.w, wc.wp, q), q);
    }
    NTT_HD static void ct2(uint32_t& x, uint32_t& y, TwPair a, TwPair b, uint32_t q,
                           uint32_t q2) {
        y = shoup_mul(y, b.w, b.wp, q);
        ct(x, y, a.w, a.wp, q, q2);
    }
    NTT_HD static void gs2(uint32_t& x, uint32_t& y, TwPair a, TwPair b, uint32_t q,
                           uint32_t q2) {
        gs(x, y, a.w, a.wp, q, q2);
        y = csub(shoup_mul(y, b.w, b.wp, q), q);
    }
};

// Montgomery product x*y*2^-32 mod q (REDC, as the reference's mont_mul,
// src/v04_montgomery.cu:110-123), for x, y < q < 2^31 and qinv = -q^{-1}
// mod 2^32; canonical output.  Used once per coefficient by the fused
// multiply (pointwise product of two Montgomery-domain spectra).
NTT_HD uint32_t mont_mul(uint32_t x, uint32_t y, uint32_t q, uint32_t qinv) {
    const uint64_t t = (uint64_t)x * y;
    const uint32_t m = (uint32_t)t * qinv;
    const uint32_t u = (uint32_t)((t + (uint64_t)m * q) >> 32);
    return csub(u, q);
}

// ---- host-side helpers for table construction ------------------------------

inline uint32_t shoup_companion(uint32_t w, uint32_t q) {
    return (uint32_t)(((uint64_t)w << 32) / q);
}

}  // namespace nttb
