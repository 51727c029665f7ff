// Warp-per-limb transforms of small limbs (2^6 <= N <= 2^9, sm_100a).
//
// One warp holds a whole limb in registers: lane l owns words l, l + 32,
// l + 64, ... (E = N / 32 of them), so every load and store instruction of
// the warp moves one 128-byte line.  A stage whose butterfly distance d is
// at least 32 words pairs two registers of the same lane (register distance
// d / 32); the last five stages (d = 16, 8, 4, 2, 1) pair lane l with lane
// l ^ d in the same register and exchange the words with one shfl.xor per
// register.  Both lanes of such a pair then run the complete butterfly on
// (their word, the partner's word) in the right order and keep their half,
// so the lazy ranges are exactly those of a register butterfly (Arith::ct /
// Arith::gs) and the results are those of every other kernel.  No shared
// memory, no CTA barrier: the single-CTA kernel of small.cu spends one
// shared-memory round trip and one barrier per stage.
//
// Same table layout and folds as the other kernels (logN < 10: natural
// order; entries 0 and 1 carry the stage-0 constants), the same optional
// per-limb scale, limb map and subtract-and-scale output (SmallArgs).
// Reference: the per-stage butterfly loops of NTTPhase1/2 and
// INTTPhase1/2, src/v04_montgomery.cu:196-565.
#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>
#include <utility>

#include "arith.cuh"
#include "pdl.cuh"
#include "small.h"

namespace nttb {

namespace {

constexpr int kWarpsPerBlock = 8;

// f(integral_constant<int, i>) for i = 0 .. N-1 (stage loops with
// compile-time stage numbers).
template <class F, int... Is>
__device__ __forceinline__ void ct_for_w_impl(F&& f, std::integer_sequence<int, Is...>) {
    (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void ct_for_w(F&& f) {
    ct_for_w_impl(f, std::make_integer_sequence<int, N>{});
}

__device__ __forceinline__ TwPair warp_scaled(TwPair t, uint32_t c, uint32_t q) {
    const uint32_t w = (uint32_t)(((unsigned long long)t.w * c) % q);
    return TwPair{w, (uint32_t)(((unsigned long long)w << 32) / q)};
}

template <int LOGN, class Arith, bool Fwd>
__device__ __forceinline__ void warp_body(uint32_t* a, const TwPair* __restrict__ tw, uint32_t q,
                                          TwPair f0, TwPair f1, const uint32_t* sb, TwPair e) {
    constexpr int E = (1 << LOGN) / 32;
    const uint32_t lane = threadIdx.x & 31u, q2 = 2u * q;
    uint32_t v[E];
#pragma unroll
    for (int r = 0; r < E; ++r) v[r] = a[r * 32 + lane];

    // stage s: butterfly distance d = N >> (s + 1), block j of the lower word
    // i uses twiddle 2^s + i / (2d)
    auto reg_stage = [&](auto S) {
        constexpr int s = decltype(S)::value;
        constexpr int d = (1 << LOGN) >> (s + 1);
        constexpr int dr = d / 32;
#pragma unroll
        for (int r = 0; r < E; ++r) {
            if ((r & dr) != 0) continue;  // r is the lower register of its pair
            if constexpr (s == 0) {
                if constexpr (Fwd) Arith::ct_first(v[r], v[r + dr], f0, f1, q, q2);
                else Arith::gs_last(v[r], v[r + dr], f0, f1, q, q2);
            } else {
                const TwPair w = tw[(1u << s) + (uint32_t)(r * 32) / (2u * d)];  // same for all lanes
                if constexpr (Fwd) Arith::ct(v[r], v[r + dr], w.w, w.wp, q, q2);
                else Arith::gs(v[r], v[r + dr], w.w, w.wp, q, q2);
            }
        }
    };
    auto lane_stage = [&](auto S) {
        constexpr int s = decltype(S)::value;
        constexpr int d = (1 << LOGN) >> (s + 1);
        const bool upper = (lane & (uint32_t)d) != 0;
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const TwPair w = tw[(1u << s) + (uint32_t)(r * 32 + lane) / (2u * d)];
            const uint32_t other = __shfl_xor_sync(0xFFFFFFFFu, v[r], d);
            uint32_t x = upper ? other : v[r], y = upper ? v[r] : other;
            if constexpr (Fwd) Arith::ct(x, y, w.w, w.wp, q, q2);
            else Arith::gs(x, y, w.w, w.wp, q, q2);
            v[r] = upper ? y : x;
        }
    };
    if constexpr (Fwd) {
        ct_for_w<LOGN - 5>([&](auto S) { reg_stage(S); });
        ct_for_w<5>([&](auto K) { lane_stage(std::integral_constant<int, LOGN - 5 + decltype(K)::value>{}); });
    } else {
        ct_for_w<5>([&](auto K) { lane_stage(std::integral_constant<int, LOGN - 1 - decltype(K)::value>{}); });
        ct_for_w<LOGN - 5>([&](auto K) { reg_stage(std::integral_constant<int, LOGN - 6 - decltype(K)::value>{}); });
    }
#pragma unroll
    for (int r = 0; r < E; ++r) {
        uint32_t y = v[r];
        if constexpr (Fwd) {
            y = Arith::fwd_final(y, q, q2);
            if (sb) y = sub_scaled(y, sb[r * 32 + lane], e, q);
        }
        a[r * 32 + lane] = y;
    }
}

template <int LOGN, bool Fwd>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) warp_kernel(SmallArgs p) {
    pdl_enter();  // launched with programmatic dependent launch (launch_warp_n)
    const uint32_t job = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    if (job >= p.jobs) return;  // uniform per warp: the shuffles see all 32 lanes
    const uint32_t jl = job % p.limbs, poly = job / p.limbs;
    const uint32_t limb = jl >= p.skip_at ? jl + p.skip_len : jl;
    uint32_t* a = p.data + (size_t)poly * p.poly_stride + ((size_t)limb << LOGN);
    const TwPair* tw = p.tw + ((size_t)limb << LOGN);
    const uint32_t q = p.q[limb];
    TwPair f0 = tw[0], f1 = tw[1];
    if (p.scale) {
        const uint32_t c = p.scale[limb] % q;
        f0 = warp_scaled(f0, c, q);
        f1 = warp_scaled(f1, c, q);
    }
    const uint32_t* sb = nullptr;
    TwPair e{0u, 0u};
    if (Fwd && p.sub && limb >= p.sub_begin && limb < p.sub_end) {
        const uint32_t k = limb - p.sub_begin;
        unsigned long long c = p.scale ? p.scale[limb] % q : 1ull;
        if (p.sub_mul) c = c * (p.sub_mul[k] % q) % q;
        e = TwPair{(uint32_t)c, (uint32_t)((c << 32) / q)};
        sb = p.sub + (size_t)poly * p.sub_stride + ((size_t)k << LOGN);
    }
    if (q < (1u << 30)) warp_body<LOGN, Lazy4, Fwd>(a, tw, q, f0, f1, sb, e);
    else warp_body<LOGN, Lazy2, Fwd>(a, tw, q, f0, f1, sb, e);
}

template <int LOGN>
cudaError_t launch_warp_n(const SmallArgs& a, bool fwd, cudaStream_t s) {
    const dim3 block(32 * kWarpsPerBlock), grid((a.jobs + kWarpsPerBlock - 1) / kWarpsPerBlock);
    return fwd ? launch_pdl(warp_kernel<LOGN, true>, grid, block, 0, s, a)
               : launch_pdl(warp_kernel<LOGN, false>, grid, block, 0, s, a);
}

}  // namespace

cudaError_t launch_warp(const SmallArgs& a, bool fwd, cudaStream_t s) {
    if (a.jobs == 0) return cudaSuccess;
    switch (a.logN) {
        case 6: return launch_warp_n<6>(a, fwd, s);
        case 7: return launch_warp_n<7>(a, fwd, s);
        case 8: return launch_warp_n<8>(a, fwd, s);
        case 9: return launch_warp_n<9>(a, fwd, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace nttb
