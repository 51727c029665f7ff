// Transforms of small limbs (N <= 2^9): one CTA per limb, one shared-memory
// round per radix-2 stage.  Same table layout, folds and lazy arithmetic as
// the fused kernels; these sizes are latency-bound, not throughput-bound.
#include <cuda_runtime.h>
#include <cstdint>
#include "arith.cuh"
#include "small.h"

namespace nttb {

// Table entry t times c (normal domain) with its Shoup companion.
__device__ __forceinline__ TwPair small_scaled(TwPair t, uint32_t c, uint32_t q) {
    const uint32_t w = (uint32_t)(((unsigned long long)t.w * c) % q);
    return TwPair{w, (uint32_t)(((unsigned long long)w << 32) / q)};
}

// f0, f1: table entries 0 and 1 (the constants folded into stage 0), already
// scaled by the launch's limb constant if it carries one.
// sb (forward): the limb's subtrahend (nullptr: none), e its constant.
template <class Arith, bool Fwd>
__device__ void small_body(uint32_t* a, const TwPair* tw, uint32_t q, int logN, uint32_t* s,
                           TwPair f0, TwPair f1, const uint32_t* sb, TwPair e) {
    const uint32_t N = 1u << logN, half = N >> 1, q2 = 2u * q;
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) s[i] = a[i];
    __syncthreads();
    for (int st = 0; st < logN; ++st) {
        // forward: stage st (t = N >> (st+1)); inverse: stage logN-1-st
        const int sg = Fwd ? st : (logN - 1 - st);
        const uint32_t t = N >> (sg + 1);
        for (uint32_t b = threadIdx.x; b < half; b += blockDim.x) {
            const uint32_t j = b / t, k = j * 2 * t + (b % t);
            uint32_t x = s[k], y = s[k + t];
            if (Fwd) {
                if (sg == 0) Arith::ct_first(x, y, f0, f1, q, q2);
                else {
                    const TwPair w = tw[(1u << sg) + j];
                    Arith::ct(x, y, w.w, w.wp, q, q2);
                }
            } else {
                if (sg == 0) Arith::gs_last(x, y, f0, f1, q, q2);
                else {
                    const TwPair w = tw[(1u << sg) + j];
                    Arith::gs(x, y, w.w, w.wp, q, q2);
                }
            }
            s[k] = x;
            s[k + t] = y;
        }
        __syncthreads();
    }
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
        if (Fwd) {
            const uint32_t y = Arith::fwd_final(s[i], q, q2);
            a[i] = sb ? sub_scaled(y, sb[i], e, q) : y;
        } else {
            a[i] = s[i];
        }
    }
}

template <bool Fwd>
__global__ void small_kernel(SmallArgs p) {
    __shared__ uint32_t s[1u << kSmallMaxLogN];
    const uint32_t job = blockIdx.x;
    const uint32_t jl = job % p.limbs, poly = job / p.limbs;
    const uint32_t limb = jl >= p.skip_at ? jl + p.skip_len : jl;
    uint32_t* a = p.data + (size_t)poly * p.poly_stride + ((size_t)limb << p.logN);
    const TwPair* tw = p.tw + ((size_t)limb << p.logN);
    const uint32_t q = p.q[limb];
    TwPair f0 = tw[0], f1 = tw[1];
    if (p.scale) {
        const uint32_t c = p.scale[limb] % q;
        f0 = small_scaled(f0, c, q);
        f1 = small_scaled(f1, c, q);
    }
    const uint32_t* sb = nullptr;
    TwPair e{0u, 0u};
    if (Fwd && p.sub && limb >= p.sub_begin && limb < p.sub_end) {
        const uint32_t k = limb - p.sub_begin;
        unsigned long long c = p.scale ? p.scale[limb] % q : 1ull;
        if (p.sub_mul) c = c * (p.sub_mul[k] % q) % q;
        e = TwPair{(uint32_t)c, (uint32_t)((c << 32) / q)};
        sb = p.sub + (size_t)poly * p.sub_stride + ((size_t)k << p.logN);
    }
    if (q < (1u << 30)) small_body<Lazy4, Fwd>(a, tw, q, p.logN, s, f0, f1, sb, e);
    else small_body<Lazy2, Fwd>(a, tw, q, p.logN, s, f0, f1, sb, e);
}

cudaError_t launch_small(const SmallArgs& a, bool fwd, cudaStream_t s) {
    if (a.logN < 1 || a.logN > kSmallMaxLogN) return cudaErrorInvalidValue;
    if (a.jobs == 0) return cudaSuccess;
    const uint32_t half = 1u << (a.logN - 1);
    dim3 block(half < 32 ? 32 : half), grid(a.jobs);
    // a plain launch: with programmatic dependent launch (waiting at the
    // start, the trigger at the start or at the end) a batch of 2048 x 16
    // limbs at logN 2 / 4 took 69-73 us per forward + inverse against 41-44
    // us without it on B200, for 9.2 against 10.2 us on one-polynomial calls
    if (fwd) small_kernel<true><<<grid, block, 0, s>>>(a);
    else small_kernel<false><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace nttb
