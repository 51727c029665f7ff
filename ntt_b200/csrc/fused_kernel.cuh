// Device context and the fused cluster kernel template (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include "ntt_core.cuh"

namespace nttb {

// Arguments of one launch over `jobs` limb transforms of one plan.
// Job j is limb (j % limbs) of polynomial (j / limbs); polynomial p starts
// at data + p * poly_stride (words), limb l at + l * N.
struct FusedArgs {
    uint32_t* data;
    const TwPair* tw;      // [limbs][N] forward or inverse table (see twiddle.cu)
    const uint32_t* q;     // [limbs]
    uint32_t limbs;
    uint32_t jobs;
    unsigned long long poly_stride;
};

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cluster_arrive_release() {
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait_acquire() {
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <int C>
struct DevCtx {
    uint32_t* __restrict__ g;
    const TwPair* __restrict__ twp;
    uint32_t* smem;
    uint32_t smem_sa;  // .shared window address of smem
    uint32_t q, q2, rank;

    __device__ __forceinline__ uint32_t gload(uint32_t o) const {
        uint32_t v;
        asm volatile("ld.global.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(g + o));
        return v;
    }
    __device__ __forceinline__ void gload4(uint32_t o, uint32_t& a, uint32_t& b, uint32_t& c,
                                           uint32_t& d) const {
        asm volatile("ld.global.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
                     : "=r"(a), "=r"(b), "=r"(c), "=r"(d)
                     : "l"(g + o));
    }
    __device__ __forceinline__ void gstore(uint32_t o, uint32_t v) const { g[o] = v; }
    __device__ __forceinline__ void gstore4(uint32_t o, uint32_t a, uint32_t b, uint32_t c,
                                            uint32_t d) const {
        *reinterpret_cast<uint4*>(g + o) = make_uint4(a, b, c, d);
    }
    __device__ __forceinline__ uint32_t sload(uint32_t w) const { return smem[w]; }
    __device__ __forceinline__ void sstore(uint32_t w, uint32_t v) const { smem[w] = v; }
    __device__ __forceinline__ void rstore(uint32_t dst, uint32_t w, uint32_t v) const {
        if constexpr (C == 1) {
            smem[w] = v;
        } else {
            uint32_t ra;
            asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(smem_sa), "r"(dst));
            asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(ra + 4u * w), "r"(v)
                         : "memory");
        }
    }
    __device__ __forceinline__ TwPair tw(uint32_t i) const {
        uint2 t = __ldg(reinterpret_cast<const uint2*>(twp) + i);
        return TwPair{t.x, t.y};
    }
    __device__ __forceinline__ void after_local_reads() const {
        if constexpr (C > 1) cluster_arrive_release();
    }
    __device__ __forceinline__ void before_scatter() const {
        if constexpr (C > 1) cluster_wait_acquire();
    }
};

template <class G>
__device__ __forceinline__ void cta_or_cluster_sync() {
    if constexpr (G::C > 1) {
        cluster_arrive_release();
        cluster_wait_acquire();
    } else {
        __syncthreads();
    }
}

template <class G, class Arith>
__device__ __forceinline__ void fused_forward_body(DevCtx<G::C>& ctx) {
    using F = Forward<G, Arith, DevCtx<G::C>>;
    const uint32_t tid = threadIdx.x;
    F::pass1a(ctx, tid);
    if constexpr (G::K1B > 0) {
        __syncthreads();
        F::pass1b(ctx, tid);
    }
    cta_or_cluster_sync<G>();
    F::pass2a(ctx, tid);
    if constexpr (G::K2B > 0) {
        __syncthreads();
        F::pass2b(ctx, tid);
    }
}

template <class G, class Arith>
__device__ __forceinline__ void fused_inverse_body(DevCtx<G::C>& ctx) {
    using I = Inverse<G, Arith, DevCtx<G::C>>;
    const uint32_t tid = threadIdx.x;
    if constexpr (G::K2B > 0) {
        I::pass2b(ctx, tid);
        __syncthreads();
    }
    I::pass2a(ctx, tid);
    cta_or_cluster_sync<G>();
    if constexpr (G::K1B > 0) {
        I::pass1b(ctx, tid);
        __syncthreads();
    }
    I::pass1a(ctx, tid);
}

// One cluster of G::C CTAs per limb transform; grid.x = C * jobs.
template <class G, bool Fwd>
__global__ void __launch_bounds__(G::THREADS) fused_kernel(FusedArgs a) {
    extern __shared__ __align__(16) uint32_t smem[];
    const uint32_t rank = (G::C > 1) ? cluster_rank() : 0u;
    const uint32_t job = blockIdx.x / G::C;
    const uint32_t limb = job % a.limbs;
    const uint32_t poly = job / a.limbs;
    DevCtx<G::C> ctx;
    ctx.g = a.data + (size_t)poly * a.poly_stride + ((size_t)limb << G::LOGN);
    ctx.twp = a.tw + ((size_t)limb << G::LOGN);
    ctx.smem = smem;
    ctx.smem_sa = (uint32_t)__cvta_generic_to_shared(smem);
    ctx.q = __ldg(a.q + limb);
    ctx.q2 = 2u * ctx.q;
    ctx.rank = rank;
    if (ctx.q < (1u << 30)) {
        if constexpr (Fwd) fused_forward_body<G, Lazy4>(ctx);
        else fused_inverse_body<G, Lazy4>(ctx);
    } else {
        if constexpr (Fwd) fused_forward_body<G, Lazy2>(ctx);
        else fused_inverse_body<G, Lazy2>(ctx);
    }
}

}  // namespace nttb
