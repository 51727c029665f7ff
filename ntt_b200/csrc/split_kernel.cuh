// Split transform kernels (sm_100a): the limb's two phases exchange through
// L2 instead of distributed shared memory.
//
// Same math and the same twiddle tables as the cluster kernels
// (fused_kernel.cuh; reference: NTTPhase1/NTTPhase2, INTTPhase1/INTTPhase2,
// src/v04_montgomery.cu:196-565).  The limb of N = 2^n words is a
// 2^R1 x 2^R2 matrix, R1 = EB:
//  * phase 1 (forward stages 0..R1-1, on the row bits): each thread owns one
//    column, loads its 2^EB words straight from global memory (the 32 lanes
//    of a warp read 32 consecutive columns: one 128-byte line per
//    instruction), runs every phase-1 stage in registers and stores the
//    column back in place.  No shared memory and no barrier;
//  * one cluster barrier (release / acquire) makes the limb's phase-1 words
//    visible to the CTAs of the limb;
//  * phase 2 (stages R1..n-1, on the column bits): CTA r owns the
//    contiguous rows [r*M, (r+1)*M); its first register pass reads them from
//    L2 (loads that bypass L1: this SM may hold stale lines of them), the
//    other passes exchange through the work buffer, and the last one leaves
//    the canonical words in the work buffer for the coalesced warp-chunk
//    store (slab_out).
// The inverse runs the same steps backwards (Gentleman-Sande, the N^{-1}
// and Montgomery->normal factors folded into the last stage).
//
// Why: on B200 a distributed-shared-memory scatter moves 11-15 bytes per SM
// cycle against ~80 for local shared memory, and ~88% of every limb crossed
// it; the phase-1 words written back in place stay in the 126 MB L2 (the
// limbs in flight hold ~22 MB) and are overwritten by the phase-2 output
// before they are evicted, so HBM traffic stays one read and one write.
#pragma once
#include <type_traits>

#include "fused_kernel.cuh"
#include "split_geo.cuh"

namespace nttb {

template <bool WarpLocal>
__device__ __forceinline__ void split_sync() {
    if constexpr (WarpLocal) __syncwarp();
    else __syncthreads();
}

// The cluster kernels' device context, with global loads that either stream
// (phase-1 input, read once) or bypass L1 (words other CTAs of the cluster
// rewrote after this SM may have cached their lines).
template <int C, int Out = kOutPlain, bool Comp = false>
struct SplitCtx : DevCtx<C, false, 1, false, Out> {
    static constexpr bool kCompTw = Comp;  // compressed twiddle tables (arith.cuh)
    bool cg = false;
    const uint32_t* sb_final = nullptr;  // Out: the second operand, armed for the last store
    __device__ __forceinline__ uint32_t g_ld(const uint32_t* b, uint32_t c) const {
        return cg ? __ldcg(b + c) : __ldca(b + c);
    }
    __device__ __forceinline__ void g_ld4(const uint32_t* b, uint32_t c, uint32_t& x, uint32_t& y,
                                          uint32_t& z, uint32_t& w) const {
        const uint4* p = reinterpret_cast<const uint4*>(b + c);
        const uint4 t = cg ? __ldcg(p) : __ldca(p);
        x = t.x;
        y = t.y;
        z = t.z;
        w = t.w;
    }
};

// The limb's phase-1 words are in place: make them visible to its CTAs.
__device__ __forceinline__ void split_exchange() {
    cluster_arrive_release();
    cluster_wait_acquire();
}

// Where a split launch lets the next launch in its stream be scheduled
// (programmatic dependent launch): at its start up to logN 16, after the
// phase exchange at logN 17.  Measured on B200, one polynomial of 16 limbs
// per call, forward + inverse: at 2^16 17.7 us at the start against 19.6 us
// after the exchange (2^16 x 32 limbs 24.5 against 27.5 us), at 2^17 35.2 us
// without the attribute against 31.3 us after the exchange (39-40 us at the
// start: waiting CTAs of the next launch sit beside the whole 17-us grid).
template <class G>
constexpr bool kSplitLateTrigger = G::LOGN >= 17;

template <class G, class Arith, class Ctx>
__device__ __forceinline__ void split_forward_body(Ctx& ctx) {
    using F = SplitFwd<G, Arith, Ctx>;
    const uint32_t tid = threadIdx.x;
    F::p1(ctx, tid);
    split_exchange();
    if constexpr (kSplitLateTrigger<G>) pdl_trigger();
    ctx.cg = true;
    F::p2a(ctx, tid);
    split_sync<G::kABWarp>();
    F::p2b(ctx, tid);
    if constexpr (G::K2C > 0) {
        split_sync<G::kBCWarp>();
        F::p2c(ctx, tid);
    }
    split_sync<G::kChunkWarp>();  // the warp's chunk holds the words it wrote
    if constexpr (Ctx::kSub) ctx.sb[0] = ctx.sb_final;  // phase 1 stored plain words
    F::out(ctx, tid);
}

template <class G, class Arith, class Ctx>
__device__ __forceinline__ void split_inverse_body(Ctx& ctx) {
    using I = SplitInv<G, Arith, Ctx>;
    const uint32_t tid = threadIdx.x;
    I::in(ctx, tid);
    split_sync<G::kChunkWarp>();
    if constexpr (G::K2C > 0) {
        I::p2c(ctx, tid);
        split_sync<G::kBCWarp>();
    }
    I::p2b(ctx, tid);
    split_sync<G::kABWarp>();
    I::p2a(ctx, tid);
    split_exchange();
    if constexpr (kSplitLateTrigger<G>) pdl_trigger();
    ctx.cg = true;
    I::p1(ctx, tid);
}

// One launch over the limb transforms of a plan (FusedArgs; one polynomial
// per job): cluster c runs job c.  The launcher always gives one job per
// cluster (the hardware schedules the clusters); a loop over several jobs
// made the compiler keep per-thread addresses live across jobs and spill.
// Out (forward only): the final store's output mode (kOutSubScale: the
// subtract-and-scale output of FusedArgs; kOutMulSpec: the product with a
// resident spectrum).  Comp: compressed twiddle tables (tw_comp_entries
// pairs per limb; the last four stages multiply by two factors).
template <class G, bool Fwd, class Arith, int Out = kOutPlain, bool Comp = false>
__global__ void __launch_bounds__(G::THREADS, G::MIN_BLOCKS) split_kernel(FusedArgs a) {
    static_assert(Out == kOutPlain || Fwd, "the output modes follow a forward");
    static_assert(!Comp || G::LOGN >= kTwCompMinLogN, "compressed tables start at logN 15");
    constexpr uint32_t kTwStride = Comp ? tw_comp_entries(G::LOGN) : (1u << G::LOGN);
    pdl_wait();
    if constexpr (!kSplitLateTrigger<G>) pdl_trigger();
    extern __shared__ __align__(16) uint32_t smem[];
    const uint32_t rank = cluster_rank();
    const uint32_t cluster = blockIdx.x / G::C;
    const uint32_t j0 = cluster * a.jobs_per_cluster;
    const uint32_t j1 = min(j0 + a.jobs_per_cluster, a.jobs);
    SplitCtx<G::C, Out, Comp> ctx;
    ctx.smem = smem;
    ctx.stage = nullptr;
    ctx.smem_sa = (uint32_t)__cvta_generic_to_shared(smem);
    ctx.rank = rank;
    if (j1 > j0) {  // one job per cluster
        const uint32_t job = j0;
        const uint32_t jl = job / a.polys, poly = job - jl * a.polys;
        const uint32_t limb = map_limb(a, jl);
        ctx.o[0] = a.data + (size_t)poly * a.poly_stride + ((size_t)limb << G::LOGN);
        ctx.g[0] = ctx.o[0];
        ctx.twp = a.tw + (size_t)limb * kTwStride;
        ctx.q = __ldg(a.q + limb);
        ctx.q2 = 2u * ctx.q;
        ctx.scale_c = a.scale ? __ldg(a.scale + limb) % ctx.q : kNoScale;
        ctx.cg = false;
        if constexpr (Out == kOutSubScale) {
            const SubJob sj = sub_job<G::LOGN>(a, limb, poly, ctx.q);
            ctx.sb[0] = nullptr;
            ctx.sb_final = sj.base;
            ctx.sub_e = sj.e;
        } else if constexpr (Out == kOutMulSpec) {
            ctx.sb[0] = nullptr;
            ctx.sb_final = a.spec + (size_t)poly * a.spec_stride + ((size_t)limb << G::LOGN);
            ctx.qinv = neg_qinv_dev(ctx.q);
        }
        if constexpr (Fwd) split_forward_body<G, Arith>(ctx);
        else split_inverse_body<G, Arith>(ctx);
    }
}

// ---------------------------------------------------------------------------
// Negacyclic product in one launch: b <- INTT(NTT(a) (.) NTT(b)) per limb of
// each pair (Montgomery-domain pointwise product, as ntt_pointwise_mul).
// a is only read; b's buffer carries both forwards' phase-1 words and the
// inverse's phase-2 words through L2, and NTT(b) waits in a second work
// buffer until NTT(a) reaches it, so HBM sees a read once, b read once and
// written once (12 bytes per coefficient; the unfused calls move 36).
// ---------------------------------------------------------------------------
struct SplitMulArgs {
    uint32_t* b;
    const uint32_t* a;
    const TwPair* tw_fwd;  // [limbs][N] forward / inverse tables
    const TwPair* tw_inv;
    const uint32_t* q;     // [limbs]
    uint32_t limbs, pairs, jobs, jobs_per_cluster;
    unsigned long long b_stride, a_stride;  // words between pairs
};

template <class G>
struct SplitMulGeo {
    static constexpr uint32_t SMEM_BYTES = 2u * G::SLAB_WORDS * 4u;  // work | NTT(b)
    // the two buffers allow 3 CTAs per SM; 32 words per thread fit 85
    // registers, 16 words per thread at 512 threads get 64 (2 CTAs per SM)
    static constexpr int MIN_BLOCKS = G::EB >= 5 ? 3 : 2;
};

// v <- v (.) S over a pass's registers (S in the work-buffer layout).
template <class L, class X, class Ctx>
__device__ __forceinline__ void mul_by_smem(Ctx& ctx, uint32_t (&v)[1][L::E], uint32_t d,
                                            const uint32_t* S, uint32_t qinv) {
    const uint32_t* sb = S + X::phys(d);
    ct_for<L::E>([&](auto R) {
        constexpr int r = decltype(R)::value;
        v[0][r] = mont_mul(v[0][r], sb[X::phys(L::off(r))], ctx.q, qinv);
    });
}

// The forward phase-2 passes before the last one (the first from L2).
template <class G, class Arith, class Ctx>
__device__ __forceinline__ void split_fwd_head(Ctx& ctx, uint32_t tid) {
    using X = typename G::XW;
    using P2A = typename G::P2A;
    using P2B = typename G::P2B;
    {
        uint32_t v[1][P2A::E];
        const uint32_t d = P2A::dep(tid);
        load_global<P2A, (1u << 30), G2Map>(ctx, v, d + ctx.rank * G::M);
        run_stages<G, P2A, Arith, true, true, false>(ctx, v, d);
        store_smem<P2A, X, G::SLAB_WORDS>(ctx, v, d);
    }
    split_sync<G::kABWarp>();
    if constexpr (G::K2C > 0) {
        uint32_t v[1][P2B::E];
        const uint32_t d = P2B::dep(tid);
        load_smem<P2B, X, G::SLAB_WORDS>(ctx, v, d);
        run_stages<G, P2B, Arith, true, true, false>(ctx, v, d);
        store_smem<P2B, X, G::SLAB_WORDS>(ctx, v, d);
        split_sync<G::kBCWarp>();
    }
}

template <class G, class Arith>
__global__ void __launch_bounds__(G::THREADS, SplitMulGeo<G>::MIN_BLOCKS)
    split_mul_kernel(SplitMulArgs a) {
    using Mp = Maps<G>;
    using X = typename G::XW;
    using P1 = typename G::P1;
    using P2A = typename G::P2A;
    using P2B = typename G::P2B;
    using P2C = typename G::P2C;
    using PL = typename G::PLast;
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* W = smem;
    uint32_t* S = smem + G::SLAB_WORDS;
    const uint32_t rank = cluster_rank();
    const uint32_t cluster = blockIdx.x / G::C;
    const uint32_t j0 = cluster * a.jobs_per_cluster;
    const uint32_t j1 = min(j0 + a.jobs_per_cluster, a.jobs);
    const uint32_t tid = threadIdx.x;
    SplitCtx<G::C> ctx;
    ctx.stage = nullptr;
    ctx.smem_sa = (uint32_t)__cvta_generic_to_shared(W);
    ctx.rank = rank;
    // one job per cluster (the launch covers every job): a loop over jobs
    // made the compiler keep every pass's per-thread addresses live across
    // all four transforms and spill
    if (j1 > j0) {
        const uint32_t job = j0;
        const uint32_t limb = job / a.pairs, pair = job - limb * a.pairs;
        uint32_t* bl = a.b + (size_t)pair * a.b_stride + ((size_t)limb << G::LOGN);
        const uint32_t* al = a.a + (size_t)pair * a.a_stride + ((size_t)limb << G::LOGN);
        ctx.q = __ldg(a.q + limb);
        ctx.q2 = 2u * ctx.q;
        ctx.scale_c = kNoScale;
        const uint32_t qinv = neg_qinv_dev(ctx.q);
        ctx.twp = a.tw_fwd + ((size_t)limb << G::LOGN);
        ctx.smem = W;
        // ---- NTT(b): its last pass leaves the spectrum in S
        {
            uint32_t v[1][P1::E];
            const uint32_t d = P1::dep(tid);
            const uint32_t g = Mp::g1(d) + Mp::g1_rank(rank);
            ctx.g[0] = ctx.o[0] = bl;
            ctx.cg = false;
            load_global<P1, G::W1, G1Map<G>>(ctx, v, g);
            run_stages<G, P1, Arith, true, false, true>(ctx, v, d);
            store_global<P1, G::W1, G1Map<G>>(ctx, v, g, Ident{});
        }
        split_exchange();
        ctx.g[0] = bl;
        ctx.cg = true;
        split_fwd_head<G, Arith>(ctx, tid);
        {
            uint32_t v[1][PL::E];
            const uint32_t d = PL::dep(tid);
            load_smem<PL, X, G::SLAB_WORDS>(ctx, v, d);
            run_stages<G, PL, Arith, true, true, false>(ctx, v, d);
            // canonical, so that the product of a lazy word of NTT(a) with it
            // stays below q * 2^32 and REDC returns it canonical
            const FwdFinal<Arith> fin{ctx.q, ctx.q2};
            ct_for<PL::E>([&](auto R) { v[0][decltype(R)::value] = fin(v[0][decltype(R)::value]); });
            ctx.smem = S;
            store_smem<PL, X, G::SLAB_WORDS>(ctx, v, d);
            ctx.smem = W;
        }
        // every CTA has read its rows of b's phase-1 words: b's buffer is free
        cluster_arrive_relaxed();
        // ---- NTT(a): phase 1 from a into b's buffer
        {
            uint32_t v[1][P1::E];
            const uint32_t d = P1::dep(tid);
            const uint32_t g = Mp::g1(d) + Mp::g1_rank(rank);
            ctx.g[0] = const_cast<uint32_t*>(al);
            ctx.o[0] = bl;
            ctx.cg = false;
            load_global<P1, G::W1, G1Map<G>>(ctx, v, g);
            run_stages<G, P1, Arith, true, false, true>(ctx, v, d);
            cluster_wait_acquire();
            store_global<P1, G::W1, G1Map<G>>(ctx, v, g, Ident{});
        }
        split_exchange();
        ctx.g[0] = bl;
        ctx.cg = true;
        split_fwd_head<G, Arith>(ctx, tid);
        // last forward pass of a, the product with NTT(b), the first inverse pass
        {
            uint32_t v[1][PL::E];
            const uint32_t d = PL::dep(tid);
            load_smem<PL, X, G::SLAB_WORDS>(ctx, v, d);
            run_stages<G, PL, Arith, true, true, false>(ctx, v, d);
            mul_by_smem<PL, X>(ctx, v, d, S, qinv);  // canonical products
            ctx.twp = a.tw_inv + ((size_t)limb << G::LOGN);
            run_stages<G, PL, Arith, false, true, false>(ctx, v, d);
            store_smem<PL, X, G::SLAB_WORDS>(ctx, v, d);
        }
        if constexpr (G::K2C > 0) {
            split_sync<G::kBCWarp>();
            uint32_t v[1][P2B::E];
            const uint32_t d = P2B::dep(tid);
            load_smem<P2B, X, G::SLAB_WORDS>(ctx, v, d);
            run_stages<G, P2B, Arith, false, true, false>(ctx, v, d);
            store_smem<P2B, X, G::SLAB_WORDS>(ctx, v, d);
        }
        split_sync<G::kABWarp>();
        {
            uint32_t v[1][P2A::E];
            const uint32_t d = P2A::dep(tid);
            load_smem<P2A, X, G::SLAB_WORDS>(ctx, v, d);
            run_stages<G, P2A, Arith, false, true, false>(ctx, v, d);
            ctx.o[0] = bl;
            store_global<P2A, (1u << 30), G2Map>(ctx, v, d + rank * G::M, Ident{});
        }
        split_exchange();
        // ---- inverse phase 1: canonical product into b
        {
            uint32_t v[1][P1::E];
            const uint32_t d = P1::dep(tid);
            const uint32_t g = Mp::g1(d) + Mp::g1_rank(rank);
            ctx.g[0] = ctx.o[0] = bl;
            ctx.cg = true;
            load_global<P1, G::W1, G1Map<G>>(ctx, v, g);
            run_stages<G, P1, Arith, false, false, true>(ctx, v, d);
            store_global<P1, G::W1, G1Map<G>>(ctx, v, g, Ident{});
        }
    }
}

}  // namespace nttb
