// Device context and the fused cluster kernel template (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include "ntt_core.cuh"
#include "pdl.cuh"

namespace nttb {

// Arguments of one launch over the limb transforms of `polys` polynomials of
// `limbs` limbs of one plan.  A job is one limb of NP polynomials (the
// kernel's G::NP; the NP transforms share every twiddle load): `jobs` =
// limbs * ceil(polys / NP), numbered limb-major (job j: limb j / groups,
// polynomials NP * (j % groups) + 0..NP-1, groups = ceil(polys / NP)) so that
// consecutive jobs share a modulus and its twiddles.  When NP does not divide
// polys, the last group repeats the last polynomial (the same words computed
// twice and stored twice: every read of a limb precedes the cluster barrier
// that precedes every write of it).  Cluster c runs jobs
// [c * jobs_per_cluster, (c+1) * jobs_per_cluster).
// Polynomial p starts at data + p * poly_stride (words), limb l at + l * N.
// The forward kernel with the product epilogue (Mul) reads its input from
// src (polynomial p at src + p * src_stride) and stores the Montgomery
// product of each output word with the word at the same place of `data`
// (a spectrum) into that place.
struct FusedArgs {
    uint32_t* data;
    const TwPair* tw;   // [limbs][N] forward or inverse table (see twiddle.cu)
    const uint32_t* q;  // [limbs]
    uint32_t limbs;
    uint32_t polys;
    uint32_t jobs;
    uint32_t jobs_per_cluster;
    unsigned long long poly_stride;
    uint32_t* status;  // optional: bit 0 set when a bounded wait expired
    const uint32_t* src;  // Mul only: the forward's input
    unsigned long long src_stride;
    // optional per-limb constants c (normal domain): the forward transforms
    // c * x, the inverse returns c * INTT(x), both folded into stage 0
    const uint32_t* scale;
    // limb map: launch limb l is the table's limb l, or l + skip_len from
    // skip_at on (ModUp's forward leaves the limbs already in the NTT
    // domain alone).  Zero-initialised = the identity.
    uint32_t skip_at, skip_len;
    // subtract-and-scale output (forward kernels with the Sub epilogue):
    // limb l in [sub_begin, sub_end) stores y - e_l * s, s the word at the
    // output's place in sub[poly * sub_stride + (l - sub_begin) * N], e_l =
    // c_l * d_{l - sub_begin} (c = scale or 1, d = sub_mul or 1); the other
    // limbs store y.  y = NTT(c * x), so the limb stores (NTT(x) - d s) c.
    const uint32_t* sub;
    unsigned long long sub_stride;
    uint32_t sub_begin, sub_end;
    const uint32_t* sub_mul;
    // spectrum-product output (split forwards, Out == kOutMulSpec): the
    // final store writes the Montgomery product of y with the word at the
    // same place of spec[poly * spec_stride + limb * N] (another forward's
    // output, read once)
    const uint32_t* spec;
    unsigned long long spec_stride;
};

// Output modes of the transform kernels' final store.
constexpr int kOutPlain = 0;
constexpr int kOutSubScale = 1;  // y - e s (ModDown)
constexpr int kOutMulSpec = 2;   // mont_mul(y, s) (product with a resident spectrum)

__device__ __forceinline__ uint32_t map_limb(const FusedArgs& a, uint32_t l) {
    return l >= a.skip_at ? l + a.skip_len : l;
}

// The job's subtrahend base (nullptr when its limb has none) and constant
// e = c * d with its Shoup companion.
struct SubJob {
    const uint32_t* base;
    TwPair e;
};
template <int LOGN>
__device__ __forceinline__ SubJob sub_job(const FusedArgs& a, uint32_t limb, size_t poly,
                                          uint32_t q) {
    if (limb < a.sub_begin || limb >= a.sub_end) return SubJob{nullptr, TwPair{0u, 0u}};
    const uint32_t k = limb - a.sub_begin;
    unsigned long long e = a.scale ? __ldg(a.scale + limb) % q : 1ull;
    if (a.sub_mul) e = e * (__ldg(a.sub_mul + k) % q) % q;
    return SubJob{a.sub + poly * a.sub_stride + ((size_t)k << LOGN),
                  TwPair{(uint32_t)e, (uint32_t)((e << 32) / q)}};
}

struct SubOut {
    uint32_t* p;
    const uint32_t* s;  // nullptr: plain store
};

// The constant table entry t times c, with its Shoup companion (computed
// once per thread per job: two 64-bit divisions by q).
__device__ __forceinline__ TwPair scaled_pair(TwPair t, uint32_t c, uint32_t q) {
    const uint32_t w = (uint32_t)(((unsigned long long)t.w * c) % q);
    return TwPair{w, (uint32_t)(((unsigned long long)w << 32) / q)};
}
constexpr uint32_t kNoScale = 0xFFFFFFFFu;

// -q^{-1} mod 2^32 by Newton's iteration (q odd: q is its own inverse mod 8).
__device__ __forceinline__ uint32_t neg_qinv_dev(uint32_t q) {
    uint32_t x = q;
#pragma unroll
    for (int i = 0; i < 4; ++i) x *= 2u - q * x;
    return 0u - x;
}

// Output base of the product epilogue: the spectrum it multiplies by sits
// at the same place as the product it stores.  A job slot that repeats the
// last polynomial (NP not dividing polys) stores nothing (live == false): a
// second read-modify-write of the same words would multiply twice.
struct MulOut {
    uint32_t* p;
    bool live;
};

// Hint: fetch [src, src + bytes) from HBM into L2 (no completion tracking).
__device__ __forceinline__ void prefetch_l2(const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// Iteration bound of every mbarrier wait (each try_wait itself blocks for a
// hardware-defined interval); expiry sets the status bit instead of hanging.
constexpr uint32_t kWaitLimit = 1u << 22;
constexpr uint32_t kStatusWaitExpired = 1u;

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cluster_arrive_release() {
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_arrive_relaxed() {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait_acquire() {
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t sa, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sa), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t sa, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sa), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t sa, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(sa), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false when `limit` tries expired.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t sa, uint32_t parity,
                                                  uint32_t limit = kWaitLimit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(sa, parity)) return true;
    return false;
}
// Generic-proxy accesses of shared memory before async-proxy writes to it.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Bulk (non-tensor, non-multicast) copy global -> this CTA's shared memory.
__device__ __forceinline__ void bulk_g2s(uint32_t dst_sa, const void* src, uint32_t bytes,
                                         uint32_t mbar_sa) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
        "[%3];" ::"r"(dst_sa),
        "l"(src), "r"(bytes), "r"(mbar_sa)
        : "memory");
}

// Memory interface used by the pass code (ntt_core.cuh): every access is a
// per-thread base plus a compile-time offset, which the compiler turns into
// an immediate address offset.
// Out (kOut*): the final store's output mode; SubOut carries the word it
// reads (subtrahend or spectrum).
template <int C, bool Staged, int NP, bool Mul = false, int Out = kOutPlain>
struct DevCtx {
    static constexpr bool kStaged = Staged;
    static constexpr bool kSub = Out != kOutPlain;
    uint32_t* g[NP];  // limb base of each polynomial of the job (input)
    uint32_t* o[NP];  // ... output (the input's place, or the spectrum for Mul)
    const uint32_t* sb[NP];  // Out: the subtrahend's / spectrum's limb base (nullptr: none)
    TwPair sub_e;            // kOutSubScale: e and its Shoup companion
    uint32_t qinv;    // Mul: -q^{-1} mod 2^32
    uint32_t live;    // Mul: bit p set when slot p is not a repeated polynomial
    const TwPair* __restrict__ twp;
    uint32_t* smem;
    const uint32_t* stage;  // padded copy of this CTA's input slab (staged)
    uint32_t smem_sa;       // .shared window address of smem
    uint32_t q, q2, rank;
    uint32_t scale_c = kNoScale;  // this job's limb constant (kNoScale: none)

    // global data (direct input): L1-cached, because a thread owning a
    // contiguous run reads each 32-byte sector in two 16-byte halves
    __device__ __forceinline__ uint32_t* g_base(int p, uint32_t o) const { return g[p] + o; }
    __device__ __forceinline__ uint32_t g_ld(const uint32_t* b, uint32_t c) const {
        return __ldca(b + c);
    }
    __device__ __forceinline__ void g_ld4(const uint32_t* b, uint32_t c, uint32_t& x, uint32_t& y,
                                          uint32_t& z, uint32_t& w) const {
        const uint4 t = __ldca(reinterpret_cast<const uint4*>(b + c));
        x = t.x;
        y = t.y;
        z = t.z;
        w = t.w;
    }
    // transform output: in place, or (Mul) the product with the spectrum
    // word at the output's place (written by an earlier launch: read via L2)
    __device__ __forceinline__ auto o_base(int p, uint32_t off) const {
        if constexpr (Mul) return MulOut{o[p] + off, ((live >> p) & 1u) != 0};
        else if constexpr (Out != kOutPlain) return SubOut{o[p] + off, sb[p] ? sb[p] + off : nullptr};
        else return o[p] + off;
    }
    // kOutSubScale: y - e * s; kOutMulSpec: the Montgomery product y * s;
    // s the word at the output's place of the second operand (read once:
    // streamed)
    __device__ __forceinline__ uint32_t out_word(uint32_t v, uint32_t s) const {
        if constexpr (Out == kOutMulSpec) return mont_mul(v, s, q, qinv);
        else return sub_scaled(v, s, sub_e, q);
    }
    __device__ __forceinline__ void o_st(SubOut b, uint32_t c, uint32_t v) const {
        b.p[c] = b.s ? out_word(v, __ldcs(b.s + c)) : v;
    }
    __device__ __forceinline__ void o_st4(SubOut b, uint32_t c, uint32_t x, uint32_t y,
                                          uint32_t z, uint32_t w) const {
        if (b.s) {
            const uint4 k = __ldcs(reinterpret_cast<const uint4*>(b.s + c));
            x = out_word(x, k.x);
            y = out_word(y, k.y);
            z = out_word(z, k.z);
            w = out_word(w, k.w);
        }
        *reinterpret_cast<uint4*>(b.p + c) = make_uint4(x, y, z, w);
    }
    __device__ __forceinline__ void o_st(uint32_t* b, uint32_t c, uint32_t v) const { b[c] = v; }
    __device__ __forceinline__ void o_st4(uint32_t* b, uint32_t c, uint32_t x, uint32_t y,
                                          uint32_t z, uint32_t w) const {
        *reinterpret_cast<uint4*>(b + c) = make_uint4(x, y, z, w);
    }
    __device__ __forceinline__ void o_st(MulOut b, uint32_t c, uint32_t v) const {
        if (!b.live) return;
        b.p[c] = mont_mul(v, __ldcg(b.p + c), q, qinv);
    }
    __device__ __forceinline__ void o_st4(MulOut b, uint32_t c, uint32_t x, uint32_t y,
                                          uint32_t z, uint32_t w) const {
        if (!b.live) return;
        const uint4 k = __ldcg(reinterpret_cast<const uint4*>(b.p + c));
        *reinterpret_cast<uint4*>(b.p + c) =
            make_uint4(mont_mul(x, k.x, q, qinv), mont_mul(y, k.y, q, qinv),
                       mont_mul(z, k.z, q, qinv), mont_mul(w, k.w, q, qinv));
    }
    // stage buffer
    __device__ __forceinline__ const uint32_t* st_base(uint32_t w) const { return stage + w; }
    __device__ __forceinline__ uint32_t st_ld(const uint32_t* b, uint32_t c) const { return b[c]; }
    __device__ __forceinline__ void st_ld4(const uint32_t* b, uint32_t c, uint32_t& x, uint32_t& y,
                                           uint32_t& z, uint32_t& w) const {
        const uint4 t = *reinterpret_cast<const uint4*>(b + c);
        x = t.x;
        y = t.y;
        z = t.z;
        w = t.w;
    }
    // local shared memory (work buffer)
    __device__ __forceinline__ uint32_t* s_base(uint32_t w) const { return smem + w; }
    __device__ __forceinline__ uint32_t s_ld(const uint32_t* b, uint32_t c) const { return b[c]; }
    __device__ __forceinline__ void s_st(uint32_t* b, uint32_t c, uint32_t v) const { b[c] = v; }
    __device__ __forceinline__ void s_ld4(const uint32_t* b, uint32_t c, uint32_t& x, uint32_t& y,
                                          uint32_t& z, uint32_t& w) const {
        const uint4 t = *reinterpret_cast<const uint4*>(b + c);
        x = t.x;
        y = t.y;
        z = t.z;
        w = t.w;
    }
    __device__ __forceinline__ void s_st4(uint32_t* b, uint32_t c, uint32_t x, uint32_t y,
                                          uint32_t z, uint32_t w) const {
        *reinterpret_cast<uint4*>(b + c) = make_uint4(x, y, z, w);
    }
    __device__ __forceinline__ void s_ld2(const uint32_t* b, uint32_t c, uint32_t& x,
                                          uint32_t& y) const {
        const uint2 t = *reinterpret_cast<const uint2*>(b + c);
        x = t.x;
        y = t.y;
    }
    __device__ __forceinline__ void s_st2(uint32_t* b, uint32_t c, uint32_t x, uint32_t y) const {
        *reinterpret_cast<uint2*>(b + c) = make_uint2(x, y);
    }
    // scatter target: the owner CTA's work buffer (DSMEM address when C > 1)
    __device__ __forceinline__ auto r_base(uint32_t dst, uint32_t w) const {
        if constexpr (C == 1) {
            return smem + w;
        } else {
            uint32_t ra;
            asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(smem_sa + 4u * w), "r"(dst));
            return ra;
        }
    }
    template <uint32_t Off, class B>
    __device__ __forceinline__ void r_st(B rb, uint32_t v) const {
        if constexpr (C == 1) {
            rb[Off] = v;
        } else {
            asm volatile("st.shared::cluster.u32 [%0+%2], %1;" ::"r"(rb), "r"(v), "n"(Off * 4u)
                         : "memory");
        }
    }
    // twiddles: re-read by every limb with this modulus (read-only cache)
    __device__ __forceinline__ TwPair tw_at(uint32_t i) const {
        const uint2 t = __ldg(reinterpret_cast<const uint2*>(twp) + i);
        return TwPair{t.x, t.y};
    }
    // table entries 0 and 1 (the constants folded into the limb's stage 0),
    // times the job's limb constant when the launch carries one
    __device__ __forceinline__ TwPair fold_at(uint32_t i) const {
        const TwPair t = tw_at(i);
        return scale_c == kNoScale ? t : scaled_pair(t, scale_c, q);
    }
    __device__ __forceinline__ const TwPair* tw_base(uint32_t i) const { return twp + i; }
    __device__ __forceinline__ TwPair tw_ld(const TwPair* b, uint32_t c) const {
        const uint2 t = __ldg(reinterpret_cast<const uint2*>(b + c));
        return TwPair{t.x, t.y};
    }
    __device__ __forceinline__ void tw_ld2(const TwPair* b, uint32_t c, TwPair& x,
                                           TwPair& y) const {
        const uint4 t = __ldg(reinterpret_cast<const uint4*>(b + c));
        x = TwPair{t.x, t.y};
        y = TwPair{t.z, t.w};
    }
    // Every loaded word has been consumed by register arithmetic when this is
    // called, so a relaxed arrive is enough to order those reads before the
    // peers' scatter into this CTA.
    __device__ __forceinline__ void after_local_reads() const {
        if constexpr (C > 1) cluster_arrive_relaxed();
    }
    __device__ __forceinline__ void before_scatter() const {
        if constexpr (C > 1) cluster_wait_acquire();
    }
    // Phase boundary: after the scatter, every scattered word must be visible
    // to its owner before phase 2 (forward) / phase 1 (inverse) reads it.
    __device__ __forceinline__ void phase_sync() const {
        if constexpr (C > 1) {
            cluster_arrive_release();
            cluster_wait_acquire();
        } else {
            __syncthreads();
        }
    }
};

// Exchange between two register passes of one phase: a warp barrier when
// each warp owns the same elements in both passes.
template <bool WarpLocal>
__device__ __forceinline__ void pass_sync() {
    if constexpr (WarpLocal) __syncwarp();
    else __syncthreads();
}

// Issue the bulk copies of job `job`'s input slab into the stage buffer
// (called by every thread once the whole CTA has read the previous slab).
template <class G, bool Fwd>
__device__ __forceinline__ void issue_slab(const FusedArgs& a, uint32_t job, uint32_t rank,
                                           uint32_t stage_sa, uint32_t mbar_sa) {
    const uint32_t jl = job / a.polys, poly = job - jl * a.polys;
    const uint32_t limb = map_limb(a, jl);
    const uint32_t* src = a.data + (size_t)poly * a.poly_stride + ((size_t)limb << G::LOGN);
    fence_proxy_async_smem();
    if (threadIdx.x == 0) mbar_arrive_expect_tx(mbar_sa, G::M * 4u);
    for (uint32_t i = threadIdx.x; i < slab_copies<G, Fwd>(); i += G::THREADS) {
        const SlabCopy c = slab_copy<G, Fwd>(rank, i);
        bulk_g2s(stage_sa + 4u * c.dst, src + c.src, 4u * c.words, mbar_sa);
    }
}

// One limb transform; `prefetch()` is called once the stage buffer is free.
template <class G, class Arith, class Ctx, class Pre>
__device__ __forceinline__ void fused_forward_body(Ctx& ctx, Pre&& prefetch) {
    using F = Forward<G, Arith, Ctx>;
    const uint32_t tid = threadIdx.x;
    F::pass1a(ctx, tid);
    if constexpr (G::K1B > 0) {
        pass_sync<G::WARP1>();
        F::pass1b(ctx, tid);
    }
    ctx.phase_sync();
    prefetch();  // every warp has read the stage buffer
    F::pass2a(ctx, tid);
    if constexpr (G::K2B > 0) {
        pass_sync<G::WARP2>();
        F::pass2b(ctx, tid);
        pass_sync<G::WARP2>();  // the warp's chunk is the words it wrote
        F::pass2c(ctx, tid);
    }
}

template <class G, class Arith, class Ctx, class Pre>
__device__ __forceinline__ void fused_inverse_body(Ctx& ctx, Pre&& prefetch) {
    using I = Inverse<G, Arith, Ctx>;
    const uint32_t tid = threadIdx.x;
    if constexpr (I::kChunkIn) {
        I::pass2c(ctx, tid);
        pass_sync<G::WARP2>();  // the warp's chunk holds its pass-2b words
    }
    if constexpr (G::K2B > 0) {
        I::pass2b(ctx, tid);
        pass_sync<G::WARP2>();
    }
    I::pass2a(ctx, tid);
    ctx.phase_sync();
    prefetch();  // every warp has read the stage buffer
    if constexpr (G::K1B > 0) {
        I::pass1b(ctx, tid);
        pass_sync<G::WARP1>();
    }
    I::pass1a(ctx, tid);
}

// Each cluster of G::C CTAs runs a contiguous chunk of limb-major jobs
// [j0, j1).  Staged: the CTA's input slab is bulk-copied into the stage
// buffer one job ahead (mbarrier-tracked, bounded waits); otherwise the
// first pass loads straight from global memory.  grid.x = C * clusters.
// Arith: the range discipline of every limb of the launch (Lazy4 needs all
// moduli below 2^30; Lazy2 takes any below 2^31), fixed per kernel so that
// one path's registers fit the launch bounds.
// Mul (forward, direct only): the product epilogue of FusedArgs.
// Sub (forward, direct only): the subtract-and-scale output of FusedArgs.
template <class G, bool Fwd, bool Staged, class Arith, bool Mul = false, bool Sub = false>
__global__ void __launch_bounds__(G::THREADS, G::MIN_BLOCKS) fused_kernel(FusedArgs a) {
    static_assert(!Mul || (Fwd && !Staged), "the product epilogue follows a direct forward");
    static_assert(!Sub || (Fwd && !Staged && !Mul), "the subtract-and-scale output follows a direct forward");
    pdl_enter();
    extern __shared__ __align__(16) uint32_t smem[];
    const uint32_t rank = (G::C > 1) ? cluster_rank() : 0u;
    const uint32_t cluster = blockIdx.x / G::C;
    const uint32_t j0 = cluster * a.jobs_per_cluster;
    const uint32_t j1 = min(j0 + a.jobs_per_cluster, a.jobs);
    const uint32_t smem_sa = (uint32_t)__cvta_generic_to_shared(smem);
    const uint32_t stage_sa = smem_sa + 4u * G::STAGE_OFF_WORDS;
    const uint32_t mbar_sa = smem_sa + 4u * G::MBAR_OFF_WORDS;
    if constexpr (Staged) {
        if (threadIdx.x == 0) {
            mbar_init(mbar_sa, 1);
            fence_mbar_init();
        }
        __syncthreads();
        if (j0 < j1) issue_slab<G, Fwd>(a, j0, rank, stage_sa, mbar_sa);
    }
    static_assert(!Staged || G::NP == 1, "the staged schedule carries one polynomial per job");
    DevCtx<G::C, Staged, G::NP, Mul, Sub ? kOutSubScale : kOutPlain> ctx;
    const uint32_t groups = (a.polys + G::NP - 1) / G::NP;
    ctx.smem = smem;
    ctx.stage = smem + G::STAGE_OFF_WORDS;
    ctx.smem_sa = smem_sa;
    ctx.rank = rank;
    uint32_t parity = 0;
    for (uint32_t job = j0; job < j1; ++job, parity ^= 1u) {
        const uint32_t jl = job / groups, poly0 = (job - jl * groups) * G::NP;
        const uint32_t limb = map_limb(a, jl);
        if constexpr (Mul) ctx.live = 0;
#pragma unroll
        for (int p = 0; p < G::NP; ++p) {
            const size_t poly = min(poly0 + p, a.polys - 1);
            ctx.o[p] = a.data + poly * a.poly_stride + ((size_t)limb << G::LOGN);
            if constexpr (Mul) {
                ctx.g[p] = const_cast<uint32_t*>(a.src) + poly * a.src_stride +
                           ((size_t)limb << G::LOGN);
                if (poly0 + p < a.polys) ctx.live |= 1u << p;
                // the spectrum words this CTA multiplies by at the end (its
                // phase-2 slab): start moving them into L2 now
                if (threadIdx.x == 0) prefetch_l2(ctx.o[p] + rank * G::M, G::M * 4u);
            } else {
                ctx.g[p] = ctx.o[p];
            }
        }
        ctx.twp = a.tw + ((size_t)limb << G::LOGN);
        ctx.q = __ldg(a.q + limb);
        ctx.q2 = 2u * ctx.q;
        if constexpr (Sub) {
#pragma unroll
            for (int p = 0; p < G::NP; ++p) {
                const SubJob sj = sub_job<G::LOGN>(a, limb, min(poly0 + p, a.polys - 1), ctx.q);
                ctx.sb[p] = sj.base;
                ctx.sub_e = sj.e;
            }
        }
        if (a.scale) ctx.scale_c = __ldg(a.scale + limb) % ctx.q;
        if constexpr (Mul) ctx.qinv = neg_qinv_dev(ctx.q);
        if constexpr (Staged) {
            if (!mbar_wait_bounded(mbar_sa, parity) && a.status)
                atomicOr(a.status, kStatusWaitExpired);
        }
        auto prefetch = [&]() {
            if constexpr (Staged)
                if (job + 1 < j1) issue_slab<G, Fwd>(a, job + 1, rank, stage_sa, mbar_sa);
        };
        if constexpr (Fwd) fused_forward_body<G, Arith>(ctx, prefetch);
        else fused_inverse_body<G, Arith>(ctx, prefetch);
        __syncthreads();  // the work buffer is rewritten by the next job
    }
}

}  // namespace nttb
