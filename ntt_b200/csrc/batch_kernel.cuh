// Persistent ragged-batch kernel (sm_100a).
//
// Replaces the reference's one-launch-per-transform host loop
// (launch_ntt<LC> / launch_intt<LC>, src/v04_montgomery.cu:603-658, called
// once per polynomial) with one launch over a ragged set of (polynomial,
// limb) tiles of different sizes, moduli and operations.  Resident clusters
// of CL CTAs repeatedly take the next "group" from a device-side counter; a
// group places tiles in aligned power-of-two CTA ranges of the cluster
// (batch_geo.h), and every tile runs the same fused transform bodies as the
// plain kernel with its own modulus and twiddle tables.
//
// Cluster-barrier protocol: each transform body performs exactly one relaxed
// arrive (after its last local read of phase 1), one wait (before the DSMEM
// scatter) and one release/acquire barrier (after the scatter).  A group's
// CTAs all run the same number of such rounds (the group's `rounds`): a
// multiply tile runs three bodies (two when the operand is already a
// spectrum), a forward/inverse tile one, and any CTA with fewer bodies (or
// no tile) runs empty rounds with the same barriers.
//
// Multiply tiles pass their intermediate spectra through the tile's own
// slab of the output limb in global memory (L2-resident between bodies):
// every geometry gives CTA `rank` the same phase-2 slab and a CTA barrier
// separates the bodies, so shared memory -- hence occupancy -- stays that
// of a plain transform.
// The index of the next group is fetched by CTA 0 during the current group
// and stored into every CTA's slot word before the last round's release
// barrier, so no extra barrier is spent on distributing work.
#pragma once
#include "batch_geo.h"
#include "fused_kernel.cuh"

namespace nttb {

// Geometry of a tile of each logN (and direction); all have 256 threads.
template <int LOGN, bool Fwd>
struct BatchGeo;
template <bool F> struct BatchGeo<17, F> { using G = Geometry<17, 4, 8, 5, 3, 5>; };
template <> struct BatchGeo<16, true> { using G = Geometry<16, 3, 8, 5, 3, 4>; };
template <> struct BatchGeo<16, false> { using G = Geometry<16, 3, 7, 5, 3, 5>; };
template <bool F> struct BatchGeo<15, F> { using G = Geometry<15, 2, 8, 5, 3, 4>; };
template <bool F> struct BatchGeo<14, F> { using G = Geometry<14, 1, 9, 5, 4, 5>; };
template <bool F> struct BatchGeo<13, F> { using G = Geometry<13, 0, 8, 5, 3, 5>; };
template <bool F> struct BatchGeo<12, F> { using G = Geometry<12, 0, 6, 4, 3, 3>; };

template <int LOGN, bool F>
constexpr bool batch_geo_ok() {
    using G = typename BatchGeo<LOGN, F>::G;
    return G::THREADS == kBatchThreads && G::CLOG == batch_tile_clog(LOGN);
}
static_assert(batch_geo_ok<17, true>() && batch_geo_ok<16, true>() && batch_geo_ok<16, false>() &&
                  batch_geo_ok<15, true>() && batch_geo_ok<14, true>() &&
                  batch_geo_ok<13, true>() && batch_geo_ok<12, true>(),
              "batch tile geometries must match batch_geo.h");

template <int A, int B>
constexpr int cmax() {
    return A > B ? A : B;
}
// Largest work buffer / phase-2 slab of the tile geometries (words).
constexpr uint32_t kBatchWorkWords = (uint32_t)cmax<
    cmax<cmax<BatchGeo<17, true>::G::SMEM_WORDS, BatchGeo<16, true>::G::SMEM_WORDS>(),
         cmax<BatchGeo<16, false>::G::SMEM_WORDS, BatchGeo<15, true>::G::SMEM_WORDS>()>(),
    cmax<cmax<BatchGeo<14, true>::G::SMEM_WORDS, BatchGeo<13, true>::G::SMEM_WORDS>(),
         BatchGeo<12, true>::G::SMEM_WORDS>()>();
// dynamic shared memory: work buffer | 2 slot words (and padding)
template <bool Mul>
constexpr uint32_t batch_smem_words() {
    return ((kBatchWorkWords + 3u) & ~3u) + 4u;
}
template <bool Mul>
constexpr uint32_t batch_smem_bytes() {
    return 4u * batch_smem_words<Mul>();
}

// Where a body reads its input and writes its output.  GlobalCG: a limb
// slab this kernel wrote earlier (read through L2, not the read-only or L1
// paths).  MulGlobal: the output word is the Montgomery product of the
// transform's word and the word at the same offset of `gmul` (read first,
// through L2), then stored to `gout`.
enum class BIn { Global, GlobalCG };
enum class BOut { Global, MulGlobal };

// Hand-off of the next group index: CTA 0's thread 0 stores `value` into the
// slot word at `slot_sa` of every CTA of the cluster.
struct Bcast {
    uint32_t value;
    uint32_t slot_sa;
    bool on;
};

__device__ __forceinline__ void st_cluster_u32(uint32_t local_sa, uint32_t cta, uint32_t v) {
    uint32_t ra;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(local_sa), "r"(cta));
    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(ra), "r"(v) : "memory");
}

template <int CL>
__device__ __forceinline__ void bcast_release(const Bcast& bc) {
    if (bc.on) {
#pragma unroll
        for (int c = 0; c < CL; ++c) st_cluster_u32(bc.slot_sa, (uint32_t)c, bc.value);
    }
    __syncwarp();
    cluster_arrive_release();
    cluster_wait_acquire();
}

// Memory interface of one tile body (see DevCtx for the pass code's use).
template <class G, int CL, BIn IM, BOut OM>
struct BatchCtx {
    static constexpr bool kStaged = false;
    static constexpr int C = G::C;
    const uint32_t* __restrict__ gin;
    uint32_t* gout;
    const uint32_t* gmul;
    const TwPair* __restrict__ twp;
    uint32_t* smem;
    const uint32_t* stage;  // unused (direct input)
    uint32_t smem_sa;
    uint32_t q, q2, qinv, rank, base;
    Bcast bc;

    // ---- input ----
    // (a tile is one polynomial's limb: the polynomial index is always 0)
    __device__ __forceinline__ const uint32_t* g_base(int, uint32_t o) const { return gin + o; }
    __device__ __forceinline__ uint32_t g_ld(const uint32_t* b, uint32_t c) const {
        if constexpr (IM == BIn::Global) return __ldca(b + c);
        else return __ldcg(b + c);
    }
    __device__ __forceinline__ void g_ld4(const uint32_t* b, uint32_t c, uint32_t& x, uint32_t& y,
                                          uint32_t& z, uint32_t& w) const {
        uint4 t;
        if constexpr (IM == BIn::Global) t = __ldca(reinterpret_cast<const uint4*>(b + c));
        else t = __ldcg(reinterpret_cast<const uint4*>(b + c));
        x = t.x;
        y = t.y;
        z = t.z;
        w = t.w;
    }
    __device__ __forceinline__ const uint32_t* st_base(uint32_t w) const { return stage + w; }
    __device__ __forceinline__ uint32_t st_ld(const uint32_t* b, uint32_t c) const { return b[c]; }
    __device__ __forceinline__ void st_ld4(const uint32_t*, uint32_t, uint32_t&, uint32_t&,
                                           uint32_t&, uint32_t&) const {}
    // ---- output ----
    __device__ __forceinline__ uint32_t* o_base(int, uint32_t o) const { return gout + o; }
    __device__ __forceinline__ uint32_t mix(uint32_t v, uint32_t k) const {
        return mont_mul(v, k, q, qinv);
    }
    __device__ __forceinline__ void o_st(uint32_t* b, uint32_t c, uint32_t v) const {
        if constexpr (OM == BOut::MulGlobal) v = mix(v, __ldcg(gmul + (b - gout) + c));
        b[c] = v;
    }
    __device__ __forceinline__ void o_st4(uint32_t* b, uint32_t c, uint32_t x, uint32_t y,
                                          uint32_t z, uint32_t w) const {
        if constexpr (OM == BOut::MulGlobal) {
            const uint4 k = __ldcg(reinterpret_cast<const uint4*>(gmul + (b - gout) + c));
            x = mix(x, k.x);
            y = mix(y, k.y);
            z = mix(z, k.z);
            w = mix(w, k.w);
        }
        *reinterpret_cast<uint4*>(b + c) = make_uint4(x, y, z, w);
    }
    // ---- work buffer and scatter ----
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
    __device__ __forceinline__ auto r_base(uint32_t dst, uint32_t w) const {
        if constexpr (C == 1) {
            return smem + w;
        } else {
            uint32_t ra;
            asm("mapa.shared::cluster.u32 %0, %1, %2;"
                : "=r"(ra)
                : "r"(smem_sa + 4u * w), "r"(base + dst));
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
    // ---- twiddles ----
    __device__ __forceinline__ TwPair tw_at(uint32_t i) const {
        const uint2 t = __ldg(reinterpret_cast<const uint2*>(twp) + i);
        return TwPair{t.x, t.y};
    }
    // table entries 0 and 1 (the constants folded into the limb's stage 0)
    __device__ __forceinline__ TwPair fold_at(uint32_t i) const { return tw_at(i); }
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
    // ---- cluster protocol (the whole cluster takes part in every round) ----
    __device__ __forceinline__ void after_local_reads() const { cluster_arrive_relaxed(); }
    __device__ __forceinline__ void before_scatter() const { cluster_wait_acquire(); }
    __device__ __forceinline__ void phase_sync() const { bcast_release<CL>(bc); }
};

// A round without a tile: the same barrier sequence as a body.
template <int CL>
__device__ __forceinline__ void idle_round(const Bcast& bc) {
    cluster_arrive_relaxed();
    cluster_wait_acquire();
    bcast_release<CL>(bc);
}

struct NoPrefetch {
    __device__ __forceinline__ void operator()() const {}
};

// Per-CTA state shared by the bodies of a tile.
struct BatchCta {
    uint32_t* smem;
    uint32_t smem_sa;
    uint32_t rank;  // in the cluster
};

// A pointer re-read from memory with a volatile load.  The two forward
// bodies of a multiply tile use the same twiddle table; with the pointer
// known equal, the compiler merges the second body's read-only twiddle loads
// into the first's and keeps them all live across the body.
__device__ __forceinline__ const void* reload_ptr(const void* const* addr) {
    uint64_t v;
    asm volatile("ld.volatile.global.u64 %0, [%1];" : "=l"(v) : "l"(addr));
    return reinterpret_cast<const void*>(v);
}
// A tile re-read field by field before each body of a multiply, so that no
// field stays live in registers across a body.
__device__ __forceinline__ BatchTile reload_tile(const BatchTile* tp) {
    BatchTile t;
    t.data = (uint32_t*)reload_ptr((const void* const*)&tp->data);
    t.operand = (const uint32_t*)reload_ptr((const void* const*)&tp->operand);
    t.tw_fwd = reload_ptr(&tp->tw_fwd);
    t.tw_inv = reload_ptr(&tp->tw_inv);
    uint32_t q, qinv;
    asm volatile("ld.volatile.global.u32 %0, [%1];" : "=r"(q) : "l"(&tp->q));
    asm volatile("ld.volatile.global.u32 %0, [%1];" : "=r"(qinv) : "l"(&tp->qinv));
    t.q = q;
    t.qinv = qinv;
    t.logn = 0;
    t.op = 0;
    return t;
}

template <class G, int CL, BIn IM, BOut OM>
__device__ __forceinline__ BatchCtx<G, CL, IM, OM> make_ctx(const BatchCta& cta,
                                                            const BatchTile& t, uint32_t sub,
                                                            const uint32_t* in, uint32_t* out,
                                                            const uint32_t* mul, const void* tw,
                                                            const Bcast& bc) {
    BatchCtx<G, CL, IM, OM> c;
    c.gin = in;
    c.gout = out;
    c.gmul = mul;
    c.twp = reinterpret_cast<const TwPair*>(tw);
    c.smem = cta.smem;
    c.stage = nullptr;
    c.smem_sa = cta.smem_sa;
    c.q = t.q;
    c.q2 = 2u * t.q;
    c.qinv = t.qinv;
    c.rank = sub;
    c.base = cta.rank - sub;
    c.bc = bc;
    return c;
}

// Runs the bodies of one tile; returns the rounds used.  `last` is the
// group's last round (the one that hands off the next group index).
template <int LOGN, int CL, bool Mul, class Arith>
__device__ __forceinline__ uint32_t run_tile_arith(const BatchCta& cta, const BatchTile& t,
                                                   const BatchTile* tp, uint32_t sub,
                                                   uint32_t last, Bcast bc) {
    const bool leader = bc.on;
    auto round_bc = [&](uint32_t r) {
        Bcast b = bc;
        b.on = leader && r == last;
        return b;
    };
    if (t.op == kOpForward) {
        using G = typename BatchGeo<LOGN, true>::G;
        auto c = make_ctx<G, CL, BIn::Global, BOut::Global>(cta, t, sub, t.data, t.data, nullptr,
                                                            t.tw_fwd, round_bc(0));
        fused_forward_body<G, Arith>(c, NoPrefetch{});
        __syncthreads();
        return 1;
    }
    if (t.op == kOpInverse) {
        using G = typename BatchGeo<LOGN, false>::G;
        auto c = make_ctx<G, CL, BIn::Global, BOut::Global>(cta, t, sub, t.data, t.data, nullptr,
                                                            t.tw_inv, round_bc(0));
        fused_inverse_body<G, Arith>(c, NoPrefetch{});
        __syncthreads();
        return 1;
    }
    if constexpr (Mul) {
        // forward bodies use the forward geometry, the inverse body the
        // inverse one: both give CTA `rank` the same phase-2 slab
        // [rank * M, (rank + 1) * M) (same cluster size), and the CTA barrier
        // between bodies makes the slab written by one body visible to every
        // thread of the next
        using G = typename BatchGeo<LOGN, true>::G;
        using GI = typename BatchGeo<LOGN, false>::G;
        static_assert(G::CLOG == GI::CLOG && G::M == GI::M, "multiply bodies share CTA slabs");
        if (t.op == kOpMultiply) {
            {   // b -> spectrum of b, in place
                const BatchTile u = reload_tile(tp);
                auto cb = make_ctx<G, CL, BIn::Global, BOut::Global>(cta, u, sub, u.data, u.data,
                                                                     nullptr, u.tw_fwd,
                                                                     round_bc(0));
                fused_forward_body<G, Arith>(cb, NoPrefetch{});
                __syncthreads();
            }
            {   // spectrum of a times spectrum of b, into b's slab
                const BatchTile u = reload_tile(tp);
                auto ca = make_ctx<G, CL, BIn::Global, BOut::MulGlobal>(
                    cta, u, sub, u.operand, u.data, u.data, u.tw_fwd, round_bc(1));
                fused_forward_body<G, Arith>(ca, NoPrefetch{});
                __syncthreads();
            }
            {
                const BatchTile u = reload_tile(tp);
                auto cc = make_ctx<GI, CL, BIn::GlobalCG, BOut::Global>(
                    cta, u, sub, u.data, u.data, nullptr, u.tw_inv, round_bc(2));
                fused_inverse_body<GI, Arith>(cc, NoPrefetch{});
                __syncthreads();
            }
            return 3;
        }
        if (t.op == kOpMultiplySpectrum) {
            {
                const BatchTile u = reload_tile(tp);
                auto cb = make_ctx<G, CL, BIn::Global, BOut::MulGlobal>(
                    cta, u, sub, u.data, u.data, u.operand, u.tw_fwd, round_bc(0));
                fused_forward_body<G, Arith>(cb, NoPrefetch{});
                __syncthreads();
            }
            {
                const BatchTile u = reload_tile(tp);
                auto cc = make_ctx<GI, CL, BIn::GlobalCG, BOut::Global>(
                    cta, u, sub, u.data, u.data, nullptr, u.tw_inv, round_bc(1));
                fused_inverse_body<GI, Arith>(cc, NoPrefetch{});
                __syncthreads();
            }
            return 2;
        }
    }
    return 0;
}

template <int CL, bool Mul, class Arith>
__device__ __forceinline__ uint32_t run_tile(const BatchCta& cta, const BatchTile* tp,
                                             uint32_t sub, uint32_t last, Bcast bc) {
    const BatchTile t = *tp;
    switch (t.logn) {
        case 12: return run_tile_arith<12, CL, Mul, Arith>(cta, t, tp, sub, last, bc);
        case 13: return run_tile_arith<13, CL, Mul, Arith>(cta, t, tp, sub, last, bc);
        case 14: return run_tile_arith<14, CL, Mul, Arith>(cta, t, tp, sub, last, bc);
        case 15: return run_tile_arith<15, CL, Mul, Arith>(cta, t, tp, sub, last, bc);
        case 16: return run_tile_arith<16, CL, Mul, Arith>(cta, t, tp, sub, last, bc);
        case 17:
            if constexpr (CL >= 16) return run_tile_arith<17, CL, Mul, Arith>(cta, t, tp, sub, last, bc);
            else return 0;
        default: return 0;
    }
}

// grid.x = CL * resident clusters; cluster dims (CL, 1, 1).  Arith: the
// range discipline of every tile of the launch (Lazy4 when all moduli are
// below 2^30, else Lazy2), fixed per kernel so that one path's registers fit
// the launch bounds (4 CTAs/SM: the persistent loop's own state does not fit
// the 48 registers of 5).
template <int CL, bool Mul, class Arith>
__global__ void __launch_bounds__(kBatchThreads, 4) batch_kernel(BatchArgs a) {
    extern __shared__ __align__(16) uint32_t smem[];
    constexpr uint32_t kSlotOff = batch_smem_words<Mul>() - 4u;
    BatchCta cta;
    cta.smem = smem;
    cta.smem_sa = (uint32_t)__cvta_generic_to_shared(smem);
    cta.rank = cluster_rank();
    const uint32_t slot_sa = cta.smem_sa + 4u * kSlotOff;
    const bool leader = cta.rank == 0 && threadIdx.x == 0;
    // every CTA of the cluster is running before any DSMEM store
    cluster_arrive_release();
    cluster_wait_acquire();
    if (leader) {
        const uint32_t g0 = atomicAdd(a.counter, 1u);
        for (int c = 0; c < CL; ++c) st_cluster_u32(slot_sa, (uint32_t)c, g0);
    }
    __syncwarp();
    cluster_arrive_release();
    cluster_wait_acquire();
    for (uint32_t it = 0;; ++it) {
        const uint32_t g = *(volatile uint32_t*)(smem + kSlotOff + (it & 1u));
        if (g >= a.groups) break;  // the same value in every CTA of the cluster
        uint32_t nxt = 0;
        if (leader) nxt = atomicAdd(a.counter, 1u);
        __syncwarp();  // reconverge before the bodies' .aligned cluster barriers
        const uint32_t rounds = __ldg(a.rounds + g);
        const uint32_t sl = __ldg(a.slots + (size_t)g * CL + cta.rank);
        const Bcast bc{nxt, slot_sa + 4u * ((it + 1u) & 1u), leader};
        uint32_t done = 0;
        if (sl != kIdleSlot) {
            done = run_tile<CL, Mul, Arith>(cta, a.tiles + (sl & kSlotTileMask), sl >> kSlotSubShift,
                                     rounds - 1u, bc);
        }
        for (uint32_t r = done; r < rounds; ++r) {
            Bcast b = bc;
            b.on = leader && r == rounds - 1u;
            idle_round<CL>(b);
        }
    }
}

}  // namespace nttb
