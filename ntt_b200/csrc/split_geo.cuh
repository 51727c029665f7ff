// Geometry and passes of the split transform kernels (split_kernel.cuh),
// kept free of device-only code so that the CPU emulator of tests/emu can
// run the same pass functions thread by thread.
#pragma once
#include <type_traits>

#include "ntt_core.cuh"

namespace nttb {

// Extra register bits of the first phase-2 pass: the lowest positions from
// bit 5 up outside its butterfly range, so that its lanes are bits 0..4.
template <int MB, int PLO, int KB, int XB>
constexpr uint32_t split_first_extras() {
    uint32_t m = 0;
    for (int p = 5, c = 0; p < MB && c < XB; ++p)
        if (!(p >= PLO && p < PLO + KB)) {
            m |= 1u << p;
            ++c;
        }
    return m;
}

// Geometry of split configuration S(LOGN, CLOG, EB, K2A, K2B) (configs.h).
template <int LOGN_, int CLOG_, int EB_, int K2A_, int K2B_>
struct SplitGeo {
    static constexpr int LOGN = LOGN_, CLOG = CLOG_, EB = EB_, NP = 1;
    static constexpr int R1 = EB, R2 = LOGN - R1;
    static constexpr int K2A = K2A_, K2B = K2B_, K2C = R2 - K2A_ - K2B_;
    static constexpr int C = 1 << CLOG;
    static constexpr int MB = LOGN - CLOG;
    static constexpr uint32_t M = 1u << MB;
    static constexpr int S1 = R2 - CLOG;
    static constexpr uint32_t W1 = 1u << S1;
    static constexpr uint32_t H2 = 1u << (R1 - CLOG);
    static constexpr int TB = MB - EB;
    static constexpr int THREADS = 1 << TB;
    static_assert(C > 1 && R1 >= CLOG, "each CTA of the cluster owns at least one row");
    static_assert(S1 >= 5, "phase-1 lanes take 32 consecutive columns");
    static_assert(R2 - K2A >= 5, "the first phase-2 pass keeps bits 0..4 for its lanes");
    static_assert(K2A >= 1 && K2A <= EB && K2B >= 1 && K2B <= EB && K2C >= 0 && K2C <= EB,
                  "phase-2 passes");
    static_assert(TB >= 5 && TB <= 10, "32..1024 threads per CTA");
    static_assert(LOGN < kTwPermMinLogN || R2 >= kTwPermStages,
                  "the interleaved twiddle stages must all lie in phase 2");
    // registers: the 2^EB data words plus 32.  Measured on B200 at 2^16 x 16
    // (EB 5): 64 registers and 4 CTAs per SM against 48 and 5 give the same
    // batched times (forward 2% faster, inverse 0.5% slower) and a 9% faster
    // one-polynomial call (the 16-CTA split: 256 CTAs of 128 threads, under
    // two per SM, so per-thread ILP decides).
    static constexpr int REG_BUDGET = (1 << EB) + 32;
    static constexpr int MIN_BLOCKS = 65536 / (THREADS * REG_BUDGET) > 0
                                          ? 65536 / (THREADS * REG_BUDGET) : 1;

    using P1 = PassLayout<MB, MB - EB, EB, EB, 0>;
    using P2A = PassLayoutX<MB, R2 - K2A, K2A, EB,
                            split_first_extras<MB, R2 - K2A, K2A, EB - K2A>()>;
    using P2B = PassLayout<MB, R2 - K2A - K2B, K2B, EB, 0>;
    using P2C = PassLayout<MB, 0, (K2C > 0 ? K2C : 1), EB, 0>;
    using PLast = std::conditional_t<(K2C > 0), P2C, P2B>;

    using LT = SplitLayoutTable<LOGN, CLOG, EB, K2A, K2B>;
    static_assert(LT::lanes_P2A == P2A::kLanes && LT::lanes_P2B == P2B::kLanes,
                  "layouts_gen.h is stale: rerun gen_layouts.py");
    using XW = Spread<LT::XW[0], LT::XW[1], LT::XW[2], LT::XW[3]>;
    static constexpr uint32_t SLAB_WORDS = ((uint32_t)LT::XW[4] + 3u) & ~3u;
    static constexpr uint32_t SMEM_BYTES = SLAB_WORDS * 4u;

    // exchanges between passes that keep every warp's words stay warp-local
    static constexpr uint32_t kChunkWarps = ((THREADS / 32u) - 1u) << (MB - (TB - 5));
    static constexpr bool kABWarp = warp_bits<P2A>() == warp_bits<P2B>();
    static constexpr bool kBCWarp = warp_bits<P2B>() == warp_bits<P2C>();
    static constexpr bool kChunkWarp = warp_bits<PLast>() == kChunkWarps;
};

// The passes of the split transforms, each run by every thread of every CTA
// of the limb's cluster between barriers (the kernels below; the CPU
// emulator of tests/emu runs them thread by thread).  Phase-1 loads stream
// from global memory; phase-2 loads of the words other CTAs wrote must
// bypass L1 (the kernels switch ctx.cg between the two).
template <class G, class Arith, class Ctx>
struct SplitFwd {
    using Mp = Maps<G>;
    using X = typename G::XW;
    using P1 = typename G::P1;
    using P2A = typename G::P2A;
    using P2B = typename G::P2B;
    using P2C = typename G::P2C;
    // phase 1: the thread's column, from and back to global memory in place
    NTT_HD static void p1(Ctx& ctx, uint32_t tid) {
        uint32_t v[1][P1::E];
        const uint32_t d = P1::dep(tid);
        const uint32_t g = Mp::g1(d) + Mp::g1_rank(ctx.rank);
        load_global<P1, G::W1, G1Map<G>>(ctx, v, g);
        run_stages<G, P1, Arith, true, false, true>(ctx, v, d);
        store_global<P1, G::W1, G1Map<G>>(ctx, v, g, Ident{});
    }
    // phase 2, first pass: the CTA's rows from L2 into the work buffer
    NTT_HD static void p2a(Ctx& ctx, uint32_t tid) {
        uint32_t v[1][P2A::E];
        const uint32_t d = P2A::dep(tid);
        load_global<P2A, (1u << 30), G2Map>(ctx, v, d + ctx.rank * G::M);
        run_stages<G, P2A, Arith, true, true, false>(ctx, v, d);
        store_smem<P2A, X, G::SLAB_WORDS>(ctx, v, d);
    }
    NTT_HD static void p2b(Ctx& ctx, uint32_t tid) {
        const FwdFinal<Arith> fin{ctx.q, ctx.q2};
        uint32_t v[1][P2B::E];
        const uint32_t d = P2B::dep(tid);
        load_smem<P2B, X, G::SLAB_WORDS>(ctx, v, d);
        run_stages<G, P2B, Arith, true, true, false>(ctx, v, d);
        if constexpr (G::K2C == 0)
            ct_for<P2B::E>([&](auto R) { v[0][decltype(R)::value] = fin(v[0][decltype(R)::value]); });
        store_smem<P2B, X, G::SLAB_WORDS>(ctx, v, d);
    }
    NTT_HD static void p2c(Ctx& ctx, uint32_t tid) {
        if constexpr (G::K2C > 0) {
            const FwdFinal<Arith> fin{ctx.q, ctx.q2};
            uint32_t v[1][P2C::E];
            const uint32_t d = P2C::dep(tid);
            load_smem<P2C, X, G::SLAB_WORDS>(ctx, v, d);
            run_stages<G, P2C, Arith, true, true, false>(ctx, v, d);
            ct_for<P2C::E>([&](auto R) { v[0][decltype(R)::value] = fin(v[0][decltype(R)::value]); });
            store_smem<P2C, X, G::SLAB_WORDS>(ctx, v, d);
        }
    }
    // the canonical words leave in warp chunks
    NTT_HD static void out(Ctx& ctx, uint32_t tid) { slab_out<G, X>(ctx, tid); }
};

template <class G, class Arith, class Ctx>
struct SplitInv {
    using Mp = Maps<G>;
    using X = typename G::XW;
    using P1 = typename G::P1;
    using P2A = typename G::P2A;
    using P2B = typename G::P2B;
    using P2C = typename G::P2C;
    // the CTA's rows enter the work buffer in warp chunks
    NTT_HD static void in(Ctx& ctx, uint32_t tid) { slab_in<G, X>(ctx, tid); }
    NTT_HD static void p2c(Ctx& ctx, uint32_t tid) {
        if constexpr (G::K2C > 0) {
            uint32_t v[1][P2C::E];
            const uint32_t d = P2C::dep(tid);
            load_smem<P2C, X, G::SLAB_WORDS>(ctx, v, d);
            run_stages<G, P2C, Arith, false, true, false>(ctx, v, d);
            store_smem<P2C, X, G::SLAB_WORDS>(ctx, v, d);
        }
    }
    NTT_HD static void p2b(Ctx& ctx, uint32_t tid) {
        uint32_t v[1][P2B::E];
        const uint32_t d = P2B::dep(tid);
        load_smem<P2B, X, G::SLAB_WORDS>(ctx, v, d);
        run_stages<G, P2B, Arith, false, true, false>(ctx, v, d);
        store_smem<P2B, X, G::SLAB_WORDS>(ctx, v, d);
    }
    // last phase-2 pass: back to the CTA's rows in place
    NTT_HD static void p2a(Ctx& ctx, uint32_t tid) {
        uint32_t v[1][P2A::E];
        const uint32_t d = P2A::dep(tid);
        load_smem<P2A, X, G::SLAB_WORDS>(ctx, v, d);
        run_stages<G, P2A, Arith, false, true, false>(ctx, v, d);
        store_global<P2A, (1u << 30), G2Map>(ctx, v, d + ctx.rank * G::M, Ident{});
    }
    // phase 1 (after the exchange): the thread's column, read through L2
    NTT_HD static void p1(Ctx& ctx, uint32_t tid) {
        uint32_t v[1][P1::E];
        const uint32_t d = P1::dep(tid);
        const uint32_t g = Mp::g1(d) + Mp::g1_rank(ctx.rank);
        load_global<P1, G::W1, G1Map<G>>(ctx, v, g);
        run_stages<G, P1, Arith, false, false, true>(ctx, v, d);
        store_global<P1, G::W1, G1Map<G>>(ctx, v, g, Ident{});
    }
};

}  // namespace nttb
