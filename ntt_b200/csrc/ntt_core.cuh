// Register-pass machinery of the fused two-phase NTT / INTT (host + device).
//
// Math (same map as the reference's cpu_ntt_butterfly / cpu_intt_butterfly,
// src/v04_montgomery.cu:742-784, and its two-phase kernels v04:196-565):
// a limb of N = 2^n words is viewed as a 2^R1 x 2^R2 row-major matrix
// (i = rho * 2^R2 + kappa).  Forward CT stages 0..R1-1 ("phase 1") act on
// the row bits -- independent column transforms whose twiddles depend only on
// rho; stages R1..n-1 ("phase 2") act on the column bits -- independent row
// transforms.  Stage s pairs i and i + 2^(n-1-s) with twiddle
// tw[2^s + (i >> (n-s))], tw[i] = psi^bitrev(i).
//
// B200 mapping: one limb is spread over a thread-block cluster of C = 2^c
// CTAs, each holding M = N / C words in shared memory.  In phase 1, CTA r
// owns the column slab kappa in [r*W1, (r+1)*W1) (W1 = 2^(R2-c)); in phase 2
// it owns the row slab rho in [r*H2, (r+1)*H2) (H2 = 2^(R1-c)), which is the
// contiguous range [r*M, (r+1)*M).  Between the phases every CTA scatters its
// slab into the owners' shared memory over DSMEM (st.shared::cluster), so a
// limb is read from HBM once and written once.  C = 1 is the same code with
// the scatter landing in the CTA's own shared memory.
//
// Inside a phase, stages run in "register passes": each thread loads E = 2^EB
// words, runs KB <= EB radix-2 stages on them in registers, and stores them
// back.  A pass is described at compile time by the bit positions of the
// CTA-local index lambda that it owns (PassLayout): the KB butterfly bits
// [PLO, PLO+KB), plus EB-KB "extra" bits (the lowest positions outside the
// butterfly range, so each thread's words form contiguous runs for 128-bit
// global access), the remaining bits being the thread index.  All index maps
// below are linear over disjoint bit sets, so every per-register address is a
// per-thread base plus a compile-time constant.
#pragma once
#include "arith.cuh"

namespace nttb {

// ---------------------------------------------------------------------------
// Compile-time layout of one register pass.
// ---------------------------------------------------------------------------
template <int MB_, int PLO_, int KB_, int EB_>
struct PassLayout {
    static constexpr int MB = MB_, PLO = PLO_, KB = KB_, EB = EB_;
    static constexpr int XB = EB - KB;
    static constexpr int E = 1 << EB;
    static_assert(KB >= 1 && KB <= EB && EB <= MB, "bad pass layout");
    static_assert(PLO >= 0 && PLO + KB <= MB, "bad pass layout");

    static constexpr bool in_bfly(int p) { return p >= PLO && p < PLO + KB; }
    // j-th extra position: the XB lowest positions outside the butterfly range.
    static constexpr int xpos(int j) {
        int cnt = 0;
        for (int p = 0; p < MB; ++p) {
            if (in_bfly(p)) continue;
            if (cnt == j) return p;
            ++cnt;
        }
        return -1;
    }
    static constexpr uint32_t reg_mask() {
        uint32_t m = 0;
        for (int p = PLO; p < PLO + KB; ++p) m |= 1u << p;
        for (int j = 0; j < XB; ++j) m |= 1u << xpos(j);
        return m;
    }
    // lambda offset of register r: low XB bits of r = extra coordinate,
    // high KB bits = butterfly coordinate.
    static constexpr uint32_t off(int r) {
        uint32_t o = (uint32_t)(r >> XB) << PLO;
        for (int j = 0; j < XB; ++j)
            if ((r >> j) & 1) o |= 1u << xpos(j);
        return o;
    }
    static constexpr int reg_of(uint32_t o) {
        for (int r = 0; r < E; ++r)
            if (off(r) == o) return r;
        return -1;
    }
    // number of low lambda bits owned by registers (contiguous run = 2^run)
    static constexpr int run_bits() {
        int v = 0;
        while (v < MB && ((reg_mask() >> v) & 1u)) ++v;
        return v;
    }
    // extra coordinate bits that sit above the butterfly range
    static constexpr int xhi_bits() {
        int c = 0;
        for (int j = 0; j < XB; ++j)
            if (xpos(j) > PLO + KB - 1) ++c;
        return c;
    }
    // Deposit the thread index into the non-register positions (ascending).
    NTT_HD static uint32_t dep(uint32_t t) {
        uint32_t v = t;
#pragma unroll
        for (int p = 0; p < MB; ++p) {
            if ((reg_mask() >> p) & 1u) v = ((v >> p) << (p + 1)) | (v & ((1u << p) - 1u));
        }
        return v;
    }
};

// ---------------------------------------------------------------------------
// Geometry of one fused transform configuration.
//   LOGN: n;  CLOG: c (cluster of 2^c CTAs);  R1: phase-1 stages;
//   EB: log2 words per thread per pass;  K1A / K2A: stages of the first
//   register pass of phase 1 / phase 2 (the rest, if any, is a second pass).
// ---------------------------------------------------------------------------
template <int LOGN_, int CLOG_, int R1_, int EB_, int K1A_, int K2A_>
struct Geometry {
    static constexpr int LOGN = LOGN_, CLOG = CLOG_, R1 = R1_, EB = EB_;
    static constexpr int R2 = LOGN - R1;
    static constexpr int C = 1 << CLOG;
    static constexpr int MB = LOGN - CLOG;  // local bits
    static constexpr uint32_t M = 1u << MB;
    static constexpr int S1 = R2 - CLOG;  // log2 W1
    static constexpr uint32_t W1 = 1u << S1;
    static constexpr uint32_t H2 = 1u << (R1 - CLOG);
    static constexpr int TB = MB - EB;
    static constexpr int THREADS = 1 << TB;
    static constexpr int K1A = K1A_, K1B = R1 - K1A_;
    static constexpr int K2A = K2A_, K2B = R2 - K2A_;
    static_assert(R1 >= CLOG && R2 >= CLOG, "each phase needs at least c stages");
    static_assert(K1A >= 1 && K1A <= EB && K1B >= 0 && K1B <= EB, "phase-1 passes");
    static_assert(K2A >= 1 && K2A <= EB && K2B >= 0 && K2B <= EB, "phase-2 passes");
    static_assert(TB >= 5 && TB <= 10, "32..1024 threads per CTA");
    // Padded shared-memory layout: one pad word per 32 (bank spreading).
    static constexpr uint32_t SMEM_WORDS = M + (M >> 5);
    static constexpr uint32_t SMEM_BYTES = SMEM_WORDS * 4u;

    // Pass layouts (forward order).  Phase-1 lambda bits: [S1, MB) (row bits),
    // processed top-down; phase-2 bits [0, R2) (column bits), top-down.
    using P1A = PassLayout<MB, MB - K1A, K1A, EB>;
    using P1B = PassLayout<MB, S1, (K1B > 0 ? K1B : 1), EB>;
    using P2A = PassLayout<MB, R2 - K2A, K2A, EB>;
    using P2B = PassLayout<MB, 0, (K2B > 0 ? K2B : 1), EB>;
};

NTT_HD uint32_t smem_phys(uint32_t lam) { return lam + (lam >> 5); }

// lambda maps (see file header); all linear over disjoint bit sets.
template <class G>
struct Maps {
    // phase-1 slab lambda -> word offset in the limb (without the rank term)
    NTT_HD static uint32_t g1(uint32_t lam) {
        return ((lam >> G::S1) << G::R2) + (lam & (G::W1 - 1u));
    }
    NTT_HD static uint32_t g1_rank(uint32_t rank) { return rank * G::W1; }
    // phase-2 slab lambda -> word offset (without rank term rank*M)
    NTT_HD static uint32_t g2(uint32_t lam) { return lam; }
    // forward scatter: phase-1 lambda -> destination rank / phase-2 lambda
    NTT_HD static uint32_t f_dst(uint32_t lam) { return lam >> (G::MB - G::CLOG); }
    NTT_HD static uint32_t f_lam(uint32_t lam) {
        return (((lam >> G::S1) & (G::H2 - 1u)) << G::R2) + (lam & (G::W1 - 1u));
    }
    // inverse scatter: phase-2 lambda -> destination rank / phase-1 lambda
    NTT_HD static uint32_t i_dst(uint32_t lam) {
        return (lam & ((1u << G::R2) - 1u)) >> G::S1;
    }
    NTT_HD static uint32_t i_lam(uint32_t lam) {
        return ((lam >> G::R2) << G::S1) + (lam & (G::W1 - 1u));
    }
    NTT_HD static uint32_t i_lam_rank(uint32_t rank) { return (rank * G::H2) << G::S1; }
    // twiddle index base for a stage acting on lambda bit p
    NTT_HD static uint32_t tw_base_p1(int p) { return 1u << (G::MB - 1 - p); }
    NTT_HD static uint32_t tw_base_p2(int p, uint32_t rank) {
        return (1u << (G::LOGN - 1 - p)) + (rank << (G::LOGN - G::CLOG - 1 - p));
    }
};

// ---------------------------------------------------------------------------
// Register-level stage loops.
// ---------------------------------------------------------------------------

// Load a block of 2^k consecutive twiddle pairs starting at `idx` (aligned to
// 2^k) and apply the CT (Fwd) or GS stage that uses them.
template <class L, class Arith, bool Fwd, int k, class Ctx>
NTT_HD void stage(Ctx& ctx, uint32_t (&v)[L::E], uint32_t tbase, bool fold_first,
                  bool fold_last) {
    // CT: stage k of the pass acts on lambda bit p = PLO + KB - 1 - k, groups
    // = top k butterfly-coordinate bits.  GS: stage k acts on bit p = PLO + k,
    // groups = top KB-1-k butterfly bits.
    constexpr int p = Fwd ? (L::PLO + L::KB - 1 - k) : (L::PLO + k);
    constexpr int gbits = Fwd ? k : (L::KB - 1 - k);
    constexpr int bbit = Fwd ? (L::KB - 1 - k) : k;  // butterfly coordinate bit
    constexpr int stride = 1 << (bbit + L::XB);      // register distance
    constexpr int XHB = L::xhi_bits();
    constexpr int XLB = L::XB - XHB;
    const uint32_t q = ctx.q, q2 = ctx.q2;
#pragma unroll
    for (int xh = 0; xh < (1 << XHB); ++xh) {
        // twiddle slot contribution of the extra bits above the butterfly
        // range: off >> (p+1) restricted to those bits (a multiple of 2^gbits)
        uint32_t xoff = L::off(xh << XLB) >> (p + 1);
#pragma unroll
        for (int g = 0; g < (1 << gbits); ++g) {
            TwPair w;
            if ((Fwd && fold_first) || (!Fwd && fold_last)) {
                w = ctx.tw(1u);  // stage 0 of the limb: single twiddle index 1
            } else {
                w = ctx.tw(tbase + xoff + (uint32_t)g);
            }
            // butterflies of group g: bcoord = (g << (bbit+1)) | (lo), lo < 2^bbit
#pragma unroll
            for (int lo = 0; lo < (1 << bbit); ++lo) {
#pragma unroll
                for (int xl = 0; xl < (1 << XLB); ++xl) {
                    const int bc = (g << (bbit + 1)) | lo;
                    const int r = (bc << L::XB) | (xh << XLB) | xl;
                    if (Fwd) {
                        if (fold_first)
                            Arith::ct_first(v[r], v[r + stride], ctx.tw(0u), w, q, q2);
                        else
                            Arith::ct(v[r], v[r + stride], w.w, w.wp, q, q2);
                    } else {
                        if (fold_last)
                            Arith::gs_last(v[r], v[r + stride], ctx.tw(0u), w, q, q2);
                        else
                            Arith::gs(v[r], v[r + stride], w.w, w.wp, q, q2);
                    }
                }
            }
        }
    }
}

// Run all KB stages of a pass.  `phase2` selects the twiddle base rule;
// `first_is_limb_stage0` / `last_is_limb_stage0`: this pass contains global
// stage 0 (the forward's first stage / the inverse's last stage), which gets
// the Montgomery / N^{-1} factor folded in.
template <class G, class L, class Arith, bool Fwd, bool Phase2, bool HasStage0, class Ctx>
NTT_HD void run_stages(Ctx& ctx, uint32_t (&v)[L::E], uint32_t d) {
    using Mp = Maps<G>;
#define NTTB_STAGE(K)                                                                      \
    if constexpr ((K) < L::KB) {                                                           \
        constexpr int p = Fwd ? (L::PLO + L::KB - 1 - (K)) : (L::PLO + (K));               \
        const uint32_t tb = (Phase2 ? Mp::tw_base_p2(p, ctx.rank) : Mp::tw_base_p1(p)) +   \
                            (d >> (p + 1));                                                \
        const bool s0 = HasStage0 && (Fwd ? ((K) == 0) : ((K) == L::KB - 1));             \
        stage<L, Arith, Fwd, (K)>(ctx, v, tb, Fwd && s0, !Fwd && s0);                      \
    }
    NTTB_STAGE(0)
    NTTB_STAGE(1)
    NTTB_STAGE(2)
    NTTB_STAGE(3)
    NTTB_STAGE(4)
    NTTB_STAGE(5)
#undef NTTB_STAGE
}

// ---------------------------------------------------------------------------
// Loads / stores of a pass's registers.
// ---------------------------------------------------------------------------

// Vector width (words) usable for a global access whose address map keeps
// runs of `lim` consecutive lambdas contiguous.
template <class L>
constexpr int vec_width(int lim) {
    int run = 1 << L::run_bits();
    int w = run < 4 ? run : 4;
    return w < lim ? w : lim;
}

template <class L, class Ctx, class AddrFn>
NTT_HD void load_global(Ctx& ctx, uint32_t (&v)[L::E], uint32_t gbase, AddrFn gmap,
                        int lim) {
    // gmap(off) -> global word offset contribution of register offset `off`
    if (vec_width<L>(lim) == 4 && lim >= 4) {
#pragma unroll
        for (int r = 0; r < L::E; ++r) {
            if ((L::off(r) & 3u) == 0) {
                uint32_t a, b, c, e;
                ctx.gload4(gbase + gmap(L::off(r)), a, b, c, e);
                v[L::reg_of(L::off(r) + 0)] = a;
                v[L::reg_of(L::off(r) + 1)] = b;
                v[L::reg_of(L::off(r) + 2)] = c;
                v[L::reg_of(L::off(r) + 3)] = e;
            }
        }
    } else {
#pragma unroll
        for (int r = 0; r < L::E; ++r) v[r] = ctx.gload(gbase + gmap(L::off(r)));
    }
}

template <class L, class Ctx, class AddrFn, class ValFn>
NTT_HD void store_global(Ctx& ctx, uint32_t (&v)[L::E], uint32_t gbase, AddrFn gmap,
                         int lim, ValFn fin) {
    if (vec_width<L>(lim) == 4 && lim >= 4) {
#pragma unroll
        for (int r = 0; r < L::E; ++r) {
            if ((L::off(r) & 3u) == 0) {
                ctx.gstore4(gbase + gmap(L::off(r)), fin(v[L::reg_of(L::off(r) + 0)]),
                            fin(v[L::reg_of(L::off(r) + 1)]), fin(v[L::reg_of(L::off(r) + 2)]),
                            fin(v[L::reg_of(L::off(r) + 3)]));
            }
        }
    } else {
#pragma unroll
        for (int r = 0; r < L::E; ++r) ctx.gstore(gbase + gmap(L::off(r)), fin(v[r]));
    }
}

template <class L, class Ctx>
NTT_HD void load_smem(Ctx& ctx, uint32_t (&v)[L::E], uint32_t d) {
    const uint32_t base = smem_phys(d);
#pragma unroll
    for (int r = 0; r < L::E; ++r) v[r] = ctx.sload(base + smem_phys(L::off(r)));
}

template <class L, class Ctx>
NTT_HD void store_smem(Ctx& ctx, uint32_t (&v)[L::E], uint32_t d) {
    const uint32_t base = smem_phys(d);
#pragma unroll
    for (int r = 0; r < L::E; ++r) ctx.sstore(base + smem_phys(L::off(r)), v[r]);
}

// ---------------------------------------------------------------------------
// The passes of a forward / inverse transform, one function per pass, each a
// self-contained load -> stages -> store step (barriers live in the caller).
// ---------------------------------------------------------------------------

struct Ident {
    NTT_HD uint32_t operator()(uint32_t x) const { return x; }
};

template <class Arith>
struct FwdFinal {
    uint32_t q, q2;
    NTT_HD uint32_t operator()(uint32_t x) const { return Arith::fwd_final(x, q, q2); }
};

template <class G, class Arith, class Ctx>
struct Forward {
    using Mp = Maps<G>;
    using P1A = typename G::P1A;
    using P1B = typename G::P1B;
    using P2A = typename G::P2A;
    using P2B = typename G::P2B;

    struct G1 {
        NTT_HD uint32_t operator()(uint32_t o) const { return Maps<G>::g1(o); }
    };
    struct G2 {
        NTT_HD uint32_t operator()(uint32_t o) const { return o; }
    };

    // Scatter a phase-1 pass's registers to the phase-2 owners.
    template <class L>
    NTT_HD static void scatter(Ctx& ctx, uint32_t (&v)[L::E], uint32_t d) {
        const uint32_t dd = Mp::f_dst(d);
        const uint32_t dl = Mp::f_lam(d) + Mp::g1_rank(ctx.rank);
#pragma unroll
        for (int r = 0; r < L::E; ++r) {
            const uint32_t o = L::off(r);
            ctx.rstore(dd + Mp::f_dst(o), smem_phys(dl + Mp::f_lam(o)), v[r]);
        }
    }

    // Phase-1 first pass: global (normal domain) -> stages incl. stage 0 ->
    // SMEM (if a second phase-1 pass follows) or the scatter.
    NTT_HD static void pass1a(Ctx& ctx, uint32_t tid) {
        uint32_t v[P1A::E];
        const uint32_t d = P1A::dep(tid);
        load_global<P1A>(ctx, v, Mp::g1(d) + Mp::g1_rank(ctx.rank), G1{}, (int)G::W1);
        run_stages<G, P1A, Arith, true, false, true>(ctx, v, d);
        if constexpr (G::K1B > 0) {
            store_smem<P1A>(ctx, v, d);
        } else {
            ctx.after_local_reads();
            ctx.before_scatter();
            scatter<P1A>(ctx, v, d);
        }
    }
    NTT_HD static void pass1b(Ctx& ctx, uint32_t tid) {
        uint32_t v[P1B::E];
        const uint32_t d = P1B::dep(tid);
        load_smem<P1B>(ctx, v, d);
        ctx.after_local_reads();
        run_stages<G, P1B, Arith, true, false, false>(ctx, v, d);
        ctx.before_scatter();
        scatter<P1B>(ctx, v, d);
    }
    NTT_HD static void pass2a(Ctx& ctx, uint32_t tid) {
        uint32_t v[P2A::E];
        const uint32_t d = P2A::dep(tid);
        load_smem<P2A>(ctx, v, d);
        run_stages<G, P2A, Arith, true, true, false>(ctx, v, d);
        if constexpr (G::K2B > 0) {
            store_smem<P2A>(ctx, v, d);
        } else {
            store_global<P2A>(ctx, v, d + ctx.rank * G::M, G2{}, 1 << 30,
                              FwdFinal<Arith>{ctx.q, ctx.q2});
        }
    }
    NTT_HD static void pass2b(Ctx& ctx, uint32_t tid) {
        uint32_t v[P2B::E];
        const uint32_t d = P2B::dep(tid);
        load_smem<P2B>(ctx, v, d);
        run_stages<G, P2B, Arith, true, true, false>(ctx, v, d);
        store_global<P2B>(ctx, v, d + ctx.rank * G::M, G2{}, 1 << 30,
                          FwdFinal<Arith>{ctx.q, ctx.q2});
    }
};

template <class G, class Arith, class Ctx>
struct Inverse {
    using Mp = Maps<G>;
    using P1A = typename G::P1A;
    using P1B = typename G::P1B;
    using P2A = typename G::P2A;
    using P2B = typename G::P2B;

    struct G1 {
        NTT_HD uint32_t operator()(uint32_t o) const { return Maps<G>::g1(o); }
    };
    struct G2 {
        NTT_HD uint32_t operator()(uint32_t o) const { return o; }
    };

    template <class L>
    NTT_HD static void scatter(Ctx& ctx, uint32_t (&v)[L::E], uint32_t d) {
        const uint32_t dd = Mp::i_dst(d);
        const uint32_t dl = Mp::i_lam(d) + Mp::i_lam_rank(ctx.rank);
#pragma unroll
        for (int r = 0; r < L::E; ++r) {
            const uint32_t o = L::off(r);
            ctx.rstore(dd + Mp::i_dst(o), smem_phys(dl + Mp::i_lam(o)), v[r]);
        }
    }

    // Inverse order of passes: P2B (low column bits), P2A, scatter, P1B, P1A.
    // The first pass reads the contiguous phase-2 slab from global.
    template <class L, bool Last>
    NTT_HD static void phase2_pass(Ctx& ctx, uint32_t tid, bool from_global) {
        uint32_t v[L::E];
        const uint32_t d = L::dep(tid);
        if (from_global)
            load_global<L>(ctx, v, d + ctx.rank * G::M, G2{}, 1 << 30);
        else
            load_smem<L>(ctx, v, d);
        if (Last) ctx.after_local_reads();
        run_stages<G, L, Arith, false, true, false>(ctx, v, d);
        if (Last) {
            ctx.before_scatter();
            scatter<L>(ctx, v, d);
        } else {
            store_smem<L>(ctx, v, d);
        }
    }
    NTT_HD static void pass2b(Ctx& ctx, uint32_t tid) {
        if constexpr (G::K2B > 0) phase2_pass<P2B, false>(ctx, tid, true);
    }
    NTT_HD static void pass2a(Ctx& ctx, uint32_t tid) {
        phase2_pass<P2A, true>(ctx, tid, G::K2B == 0);
    }
    NTT_HD static void pass1b(Ctx& ctx, uint32_t tid) {
        if constexpr (G::K1B > 0) {
            uint32_t v[P1B::E];
            const uint32_t d = P1B::dep(tid);
            load_smem<P1B>(ctx, v, d);
            run_stages<G, P1B, Arith, false, false, false>(ctx, v, d);
            store_smem<P1B>(ctx, v, d);
        }
    }
    // Last pass: contains global stage 0 (fold N^{-1} R^{-1}), canonical
    // output to the phase-1 slab in global memory.
    NTT_HD static void pass1a(Ctx& ctx, uint32_t tid) {
        uint32_t v[P1A::E];
        const uint32_t d = P1A::dep(tid);
        load_smem<P1A>(ctx, v, d);
        run_stages<G, P1A, Arith, false, false, true>(ctx, v, d);
        store_global<P1A>(ctx, v, Mp::g1(d) + Mp::g1_rank(ctx.rank), G1{}, (int)G::W1,
                          Ident{});
    }
};

}  // namespace nttb
