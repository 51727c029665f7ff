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
// [PLO, PLO+KB), plus EB-KB "extra" bits (the lowest free positions, so each
// thread's words form contiguous runs for 128-bit accesses), the remaining
// bits being the lane and warp index.  All index maps below are linear over
// disjoint bit sets, so every per-register address is a per-thread base plus
// a compile-time constant, and every loop over registers, stages and groups
// is a compile-time loop (ct_for), so no index arithmetic runs per element.
#pragma once
#include <type_traits>
#include <utility>

#include "arith.cuh"
#include "layouts_gen.h"

namespace nttb {

// ---------------------------------------------------------------------------
// Compile-time loops: f(std::integral_constant<int, I>) for I = 0..N-1.
// ---------------------------------------------------------------------------
template <class F, int... Is>
NTT_HD void ct_for_impl(F&& f, std::integer_sequence<int, Is...>) {
    (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F>
NTT_HD void ct_for(F&& f) {
    ct_for_impl(f, std::make_integer_sequence<int, N>{});
}

constexpr int popcount32(uint32_t x) {
    int c = 0;
    for (; x; x &= x - 1u) ++c;
    return c;
}

// ---------------------------------------------------------------------------
// Compile-time layout of one register pass.
// WM: lambda positions of the warp index (0 = no constraint: the thread
// index fills all non-register positions in ascending order).  Two passes
// with the same WM give every warp the same element set, so the exchange
// between them needs only a warp barrier.
// ---------------------------------------------------------------------------
template <int MB_, int PLO_, int KB_, int EB_, uint32_t WM_ = 0>
struct PassLayout {
    static constexpr int MB = MB_, PLO = PLO_, KB = KB_, EB = EB_;
    static constexpr uint32_t WM = WM_;
    static constexpr int XB = EB - KB;
    static constexpr int E = 1 << EB;
    static_assert(KB >= 1 && KB <= EB && EB <= MB, "bad pass layout");
    static_assert(PLO >= 0 && PLO + KB <= MB, "bad pass layout");

    static constexpr bool in_bfly(int p) { return p >= PLO && p < PLO + KB; }
    // j-th extra position: the XB lowest positions outside the butterfly
    // range and the warp positions.
    static constexpr int xpos(int j) {
        int cnt = 0;
        for (int p = 0; p < MB; ++p) {
            if (in_bfly(p) || ((WM >> p) & 1u)) continue;
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
    static constexpr uint32_t kRegMask = reg_mask();
    static_assert((kRegMask & WM) == 0, "warp positions overlap register positions");
    static constexpr int kRunBits = run_bits();
    static constexpr int kXHB = xhi_bits();
    static constexpr uint32_t kFull = (MB >= 32) ? 0xFFFFFFFFu : ((1u << MB) - 1u);
    static constexpr uint32_t kLaneMask = kFull & ~kRegMask & ~WM;
    // the 5 lambda positions that hold the lane index (tid bits 0..4)
    static constexpr uint32_t lanes() {
        uint32_t m = (WM == 0) ? (kFull & ~kRegMask) : kLaneMask, out = 0;
        for (int p = 0, c = 0; p < MB && c < 5; ++p)
            if ((m >> p) & 1u) {
                out |= 1u << p;
                ++c;
            }
        return out;
    }
    static constexpr uint32_t kLanes = lanes();
    // Deposit the bits of x into the set positions of Mask (ascending).
    template <uint32_t Mask>
    NTT_HD static uint32_t deposit(uint32_t x) {
        uint32_t v = 0;
        ct_for<MB>([&](auto P) {
            constexpr int p = decltype(P)::value;
            if constexpr (((Mask >> p) & 1u) != 0) {
                constexpr int rank = popcount32(Mask & ((1u << p) - 1u));
                v |= ((x >> rank) & 1u) << p;
            }
        });
        return v;
    }
    // lambda bits owned by thread t (its register offsets are added to this)
    NTT_HD static uint32_t dep(uint32_t t) {
        if constexpr (WM == 0) {
            return deposit<kFull & ~kRegMask>(t);
        } else {
            return deposit<kLaneMask>(t & 31u) | deposit<WM>(t >> 5);
        }
    }
};

// A register pass whose extra (non-butterfly) register bits are given
// explicitly (XM) instead of being the lowest free positions; the lane
// index fills the 5 lowest remaining positions and the warp index the rest.
// Used where a pass reads global memory and its lanes must cover 32
// consecutive words (a 128-byte line per warp instruction).
template <int MB_, int PLO_, int KB_, int EB_, uint32_t XM_>
struct PassLayoutX {
    static constexpr int MB = MB_, PLO = PLO_, KB = KB_, EB = EB_;
    static constexpr int XB = EB - KB;
    static constexpr int E = 1 << EB;
    static_assert(KB >= 1 && KB <= EB && EB <= MB && PLO + KB <= MB, "bad pass layout");
    static_assert(popcount32(XM_) == XB, "one extra mask bit per extra register bit");
    static constexpr int xpos(int j) {
        for (int p = 0, c = 0; p < MB; ++p)
            if ((XM_ >> p) & 1u) {
                if (c == j) return p;
                ++c;
            }
        return -1;
    }
    static constexpr uint32_t reg_mask() {
        uint32_t m = XM_;
        for (int p = PLO; p < PLO + KB; ++p) m |= 1u << p;
        return m;
    }
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
    static constexpr int run_bits() {
        int v = 0;
        while (v < MB && ((reg_mask() >> v) & 1u)) ++v;
        return v;
    }
    static constexpr int xhi_bits() {
        int c = 0;
        for (int j = 0; j < XB; ++j)
            if (xpos(j) > PLO + KB - 1) ++c;
        return c;
    }
    static constexpr uint32_t kRegMask = reg_mask();
    static_assert((kRegMask & ~((MB >= 32) ? 0xFFFFFFFFu : ((1u << MB) - 1u))) == 0, "bits");
    static constexpr int kRunBits = run_bits();
    static constexpr int kXHB = xhi_bits();
    static constexpr uint32_t kFull = (MB >= 32) ? 0xFFFFFFFFu : ((1u << MB) - 1u);
    static constexpr uint32_t lanes() {
        const uint32_t m = kFull & ~kRegMask;
        uint32_t out = 0;
        for (int p = 0, c = 0; p < MB && c < 5; ++p)
            if ((m >> p) & 1u) {
                out |= 1u << p;
                ++c;
            }
        return out;
    }
    static constexpr uint32_t kLanes = lanes();
    static constexpr uint32_t WM = kFull & ~kRegMask & ~kLanes;
    template <uint32_t Mask>
    NTT_HD static uint32_t deposit(uint32_t x) {
        uint32_t v = 0;
        ct_for<MB>([&](auto P) {
            constexpr int p = decltype(P)::value;
            if constexpr (((Mask >> p) & 1u) != 0) {
                constexpr int rank = popcount32(Mask & ((1u << p) - 1u));
                v |= ((x >> rank) & 1u) << p;
            }
        });
        return v;
    }
    NTT_HD static uint32_t dep(uint32_t t) { return deposit<kLanes>(t & 31u) | deposit<WM>(t >> 5); }
};

// Lambda positions of the warp index of a pass layout (either kind).
template <class L>
constexpr uint32_t warp_bits() {
    return L::kFull & ~L::kRegMask & ~L::kLanes;
}

// ---------------------------------------------------------------------------
// Shared-memory layouts.  The work buffer uses one bank-spreading layout
//     phys(l) = l + C1 * (l >> A1) + C2 * (l >> A2)
// per configuration, which is monotone (so injective) and additive over
// disjoint bit sets (so a thread's addresses stay base + compile-time
// offset).  It is the same for every pass because each pass rewrites, in
// place, exactly the words it read.  A1..C2 are chosen offline by
// gen_layouts.py (layouts_gen.h) to minimise warp-wide bank conflicts of all
// the passes' lane patterns.
// ---------------------------------------------------------------------------
template <int A1, int C1, int A2, int C2>
struct Spread {
    static constexpr uint32_t phys(uint32_t l) {
        return l + (uint32_t)C1 * (l >> A1) + (uint32_t)C2 * (l >> A2);
    }
    // every aligned run of V lambdas maps to an aligned run of V words
    template <int V>
    static constexpr bool aligned() {
        return C1 % V == 0 && C2 % V == 0 && (C1 == 0 || (1 << A1) % V == 0) &&
               (C2 == 0 || (1 << A2) % V == 0);
    }
};

// Width (words) of a pass's shared-memory accesses: 128-bit when the thread
// owns runs of 4 consecutive lambdas and the layout keeps them aligned, else
// 64-bit for runs of 2, else 32-bit (gen_layouts.py's vec_width).
template <class L, class X>
constexpr int smem_vec() {
    if constexpr (L::kRunBits >= 2 && X::template aligned<4>()) return 4;
    else if constexpr (L::kRunBits >= 1 && X::template aligned<2>()) return 2;
    else return 1;
}

// Stage buffer: one 16-byte pad per 128 bytes (conflict-free 128-bit reads
// whether a thread's run starts every 32 words or every row).
struct StageLayout {
    static constexpr uint32_t phys(uint32_t l) { return l + 4u * (l >> 5); }
};

// ---------------------------------------------------------------------------
// Geometry of one fused transform configuration.
//   LOGN: n;  CLOG: c (cluster of 2^c CTAs);  R1: phase-1 stages;
//   EB: log2 words per thread per pass;  K1A / K2A: stages of the first
//   register pass of phase 1 / phase 2 (the rest, if any, is a second pass).
// ---------------------------------------------------------------------------
template <int LOGN_, int CLOG_, int R1_, int EB_, int K1A_, int K2A_, int NP_ = 1>
struct Geometry {
    static constexpr int LOGN = LOGN_, CLOG = CLOG_, R1 = R1_, EB = EB_;
    static constexpr int NP = NP_;  // polynomials per job (same limb, same twiddles)
    static constexpr int R2 = LOGN - R1;
    static constexpr int C = 1 << CLOG;
    static constexpr int MB = LOGN - CLOG;  // local bits
    static constexpr uint32_t M = 1u << MB;
    static constexpr int S1 = R2 - CLOG;  // log2 W1
    static constexpr uint32_t W1 = 1u << S1;
    static constexpr uint32_t H2 = 1u << (R1 - CLOG);
    static constexpr int TB = MB - EB;
    static constexpr int THREADS = 1 << TB;
    // Register budget: the transforms are latency-bound and gain more from
    // resident warps than from per-thread ILP (measured on B200: 5 CTAs of
    // 256 threads at 48 registers beat 4 at 64 and 3 at 85), so ask for as
    // many resident CTAs as leave each thread its NP * 2^EB data words plus
    // 16 registers, and at least 40.
    // (24 spare registers with several polynomials per job: each keeps a
    // global base pointer of its own, and 16 spare registers spilled)
    static constexpr int REG_SPARE = NP > 1 ? 24 : 16;
    static constexpr int REG_BUDGET =
        NP * (1 << EB_) + REG_SPARE > 40 ? NP * (1 << EB_) + REG_SPARE : 40;
    static constexpr int MIN_BLOCKS =
        (65536 / (THREADS * REG_BUDGET)) > 0 ? (65536 / (THREADS * REG_BUDGET)) : 1;
    static constexpr int K1A = K1A_, K1B = R1 - K1A_;
    static constexpr int K2A = K2A_, K2B = R2 - K2A_;
    static_assert(R1 >= CLOG && R2 >= CLOG, "each phase needs at least c stages");
    static_assert(K1A >= 1 && K1A <= EB && K1B >= 0 && K1B <= EB, "phase-1 passes");
    static_assert(K2A >= 1 && K2A <= EB && K2B >= 0 && K2B <= EB, "phase-2 passes");
    static_assert(TB >= 5 && TB <= 10, "32..1024 threads per CTA");
    static_assert(LOGN < kTwPermMinLogN || R2 >= kTwPermStages,
                  "the interleaved twiddle stages must all lie in phase 2");

    // Bulk copies of the input slab in pieces of COPY_WORDS (<= 128 bytes, so
    // a piece never straddles a stage pad): forward = each phase-1 row's W1
    // words owned by this CTA; inverse = the contiguous phase-2 slab.
    static constexpr uint32_t COPY_WORDS = W1 < 32u ? W1 : 32u;
    static constexpr uint32_t FWD_COPIES = (1u << R1) * (W1 / COPY_WORDS);
    static constexpr uint32_t INV_COPIES = M / 32u;
    static constexpr uint32_t STAGE_WORDS = StageLayout::phys(M - 1u) + 1u;

    // Warp ownership.  Phase 2: the warp index sits on the top WB row bits,
    // so both register passes of phase 2 see the same elements per warp and
    // exchange through a warp barrier.  Phase 1 keeps a CTA barrier: every
    // row bit is a butterfly bit of one of its passes, so a warp-owned layout
    // would have to put the lanes on rows and break the coalescing of the
    // strided phase-1 global accesses.
    static constexpr int WB = TB - 5;
    static constexpr bool WARP1 = false;
    static constexpr bool WARP2 = K2B > 0 && (R1 - CLOG) >= WB;
    static constexpr uint32_t WM1 = 0u;
    static constexpr uint32_t WM2 = WARP2 ? (((1u << WB) - 1u) << (MB - WB)) : 0u;

    // Pass layouts (forward order).  Phase-1 lambda bits: [S1, MB) (row bits),
    // processed top-down; phase-2 bits [0, R2) (column bits), top-down.
    using P1A = PassLayout<MB, MB - K1A, K1A, EB, WM1>;
    using P1B = PassLayout<MB, S1, (K1B > 0 ? K1B : 1), EB, WM1>;
    using P2A = PassLayout<MB, R2 - K2A, K2A, EB, WM2>;
    using P2B = PassLayout<MB, 0, (K2B > 0 ? K2B : 1), EB, WM2>;

    // Work-buffer layout (chosen offline; the lane patterns it was chosen
    // for must be the ones these pass layouts produce).
    using LT = LayoutTable<LOGN, CLOG, R1, EB, K1A, K2A>;
    static_assert(LT::lanes_P1A == P1A::kLanes && LT::lanes_P1B == P1B::kLanes &&
                      LT::lanes_P2A == P2A::kLanes && LT::lanes_P2B == P2B::kLanes,
                  "layouts_gen.h is stale: rerun gen_layouts.py");
    using XW = Spread<LT::XW[0], LT::XW[1], LT::XW[2], LT::XW[3]>;
    // one slab of the layout per polynomial of the job
    static constexpr uint32_t SLAB_WORDS = ((uint32_t)LT::XW[4] + 3u) & ~3u;
    static constexpr uint32_t SMEM_WORDS = NP * SLAB_WORDS;
    // dynamic shared memory: work buffer | stage buffer | mbarrier
    static constexpr uint32_t STAGE_OFF_WORDS = SMEM_WORDS;
    static constexpr uint32_t MBAR_OFF_WORDS = (STAGE_OFF_WORDS + STAGE_WORDS + 3u) & ~3u;
    static constexpr uint32_t SMEM_BYTES = (MBAR_OFF_WORDS + 4u) * 4u;  // staged
    static constexpr uint32_t SMEM_BYTES_DIRECT = SMEM_WORDS * 4u;        // direct
};

// Bulk copy `i` of the input slab of CTA `rank`: word offset in the limb,
// word offset in the stage buffer, and length in words.  Forward: the
// phase-1 slab (row rho of the CTA's column range at lambda1 = rho * W1 +
// kappa'); inverse: the contiguous phase-2 slab [rank*M, (rank+1)*M).  The
// stage buffer holds lambda at StageLayout::phys(lambda).
struct SlabCopy {
    uint32_t src, dst, words;
};
template <class G, bool Fwd>
NTT_HD SlabCopy slab_copy(uint32_t rank, uint32_t i) {
    if constexpr (Fwd) {
        constexpr uint32_t per_row = G::W1 / G::COPY_WORDS;
        const uint32_t row = i / per_row, piece = (i % per_row) * G::COPY_WORDS;
        return SlabCopy{(row << G::R2) + rank * G::W1 + piece,
                        StageLayout::phys(row * G::W1 + piece), G::COPY_WORDS};
    } else {
        return SlabCopy{rank * G::M + 32u * i, StageLayout::phys(32u * i), 32u};
    }
}
template <class G, bool Fwd>
NTT_HD constexpr uint32_t slab_copies() {
    return Fwd ? G::FWD_COPIES : G::INV_COPIES;
}

// lambda maps (see file header); all linear over disjoint bit sets.
template <class G>
struct Maps {
    // phase-1 slab lambda -> word offset in the limb (without the rank term)
    NTT_HD static uint32_t g1(uint32_t lam) {
        return ((lam >> G::S1) << G::R2) + (lam & (G::W1 - 1u));
    }
    NTT_HD static uint32_t g1_rank(uint32_t rank) { return rank * G::W1; }
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

// Whether a memory context reads compressed twiddle tables (tw_comp_*,
// arith.cuh): Ctx::kCompTw when the context declares it, else false.
template <class Ctx, class = void>
struct CompTw : std::false_type {};
template <class Ctx>
struct CompTw<Ctx, std::void_t<decltype(Ctx::kCompTw)>> : std::bool_constant<Ctx::kCompTw> {};

// Stage k of a pass.  CT (Fwd): acts on lambda bit p = PLO + KB - 1 - k,
// groups = top k butterfly-coordinate bits.  GS: bit p = PLO + k, groups =
// top KB-1-k butterfly bits.  `tbase` is the twiddle index of group 0 for
// this thread; group g of extra-high coordinate xh uses tbase + xoff(xh) + g.
// Fold: the limb's stage 0 (one twiddle, index 1) with the factor in entry 0.
// v[p][r]: register r of polynomial p; every twiddle loaded once serves the
// same butterfly of all NP polynomials of the job.
// Perm != 0: the stage's twiddle block (starting at index H) is stored
// interleaved by Perm (tw_slot, arith.cuh): entry H + j at slot
// H + (j % Perm) * S + j / Perm.  With compressed tables (CompTw<Ctx>) the
// table holds only the slots of j % Perm == 0 (the base block, at
// (log2 Perm + 1) * S) and the 16 factors L (at 6 S): entry H + j is
// base[j / Perm] * L[j % Perm].
template <class L, class Arith, bool Fwd, int k, bool Fold, int NP, int Perm = 0,
          uint32_t H = 0, uint32_t S = 0, class Ctx>
NTT_HD void stage(Ctx& ctx, uint32_t (&v)[NP][L::E], uint32_t tbase) {
    constexpr int p = Fwd ? (L::PLO + L::KB - 1 - k) : (L::PLO + k);
    constexpr int gbits = Fwd ? k : (L::KB - 1 - k);
    constexpr int bbit = Fwd ? (L::KB - 1 - k) : k;  // butterfly coordinate bit
    constexpr int stride = 1 << (bbit + L::XB);      // register distance
    constexpr int XHB = L::kXHB;
    constexpr int XLB = L::XB - XHB;
    const uint32_t q = ctx.q, q2 = ctx.q2;
    if constexpr (Fold) {
        static_assert(gbits == 0, "stage 0 of the limb has a single group");
        const TwPair f = ctx.fold_at(0u), w = ctx.fold_at(1u);
        ct_for<(L::E >> 1)>([&](auto I) {
            constexpr int i = decltype(I)::value;
            // the E/2 pairs: the lower register has bit (bbit + XB) clear
            constexpr int r = ((i >> (bbit + L::XB)) << (bbit + L::XB + 1)) | (i & (stride - 1));
            ct_for<NP>([&](auto Pp) {
                constexpr int pp = decltype(Pp)::value;
                if constexpr (Fwd) Arith::ct_first(v[pp][r], v[pp][r + stride], f, w, q, q2);
                else Arith::gs_last(v[pp][r], v[pp][r + stride], f, w, q, q2);
            });
        });
    } else {
        ct_for<(1 << XHB)>([&](auto XH) {
            constexpr int xh = decltype(XH)::value;
            constexpr uint32_t xoff = L::off(xh << XLB) >> (p + 1);
            // twiddles of this stage for this xh: 2^gbits consecutive entries
            // (compressed: w holds the base factor and wl the unit-step one)
            TwPair w[1 << gbits];
            constexpr bool kComp = Perm != 0 && CompTw<Ctx>::value;
            [[maybe_unused]] TwPair wl[kComp ? (1 << gbits) : 1] = {};
            [[maybe_unused]] constexpr int lpc = Perm == 16 ? 4 : Perm == 8 ? 3 : Perm == 4 ? 2 : 1;
            constexpr bool kAlignedC =
                Perm != 0 &&
                ((L::kRegMask >> (p + 1)) & (uint32_t)(Perm - 1)) == (uint32_t)(Perm - 1);
            if constexpr (kComp) {
                constexpr uint32_t CB = (uint32_t)(lpc + 1) * S, LB = 6u * S;
                const uint32_t j0 = tbase - H;
                if constexpr (kAlignedC) {
                    auto tb = ctx.tw_base(CB + (j0 >> lpc));
                    ct_for<(1 << gbits)>([&](auto Gc) {
                        constexpr uint32_t c = xoff + decltype(Gc)::value;
                        w[decltype(Gc)::value] = ctx.tw_ld(tb, c >> lpc);
                        if constexpr ((c & (uint32_t)(Perm - 1)) != 0)
                            wl[decltype(Gc)::value] = ctx.tw_at(LB + (c & (uint32_t)(Perm - 1)));
                    });
                } else {
                    ct_for<(1 << gbits)>([&](auto Gc) {
                        const uint32_t j = j0 + xoff + decltype(Gc)::value;
                        w[decltype(Gc)::value] = ctx.tw_at(CB + (j >> lpc));
                        wl[decltype(Gc)::value] = ctx.tw_at(LB + (j & (uint32_t)(Perm - 1)));
                    });
                }
            } else if constexpr (Perm == 0) {
                auto tb = ctx.tw_base(tbase + xoff);
                if constexpr (gbits >= 1) {
                    ct_for<(1 << (gbits - 1))>([&](auto G2) {
                        constexpr int g2 = decltype(G2)::value;
                        ctx.tw_ld2(tb, 2 * g2, w[2 * g2], w[2 * g2 + 1]);
                    });
                } else {
                    w[0] = ctx.tw_ld(tb, 0);
                }
            } else {
                constexpr int lp = Perm == 16 ? 4 : Perm == 8 ? 3 : Perm == 4 ? 2 : 1;
                // the thread's part of the entry index, j0 = tbase - H, is a
                // multiple of Perm when the lambda bits p+1 .. p+lp are
                // register bits (zero in the thread's base): then the slot of
                // entry j0 + c is (H + j0 / Perm) + a compile-time offset
                constexpr bool kAligned =
                    ((L::kRegMask >> (p + 1)) & (uint32_t)(Perm - 1)) == (uint32_t)(Perm - 1);
                const uint32_t j0 = tbase - H;
                if constexpr (kAligned) {
                    auto tb = ctx.tw_base(H + (j0 >> lp));
                    ct_for<(1 << gbits)>([&](auto Gc) {
                        constexpr uint32_t c = xoff + decltype(Gc)::value;
                        w[decltype(Gc)::value] =
                            ctx.tw_ld(tb, (c & (uint32_t)(Perm - 1)) * S + (c >> lp));
                    });
                } else {
                    ct_for<(1 << gbits)>([&](auto Gc) {
                        const uint32_t j = j0 + xoff + decltype(Gc)::value;
                        w[decltype(Gc)::value] =
                            ctx.tw_at(H + (j & (uint32_t)(Perm - 1)) * S + (j >> lp));
                    });
                }
            }
            ct_for<(1 << gbits)>([&](auto Gc) {
                constexpr int g = decltype(Gc)::value;
                // group g needs the second factor (its unit-step index is
                // known at compile time in the aligned case; L[0] = 1)
                constexpr bool kTwo =
                    kComp && (!kAlignedC || ((xoff + (uint32_t)g) & (uint32_t)(Perm - 1)) != 0);
                ct_for<(1 << bbit)>([&](auto LO) {
                    constexpr int lo = decltype(LO)::value;
                    ct_for<(1 << XLB)>([&](auto XL) {
                        constexpr int xl = decltype(XL)::value;
                        constexpr int bc = (g << (bbit + 1)) | lo;
                        constexpr int r = (bc << L::XB) | (xh << XLB) | xl;
                        ct_for<NP>([&](auto Pp) {
                            constexpr int pp = decltype(Pp)::value;
                            if constexpr (kTwo) {
                                if constexpr (Fwd)
                                    Arith::ct2(v[pp][r], v[pp][r + stride], w[g], wl[g], q, q2);
                                else
                                    Arith::gs2(v[pp][r], v[pp][r + stride], w[g], wl[g], q, q2);
                            } else if constexpr (Fwd) {
                                Arith::ct(v[pp][r], v[pp][r + stride], w[g].w, w[g].wp, q, q2);
                            } else {
                                Arith::gs(v[pp][r], v[pp][r + stride], w[g].w, w[g].wp, q, q2);
                            }
                        });
                    });
                });
            });
        });
    }
}

// Run all KB stages of a pass.  Phase2 selects the twiddle base rule;
// HasStage0: this pass contains the limb's stage 0 (the forward's first
// stage / the inverse's last), which gets the Montgomery / N^{-1} fold.
// ArriveAfterFirst: signal the cluster (relaxed arrive) once stage 0 has
// consumed every loaded word -- this thread has finished reading its shared
// memory -- so the wait before the scatter overlaps the remaining stages.
template <class G, class L, class Arith, bool Fwd, bool Phase2, bool HasStage0,
          bool ArriveAfterFirst = false, class Ctx>
NTT_HD void run_stages(Ctx& ctx, uint32_t (&v)[G::NP][L::E], uint32_t d) {
    using Mp = Maps<G>;
    ct_for<L::KB>([&](auto K) {
        constexpr int k = decltype(K)::value;
        constexpr int p = Fwd ? (L::PLO + L::KB - 1 - k) : (L::PLO + k);
        constexpr bool s0 = HasStage0 && (Fwd ? (k == 0) : (k == L::KB - 1));
        const uint32_t tb =
            (Phase2 ? Mp::tw_base_p2(p, ctx.rank) : Mp::tw_base_p1(p)) + (d >> (p + 1));
        // phase-2 bit p < 4 is the limb's stage logN-1-p, whose twiddles are
        // stored interleaved by 16 >> p (tw_slot)
        constexpr bool kPermLayout =
            Phase2 && G::LOGN >= kTwPermMinLogN && p < kTwPermStages;
        constexpr int perm = kPermLayout ? (16 >> p) : 0;
        constexpr uint32_t h = kPermLayout ? (1u << (G::LOGN - 1 - p)) : 0u;
        constexpr uint32_t s32 = kPermLayout ? (1u << (G::LOGN - 5)) : 0u;
        stage<L, Arith, Fwd, k, s0, G::NP, perm, h, s32>(ctx, v, tb);
        if constexpr (ArriveAfterFirst && k == 0) ctx.after_local_reads();
    });
}

// ---------------------------------------------------------------------------
// Loads / stores of a pass's registers.  Every address is a per-thread base
// plus a compile-time constant (an immediate offset on the device).
// ---------------------------------------------------------------------------

// 16-byte vectors when the thread owns >= 4 consecutive lambdas and the
// address map keeps runs of `Lim` consecutive lambdas contiguous.
template <class L, uint32_t Lim>
constexpr bool use_vec4() {
    return L::kRunBits >= 2 && Lim >= 4;
}

// GMap::map(o): word offset of register offset o (linear, no base term).
// Polynomial p of the job has its own global base (ctx.g_base(p, ...)).
template <class L, uint32_t Lim, class GMap, int NP, class Ctx>
NTT_HD void load_global(Ctx& ctx, uint32_t (&v)[NP][L::E], uint32_t gbase) {
    ct_for<NP>([&](auto Pp) {
        constexpr int pp = decltype(Pp)::value;
        auto gb = ctx.g_base(pp, gbase);
        if constexpr (use_vec4<L, Lim>()) {
            ct_for<L::E>([&](auto R) {
                constexpr int r = decltype(R)::value;
                constexpr uint32_t o = L::off(r);
                if constexpr ((o & 3u) == 0) {
                    ctx.g_ld4(gb, GMap::map(o), v[pp][L::reg_of(o)], v[pp][L::reg_of(o + 1)],
                              v[pp][L::reg_of(o + 2)], v[pp][L::reg_of(o + 3)]);
                }
            });
        } else {
            ct_for<L::E>([&](auto R) {
                constexpr int r = decltype(R)::value;
                v[pp][r] = ctx.g_ld(gb, GMap::map(L::off(r)));
            });
        }
    });
}

// The transform's output goes through the context's o_* interface (global
// memory for a plain transform; a fused caller may redirect it).
template <class L, uint32_t Lim, class GMap, int NP, class Ctx, class ValFn>
NTT_HD void store_global(Ctx& ctx, uint32_t (&v)[NP][L::E], uint32_t gbase, ValFn fin) {
    ct_for<NP>([&](auto Pp) {
        constexpr int pp = decltype(Pp)::value;
        auto gb = ctx.o_base(pp, gbase);
        if constexpr (use_vec4<L, Lim>()) {
            ct_for<L::E>([&](auto R) {
                constexpr int r = decltype(R)::value;
                constexpr uint32_t o = L::off(r);
                if constexpr ((o & 3u) == 0) {
                    ctx.o_st4(gb, GMap::map(o), fin(v[pp][L::reg_of(o)]),
                              fin(v[pp][L::reg_of(o + 1)]), fin(v[pp][L::reg_of(o + 2)]),
                              fin(v[pp][L::reg_of(o + 3)]));
                }
            });
        } else {
            ct_for<L::E>([&](auto R) {
                constexpr int r = decltype(R)::value;
                ctx.o_st(gb, GMap::map(L::off(r)), fin(v[pp][r]));
            });
        }
    });
}

// Stage buffer (the bulk-copied input slab; one polynomial per job).
template <class L, int NP, class Ctx>
NTT_HD void load_stage(Ctx& ctx, uint32_t (&v)[NP][L::E], uint32_t d) {
    static_assert(NP == 1, "the staged schedule carries one polynomial per job");
    auto sb = ctx.st_base(StageLayout::phys(d));
    if constexpr (L::kRunBits >= 2) {
        ct_for<L::E>([&](auto R) {
            constexpr int r = decltype(R)::value;
            constexpr uint32_t o = L::off(r);
            if constexpr ((o & 3u) == 0)
                ctx.st_ld4(sb, StageLayout::phys(o), v[0][L::reg_of(o)], v[0][L::reg_of(o + 1)],
                           v[0][L::reg_of(o + 2)], v[0][L::reg_of(o + 3)]);
        });
    } else {
        ct_for<L::E>([&](auto R) {
            constexpr int r = decltype(R)::value;
            v[0][r] = ctx.st_ld(sb, StageLayout::phys(L::off(r)));
        });
    }
}

// The input slab of a transform: from the stage buffer (bulk-copied ahead of
// time) or straight from global memory, as the context's kStaged says.
template <class L, uint32_t Lim, class GMap, int NP, class Ctx>
NTT_HD void load_input(Ctx& ctx, uint32_t (&v)[NP][L::E], uint32_t d, uint32_t gbase) {
    if constexpr (Ctx::kStaged)
        load_stage<L>(ctx, v, d);
    else
        load_global<L, Lim, GMap>(ctx, v, gbase);
}

// Work buffer: polynomial p's slab starts Slab words after polynomial 0's.
// The thread's base d is zero on its register bits, so with runs of V the
// base and every run start are multiples of V (and so are their words).
template <class L, class X, uint32_t Slab, int NP, class Ctx>
NTT_HD void load_smem(Ctx& ctx, uint32_t (&v)[NP][L::E], uint32_t d) {
    constexpr int V = smem_vec<L, X>();
    auto sb = ctx.s_base(X::phys(d));
    ct_for<L::E>([&](auto R) {
        constexpr int r = decltype(R)::value;
        constexpr uint32_t o = L::off(r);
        ct_for<NP>([&](auto Pp) {
            constexpr int pp = decltype(Pp)::value;
            constexpr uint32_t c = pp * Slab + X::phys(o);
            if constexpr (V == 1) {
                v[pp][r] = ctx.s_ld(sb, c);
            } else if constexpr ((o & (V - 1)) == 0) {
                if constexpr (V == 4)
                    ctx.s_ld4(sb, c, v[pp][L::reg_of(o)], v[pp][L::reg_of(o + 1)],
                              v[pp][L::reg_of(o + 2)], v[pp][L::reg_of(o + 3)]);
                else
                    ctx.s_ld2(sb, c, v[pp][L::reg_of(o)], v[pp][L::reg_of(o + 1)]);
            }
        });
    });
}

template <class L, class X, uint32_t Slab, int NP, class Ctx>
NTT_HD void store_smem(Ctx& ctx, uint32_t (&v)[NP][L::E], uint32_t d) {
    constexpr int V = smem_vec<L, X>();
    auto sb = ctx.s_base(X::phys(d));
    ct_for<L::E>([&](auto R) {
        constexpr int r = decltype(R)::value;
        constexpr uint32_t o = L::off(r);
        ct_for<NP>([&](auto Pp) {
            constexpr int pp = decltype(Pp)::value;
            constexpr uint32_t c = pp * Slab + X::phys(o);
            if constexpr (V == 1) {
                ctx.s_st(sb, c, v[pp][r]);
            } else if constexpr ((o & (V - 1)) == 0) {
                if constexpr (V == 4)
                    ctx.s_st4(sb, c, v[pp][L::reg_of(o)], v[pp][L::reg_of(o + 1)],
                              v[pp][L::reg_of(o + 2)], v[pp][L::reg_of(o + 3)]);
                else
                    ctx.s_st2(sb, c, v[pp][L::reg_of(o)], v[pp][L::reg_of(o + 1)]);
            }
        });
    });
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

// Global-offset maps of the two slab layouts (register-offset part).
template <class G>
struct G1Map {
    static constexpr uint32_t map(uint32_t o) {
        return ((o >> G::S1) << G::R2) + (o & (G::W1 - 1u));
    }
};
struct G2Map {
    static constexpr uint32_t map(uint32_t o) { return o; }
};

// Scatter maps (register-offset part), see Maps.
template <class G>
struct FDst {
    static constexpr uint32_t map(uint32_t o) { return o >> (G::MB - G::CLOG); }
};
template <class G>
struct FLam {
    static constexpr uint32_t map(uint32_t o) {
        return (((o >> G::S1) & (G::H2 - 1u)) << G::R2) + (o & (G::W1 - 1u));
    }
};
template <class G>
struct IDst {
    static constexpr uint32_t map(uint32_t o) { return (o & ((1u << G::R2) - 1u)) >> G::S1; }
};
template <class G>
struct ILam {
    static constexpr uint32_t map(uint32_t o) {
        return ((o >> G::R2) << G::S1) + (o & (G::W1 - 1u));
    }
};

// Scatter one pass's registers to their owners' shared memory (DSMEM when
// C > 1).  The destination word is phys(base) + phys(map(offset)).
template <class L, class X, uint32_t Slab, int NP, class Ctx, class DstF, class LamF>
NTT_HD void scatter_regs(Ctx& ctx, uint32_t (&v)[NP][L::E], uint32_t dd, uint32_t dl) {
    ct_for<L::E>([&](auto R) {
        constexpr int r = decltype(R)::value;
        constexpr uint32_t o = L::off(r);
        auto rb = ctx.r_base(dd + DstF::map(o), X::phys(dl));
        ct_for<NP>([&](auto Pp) {
            constexpr int pp = decltype(Pp)::value;
            ctx.template r_st<pp * Slab + X::phys(LamF::map(o))>(rb, v[pp][r]);
        });
    });
}

// The contiguous phase-2 slab [rank*M, (rank+1)*M) of the limb moves between
// global memory and the work buffer in warp chunks: warp w owns the
// M / warps consecutive words from w * M / warps (exactly its elements in the
// phase-2 register passes when they are warp-owned), and lane l moves words
// l, l + 32, l + 64, ... of the chunk, so every warp instruction touches one
// 128-byte line.  A register pass's own accesses would put each lane on its
// own line (a thread holds runs of consecutive words), which costs the L1
// pipe 32 wavefronts per instruction instead of one to four.
// With a layout that keeps 4-word runs aligned, lane l moves the 16-byte
// pieces 4l, 4l + 128, ... instead (one line per quarter warp).
template <class G>
struct SlabChunk {
    static constexpr uint32_t WARPS = G::THREADS / 32u;
    static constexpr uint32_t WORDS = G::M / WARPS;
    static constexpr bool VEC = G::XW::template aligned<4>();
    static constexpr uint32_t STEP = VEC ? 128u : 32u;  // words per warp step
    static_assert(WORDS % STEP == 0, "warp chunks of whole lines");
    // lambda of this lane's first word (bit-disjoint from the per-step
    // offsets STEP * i, so phys() splits into base + immediate)
    NTT_HD static uint32_t base(uint32_t tid) {
        return (tid >> 5) * WORDS + (VEC ? 4u : 1u) * (tid & 31u);
    }
};

// Work buffer -> global: the slab's canonical words, stored through the
// context's o_* interface (plain store, or the product epilogue).
template <class G, class X, class Ctx>
NTT_HD void slab_out(Ctx& ctx, uint32_t tid) {
    using SC = SlabChunk<G>;
    const uint32_t b = SC::base(tid);
    auto sb = ctx.s_base(X::phys(b));
    ct_for<G::NP>([&](auto Pp) {
        constexpr int pp = decltype(Pp)::value;
        auto gb = ctx.o_base(pp, b + ctx.rank * G::M);
        ct_for<SC::WORDS / SC::STEP>([&](auto I) {
            constexpr uint32_t o = SC::STEP * decltype(I)::value;
            constexpr uint32_t c = pp * G::SLAB_WORDS + X::phys(o);
            if constexpr (SC::VEC) {
                uint32_t x, y, z, w;
                ctx.s_ld4(sb, c, x, y, z, w);
                ctx.o_st4(gb, o, x, y, z, w);
            } else {
                ctx.o_st(gb, o, ctx.s_ld(sb, c));
            }
        });
    });
}

// Global -> work buffer: the inverse's input slab.
template <class G, class X, class Ctx>
NTT_HD void slab_in(Ctx& ctx, uint32_t tid) {
    using SC = SlabChunk<G>;
    constexpr uint32_t K = SC::WORDS / SC::STEP, V = SC::VEC ? 4u : 1u;
    const uint32_t b = SC::base(tid);
    auto sb = ctx.s_base(X::phys(b));
    ct_for<G::NP>([&](auto Pp) {
        constexpr int pp = decltype(Pp)::value;
        auto gb = ctx.g_base(pp, b + ctx.rank * G::M);
        uint32_t w[K * V];
        ct_for<K>([&](auto I) {
            constexpr uint32_t i = decltype(I)::value;
            if constexpr (SC::VEC)
                ctx.g_ld4(gb, SC::STEP * i, w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
            else
                w[i] = ctx.g_ld(gb, SC::STEP * i);
        });
        ct_for<K>([&](auto I) {
            constexpr uint32_t i = decltype(I)::value;
            constexpr uint32_t c = pp * G::SLAB_WORDS + X::phys(SC::STEP * i);
            if constexpr (SC::VEC)
                ctx.s_st4(sb, c, w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
            else
                ctx.s_st(sb, c, w[i]);
        });
    });
}

template <class G, class Arith, class Ctx>
struct Forward {
    using Mp = Maps<G>;
    using X = typename G::XW;
    using P1A = typename G::P1A;
    using P1B = typename G::P1B;
    using P2A = typename G::P2A;
    using P2B = typename G::P2B;

    template <class L>
    NTT_HD static void scatter(Ctx& ctx, uint32_t (&v)[G::NP][L::E], uint32_t d) {
        scatter_regs<L, X, G::SLAB_WORDS, G::NP, Ctx, FDst<G>, FLam<G>>(ctx, v, Mp::f_dst(d),
                                                 Mp::f_lam(d) + Mp::g1_rank(ctx.rank));
    }

    // Phase-1 first pass: input slab (normal domain) -> stages incl. stage 0
    // -> work buffer (if a second phase-1 pass follows) or the scatter.
    NTT_HD static void pass1a(Ctx& ctx, uint32_t tid) {
        uint32_t v[G::NP][P1A::E];
        const uint32_t d = P1A::dep(tid);
        load_input<P1A, G::W1, G1Map<G>>(ctx, v, d, Mp::g1(d) + Mp::g1_rank(ctx.rank));
        run_stages<G, P1A, Arith, true, false, true, (G::K1B == 0)>(ctx, v, d);
        if constexpr (G::K1B > 0) {
            store_smem<P1A, X, G::SLAB_WORDS>(ctx, v, d);
        } else {
            ctx.before_scatter();
            scatter<P1A>(ctx, v, d);
        }
    }
    NTT_HD static void pass1b(Ctx& ctx, uint32_t tid) {
        if constexpr (G::K1B > 0) {
            uint32_t v[G::NP][P1B::E];
            const uint32_t d = P1B::dep(tid);
            load_smem<P1B, X, G::SLAB_WORDS>(ctx, v, d);
            run_stages<G, P1B, Arith, true, false, false, true>(ctx, v, d);
            ctx.before_scatter();
            scatter<P1B>(ctx, v, d);
        }
    }
    NTT_HD static void pass2a(Ctx& ctx, uint32_t tid) {
        uint32_t v[G::NP][P2A::E];
        const uint32_t d = P2A::dep(tid);
        load_smem<P2A, X, G::SLAB_WORDS>(ctx, v, d);
        run_stages<G, P2A, Arith, true, true, false>(ctx, v, d);
        if constexpr (G::K2B > 0) {
            store_smem<P2A, X, G::SLAB_WORDS>(ctx, v, d);
        } else {
            store_global<P2A, (1u << 30), G2Map>(ctx, v, d + ctx.rank * G::M,
                                                 FwdFinal<Arith>{ctx.q, ctx.q2});
        }
    }
    // With two phase-2 passes the last one writes its canonical words back
    // in place and pass2c stores the slab in warp chunks (SlabChunk).
    NTT_HD static void pass2b(Ctx& ctx, uint32_t tid) {
        if constexpr (G::K2B > 0) {
            uint32_t v[G::NP][P2B::E];
            const uint32_t d = P2B::dep(tid);
            load_smem<P2B, X, G::SLAB_WORDS>(ctx, v, d);
            run_stages<G, P2B, Arith, true, true, false>(ctx, v, d);
            const FwdFinal<Arith> fin{ctx.q, ctx.q2};
            ct_for<G::NP>([&](auto Pp) {
                ct_for<P2B::E>([&](auto R) {
                    v[decltype(Pp)::value][decltype(R)::value] =
                        fin(v[decltype(Pp)::value][decltype(R)::value]);
                });
            });
            store_smem<P2B, X, G::SLAB_WORDS>(ctx, v, d);
        }
    }
    // (after a barrier over pass2b's writes)
    NTT_HD static void pass2c(Ctx& ctx, uint32_t tid) {
        if constexpr (G::K2B > 0) slab_out<G, X>(ctx, tid);
    }
};

template <class G, class Arith, class Ctx>
struct Inverse {
    using Mp = Maps<G>;
    using X = typename G::XW;
    using P1A = typename G::P1A;
    using P1B = typename G::P1B;
    using P2A = typename G::P2A;
    using P2B = typename G::P2B;

    template <class L>
    NTT_HD static void scatter(Ctx& ctx, uint32_t (&v)[G::NP][L::E], uint32_t d) {
        scatter_regs<L, X, G::SLAB_WORDS, G::NP, Ctx, IDst<G>, ILam<G>>(ctx, v, Mp::i_dst(d),
                                                 Mp::i_lam(d) + Mp::i_lam_rank(ctx.rank));
    }

    // Inverse order of passes: P2B (low column bits), P2A, scatter, P1B, P1A.
    // The first pass reads the contiguous phase-2 slab (stage or global).
    template <class L, bool Last, bool FromInput>
    NTT_HD static void phase2_pass(Ctx& ctx, uint32_t tid) {
        uint32_t v[G::NP][L::E];
        const uint32_t d = L::dep(tid);
        if constexpr (FromInput)
            load_input<L, (1u << 30), G2Map>(ctx, v, d, d + ctx.rank * G::M);
        else
            load_smem<L, X, G::SLAB_WORDS>(ctx, v, d);
        run_stages<G, L, Arith, false, true, false, Last>(ctx, v, d);
        if constexpr (Last) {
            ctx.before_scatter();
            scatter<L>(ctx, v, d);
        } else {
            store_smem<L, X, G::SLAB_WORDS>(ctx, v, d);
        }
    }
    // With two phase-2 passes and direct input, pass2c first copies the
    // input slab into the work buffer in warp chunks (SlabChunk); the
    // staged schedule's first pass reads the bulk-copied stage buffer.
    static constexpr bool kChunkIn = G::K2B > 0 && !Ctx::kStaged;
    NTT_HD static void pass2c(Ctx& ctx, uint32_t tid) {
        if constexpr (kChunkIn) slab_in<G, X>(ctx, tid);
    }
    NTT_HD static void pass2b(Ctx& ctx, uint32_t tid) {
        if constexpr (G::K2B > 0) phase2_pass<P2B, false, !kChunkIn>(ctx, tid);
    }
    NTT_HD static void pass2a(Ctx& ctx, uint32_t tid) {
        phase2_pass<P2A, true, G::K2B == 0>(ctx, tid);
    }
    NTT_HD static void pass1b(Ctx& ctx, uint32_t tid) {
        if constexpr (G::K1B > 0) {
            uint32_t v[G::NP][P1B::E];
            const uint32_t d = P1B::dep(tid);
            load_smem<P1B, X, G::SLAB_WORDS>(ctx, v, d);
            run_stages<G, P1B, Arith, false, false, false>(ctx, v, d);
            store_smem<P1B, X, G::SLAB_WORDS>(ctx, v, d);
        }
    }
    // Last pass: contains the limb's stage 0 (fold N^{-1} R^{-1}), canonical
    // output to the phase-1 slab in global memory.
    NTT_HD static void pass1a(Ctx& ctx, uint32_t tid) {
        uint32_t v[G::NP][P1A::E];
        const uint32_t d = P1A::dep(tid);
        load_smem<P1A, X, G::SLAB_WORDS>(ctx, v, d);
        run_stages<G, P1A, Arith, false, false, true>(ctx, v, d);
        store_global<P1A, G::W1, G1Map<G>>(ctx, v, Mp::g1(d) + Mp::g1_rank(ctx.rank), Ident{});
    }
};

}  // namespace nttb
