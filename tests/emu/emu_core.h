// CPU emulator of the fused kernels' register passes (test infrastructure):
// the shared part of emu.cu and the per-list instantiation files emu_n*.cu.
//
// Runs the very same pass functions as the device kernels (ntt_core.cuh) on
// the host, thread by thread, with the barriers between passes implied, and
// checks what a GPU run cannot show safely: every global / stage / shared /
// DSMEM access is in bounds, the bulk copies cover the stage buffer and every
// scatter and store covers its destination exactly once, every read after a
// warp barrier reads words its own warp wrote, and how many ways each
// warp-wide shared-memory access is bank-conflicted.  Built by
// tests/emu/Makefile into libntt_emu.so (host code only; nothing here runs on
// a GPU).
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "../../ntt_b200/csrc/configs.h"
#include "../../ntt_b200/csrc/ntt_core.cuh"
#include "../../ntt_b200/csrc/split_geo.cuh"

using namespace nttb;

namespace emu {


struct Access {
    uint32_t warp, seq, kind, rank_dst;  // kind: 0 lds, 1 sts, 2 dsmem, 3 stage128, 4 / 5 work buffer 128 / 64-bit (rank_dst: the warp phase)
    uint32_t addr;
    uint32_t src;  // issuing CTA
};

struct EmuCluster {
    int C = 1;
    uint32_t smem_words = 0;
    std::vector<std::vector<uint32_t>> smem;
    // Scatter target: the device orders every CTA's local reads of a step
    // before any remote store lands (cluster arrive/wait), so scattered words
    // go to a shadow copy committed when the step ends.
    std::vector<std::vector<uint32_t>> shadow;
    std::vector<std::vector<uint32_t>> writes;   // per-word write count, this step
    std::vector<std::vector<uint32_t>> rwrites;  // scattered words, this step
    std::vector<std::vector<uint32_t>> writer;   // warp that last wrote each word
    std::vector<std::vector<uint32_t>> stage;    // padded input slab per CTA
    bool warp_local = false;                     // this step follows a warp barrier
    std::vector<Access> log;
    std::string err;
};

// Global words of polynomial p of a job are addressed as (p << kPolyShift) +
// word index (the pass code only adds offsets below 2^kPolyShift).
constexpr uint32_t kPolyShift = 24;

template <bool Staged, bool Comp = false>
struct EmuCtx {
    static constexpr bool kStaged = Staged;
    static constexpr bool kCompTw = Comp;  // compressed twiddle tables (arith.cuh)
    EmuCluster* cl;
    uint32_t** gp;  // the job's polynomials (limb words each)
    uint32_t glen;
    const TwPair* twp;
    uint32_t twlen;
    uint32_t q, q2, rank;
    uint32_t tid = 0, seq = 0;
    std::vector<uint32_t>* gwrites;  // per polynomial

    void fail(const char* what, uint64_t v) {
        if (cl->err.empty()) {
            char b[200];
            snprintf(b, sizeof b, "%s: %llu (rank %u tid %u)", what, (unsigned long long)v, rank,
                     tid);
            cl->err = b;
        }
    }
    // global: base and offsets are word indices into the limb of polynomial p
    uint32_t g_base(int p, uint32_t o) { return ((uint32_t)p << kPolyShift) + o; }
    uint32_t g_ld(uint32_t b, uint32_t c) {
        const uint32_t p = (b + c) >> kPolyShift, o = (b + c) & ((1u << kPolyShift) - 1u);
        if (o >= glen) {
            fail("g_ld out of range", o);
            return 0;
        }
        return gp[p][o];
    }
    void g_ld4(uint32_t b, uint32_t c, uint32_t& x, uint32_t& y, uint32_t& z, uint32_t& w) {
        const uint32_t p = (b + c) >> kPolyShift, o = (b + c) & ((1u << kPolyShift) - 1u);
        if (o % 4 || o + 3 >= glen) {
            fail("g_ld4 out of range or misaligned", o);
            x = y = z = w = 0;
            return;
        }
        x = gp[p][o];
        y = gp[p][o + 1];
        z = gp[p][o + 2];
        w = gp[p][o + 3];
    }
    // transform output (in place)
    uint32_t o_base(int p, uint32_t o) { return ((uint32_t)p << kPolyShift) + o; }
    void o_st(uint32_t b, uint32_t c, uint32_t v) {
        const uint32_t p = (b + c) >> kPolyShift, o = (b + c) & ((1u << kPolyShift) - 1u);
        if (o >= glen) {
            fail("o_st out of range", o);
            return;
        }
        gp[p][o] = v;
        gwrites[p][o]++;
    }
    void o_st4(uint32_t b, uint32_t c, uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
        const uint32_t p = (b + c) >> kPolyShift, o = (b + c) & ((1u << kPolyShift) - 1u);
        if (o % 4 || o + 3 >= glen) {
            fail("o_st4 out of range or misaligned", o);
            return;
        }
        gp[p][o] = x;
        gp[p][o + 1] = y;
        gp[p][o + 2] = z;
        gp[p][o + 3] = w;
        for (int i = 0; i < 4; ++i) gwrites[p][o + i]++;
    }
    // stage buffer
    uint32_t st_base(uint32_t w) { return w; }
    uint32_t st_ld(uint32_t b, uint32_t c) {
        const uint32_t w = b + c;
        if (w >= cl->stage[rank].size()) {
            fail("st_ld out of range", w);
            return 0;
        }
        cl->log.push_back({tid / 32, seq++, 0, rank, w, rank});
        return cl->stage[rank][w];
    }
    void st_ld4(uint32_t b, uint32_t c, uint32_t& x, uint32_t& y, uint32_t& z, uint32_t& w4) {
        const uint32_t w = b + c;
        if (w % 4 || w + 3 >= cl->stage[rank].size()) {
            fail("st_ld4 out of range or misaligned", w);
            x = y = z = w4 = 0;
            return;
        }
        cl->log.push_back({tid / 32, seq++, 3, (tid % 32) / 8, w, rank});
        x = cl->stage[rank][w];
        y = cl->stage[rank][w + 1];
        z = cl->stage[rank][w + 2];
        w4 = cl->stage[rank][w + 3];
    }
    // work buffer
    uint32_t s_base(uint32_t w) { return w; }
    uint32_t s_ld(uint32_t b, uint32_t c) {
        const uint32_t w = b + c;
        if (w >= cl->smem_words) {
            fail("s_ld out of range", w);
            return 0;
        }
        cl->log.push_back({tid / 32, seq++, 0, rank, w, rank});
        if (cl->warp_local && cl->writer[rank][w] != tid / 32)
            fail("warp-local read of another warp's word", w);
        return cl->smem[rank][w];
    }
    void s_st(uint32_t b, uint32_t c, uint32_t v) {
        const uint32_t w = b + c;
        if (w >= cl->smem_words) {
            fail("s_st out of range", w);
            return;
        }
        cl->log.push_back({tid / 32, seq++, 1, rank, w, rank});
        cl->smem[rank][w] = v;
        cl->writer[rank][w] = tid / 32;
        cl->writes[rank][w]++;
    }
    // 64- / 128-bit accesses: aligned, each word checked as a scalar one;
    // logged once per warp phase (kind 4: 16-byte pieces per quarter warp,
    // kind 5: 8-byte pieces per half warp) for the conflict accounting
    void s_vec(uint32_t b, uint32_t c, uint32_t* v, int n, bool store) {
        const uint32_t w = b + c;
        if (w % (uint32_t)n || w + n - 1 >= cl->smem_words) {
            fail(store ? "vector s_st out of range or misaligned" : "vector s_ld out of range or misaligned", w);
            return;
        }
        cl->log.push_back({tid / 32, seq++, n == 4 ? 4u : 5u, (tid % 32) / (n == 4 ? 8u : 16u), w, rank});
        for (int k = 0; k < n; ++k) {
            if (store) {
                cl->smem[rank][w + k] = v[k];
                cl->writer[rank][w + k] = tid / 32;
                cl->writes[rank][w + k]++;
            } else {
                if (cl->warp_local && cl->writer[rank][w + k] != tid / 32)
                    fail("warp-local read of another warp's word", w + k);
                v[k] = cl->smem[rank][w + k];
            }
        }
    }
    void s_ld4(uint32_t b, uint32_t c, uint32_t& x, uint32_t& y, uint32_t& z, uint32_t& w4) {
        uint32_t v[4] = {0, 0, 0, 0};
        s_vec(b, c, v, 4, false);
        x = v[0], y = v[1], z = v[2], w4 = v[3];
    }
    void s_st4(uint32_t b, uint32_t c, uint32_t x, uint32_t y, uint32_t z, uint32_t w4) {
        uint32_t v[4] = {x, y, z, w4};
        s_vec(b, c, v, 4, true);
    }
    void s_ld2(uint32_t b, uint32_t c, uint32_t& x, uint32_t& y) {
        uint32_t v[2] = {0, 0};
        s_vec(b, c, v, 2, false);
        x = v[0], y = v[1];
    }
    void s_st2(uint32_t b, uint32_t c, uint32_t x, uint32_t y) {
        uint32_t v[2] = {x, y};
        s_vec(b, c, v, 2, true);
    }
    std::pair<uint32_t, uint32_t> r_base(uint32_t dst, uint32_t w) { return {dst, w}; }
    template <uint32_t Off>
    void r_st(std::pair<uint32_t, uint32_t> rb, uint32_t v) {
        const uint32_t dst = rb.first, w = rb.second + Off;
        if (dst >= (uint32_t)cl->C) {
            fail("r_st rank out of range", dst);
            return;
        }
        if (w >= cl->smem_words) {
            fail("r_st out of range", w);
            return;
        }
        cl->log.push_back({tid / 32, seq++, 2, dst, w, rank});
        cl->shadow[dst][w] = v;
        cl->writes[dst][w]++;
        cl->rwrites[dst][w]++;
    }
    TwPair tw_at(uint32_t i) {
        if (i >= twlen) {
            fail("twiddle out of range", i);
            return TwPair{0, 0};
        }
        return twp[i];
    }
    TwPair fold_at(uint32_t i) { return tw_at(i); }
    uint32_t tw_base(uint32_t i) { return i; }
    TwPair tw_ld(uint32_t b, uint32_t c) { return tw_at(b + c); }
    void tw_ld2(uint32_t b, uint32_t c, TwPair& x, TwPair& y) {
        if ((b + c) % 2) fail("tw_ld2 misaligned", b + c);
        x = tw_at(b + c);
        y = tw_at(b + c + 1);
    }
    void after_local_reads() {}
    void before_scatter() {}
};

struct Stats {
    double worst = 0, sum = 0;
    long n = 0;
};

// optional: work buffer of every CTA after the forward scatter (emu.cu)
extern uint32_t* g_dump;

// Conflict degree of every warp-wide access of a step (emu.cu).
void account(EmuCluster& cl, Stats& st);

template <class G, class Arith, bool Fwd, bool Staged, bool Comp = false>
int run_limb(uint32_t* limb, const TwPair* tw, uint32_t q, Stats& st, std::string& err) {
    using Ctx = EmuCtx<Staged, Comp>;
    constexpr uint32_t kTwLen = Comp ? tw_comp_entries(G::LOGN) : (1u << G::LOGN);
    EmuCluster cl;
    cl.C = G::C;
    cl.smem_words = G::SMEM_WORDS;
    cl.smem.assign(G::C, std::vector<uint32_t>(G::SMEM_WORDS, 0xDEADBEEFu));
    cl.writes.assign(G::C, std::vector<uint32_t>(G::SMEM_WORDS, 0));
    cl.shadow.assign(G::C, std::vector<uint32_t>(G::SMEM_WORDS, 0));
    cl.rwrites.assign(G::C, std::vector<uint32_t>(G::SMEM_WORDS, 0));
    cl.writer.assign(G::C, std::vector<uint32_t>(G::SMEM_WORDS, 0xFFFFFFFFu));
    // the job's polynomials: poly 0 is the limb itself, poly p > 0 a
    // permutation of its words (inputs stay in range), checked at the end
    // against the one-polynomial geometry on the same input
    constexpr int NP = G::NP;
    constexpr uint32_t N = 1u << G::LOGN;
    std::vector<std::vector<uint32_t>> pw(NP, std::vector<uint32_t>(N));
    std::vector<uint32_t*> gp(NP);
    for (int p = 0; p < NP; ++p) {
        for (uint32_t i = 0; i < N; ++i) pw[p][i] = p == 0 ? limb[i] : limb[(N - 1 - i + p) % N];
        gp[p] = pw[p].data();
    }
    std::vector<std::vector<uint32_t>> gw(NP, std::vector<uint32_t>(N, 0));
    // the kernel's bulk copies of the input slab into each CTA's stage buffer
    cl.stage.assign(G::C, std::vector<uint32_t>(G::STAGE_WORDS, 0xDEADBEEFu));
    for (uint32_t r = 0; r < (uint32_t)G::C; ++r) {
        std::vector<uint32_t> cover(G::STAGE_WORDS, 0);
        for (uint32_t i = 0; i < slab_copies<G, Fwd>(); ++i) {
            const SlabCopy c = slab_copy<G, Fwd>(r, i);
            if ((c.src % 4) || (c.dst % 4) || (c.words % 4) || c.src + c.words > (1u << G::LOGN) ||
                c.dst + c.words > G::STAGE_WORDS) {
                err = "bulk copy descriptor out of range or not 16-byte granular";
                return 1;
            }
            for (uint32_t k = 0; k < c.words; ++k) {
                cl.stage[r][c.dst + k] = limb[c.src + k];
                cover[c.dst + k]++;
            }
        }
        for (uint32_t lam = 0; lam < G::M; ++lam)
            if (cover[StageLayout::phys(lam)] != 1) {
                err = "stage buffer not covered exactly once by the bulk copies";
                return 1;
            }
    }
    auto mk = [&](uint32_t rank) {
        Ctx c{&cl, gp.data(), 1u << G::LOGN, tw, kTwLen, q, 2 * q, rank};
        c.gwrites = gw.data();
        return c;
    };
    using F = Forward<G, Arith, Ctx>;
    using I = Inverse<G, Arith, Ctx>;
    // run fn for every thread of every CTA, then commit the scattered words
    auto step = [&](auto fn, bool warp_local) {
        cl.warp_local = warp_local;
        for (auto& w : cl.writes) std::fill(w.begin(), w.end(), 0u);
        for (auto& w : cl.rwrites) std::fill(w.begin(), w.end(), 0u);
        for (uint32_t r = 0; r < (uint32_t)G::C; ++r) {
            Ctx c = mk(r);
            for (uint32_t t = 0; t < (uint32_t)G::THREADS; ++t) {
                c.tid = t;
                c.seq = 0;
                fn(c, t);
            }
        }
        for (int r = 0; r < G::C; ++r)
            for (uint32_t w = 0; w < G::SMEM_WORDS; ++w)
                if (cl.rwrites[r][w]) {
                    cl.smem[r][w] = cl.shadow[r][w];
                    cl.writer[r][w] = 0xFFFFFFFFu;  // scattered words: never warp-local
                }
        account(cl, st);
    };
    // every non-pad work-buffer word written exactly once by the last step
    auto check_cover = [&](const char* what) {
        for (int r = 0; r < G::C; ++r)
            for (int p = 0; p < NP; ++p)
                for (uint32_t lam = 0; lam < G::M; ++lam)
                    if (cl.writes[r][p * G::SLAB_WORDS + G::XW::phys(lam)] != 1) {
                        if (err.empty()) err = std::string(what) + ": word not written exactly once";
                        return;
                    }
    };
    if (Fwd) {
        step([](Ctx& c, uint32_t t) { F::pass1a(c, t); }, false);
        if (G::K1B > 0) {
            check_cover("pass1a");
            step([](Ctx& c, uint32_t t) { F::pass1b(c, t); }, G::WARP1);
        }
        check_cover("forward scatter");
        if (g_dump)
            for (int r = 0; r < G::C; ++r)
                for (uint32_t lam = 0; lam < G::M; ++lam)
                    g_dump[r * G::M + lam] = cl.smem[r][G::XW::phys(lam)];
        step([](Ctx& c, uint32_t t) { F::pass2a(c, t); }, false);
        if (G::K2B > 0) {
            check_cover("pass2a");
            step([](Ctx& c, uint32_t t) { F::pass2b(c, t); }, G::WARP2);
            check_cover("pass2b");
            step([](Ctx& c, uint32_t t) { F::pass2c(c, t); }, G::WARP2);  // chunked store
        }
    } else {
        if (I::kChunkIn) {  // chunked load of the input slab
            step([](Ctx& c, uint32_t t) { I::pass2c(c, t); }, false);
            check_cover("inverse slab load");
        }
        if (G::K2B > 0) {
            step([](Ctx& c, uint32_t t) { I::pass2b(c, t); }, I::kChunkIn && G::WARP2);
            check_cover("pass2b");
        }
        step([](Ctx& c, uint32_t t) { I::pass2a(c, t); }, G::K2B > 0 && G::WARP2);
        check_cover("inverse scatter");
        if (G::K1B > 0) {
            step([](Ctx& c, uint32_t t) { I::pass1b(c, t); }, false);
            check_cover("pass1b");
        }
        step([](Ctx& c, uint32_t t) { I::pass1a(c, t); }, G::K1B > 0 && G::WARP1);
    }
    for (int p = 0; p < NP; ++p)
        for (uint32_t i = 0; i < N; ++i)
            if (gw[p][i] != 1 && err.empty()) err = "global word not written exactly once";
    if (!cl.err.empty() && err.empty()) err = cl.err;
    if (!err.empty()) return 1;
    if constexpr (NP > 1) {
        // every polynomial of the job equals its own one-polynomial transform
        using G1 = Geometry<G::LOGN, G::CLOG, G::R1, G::EB, G::K1A, G::K2A, 1>;
        for (int p = 1; p < NP; ++p) {
            std::vector<uint32_t> one(N);
            for (uint32_t i = 0; i < N; ++i) one[i] = limb[(N - 1 - i + p) % N];
            Stats st1;
            if (run_limb<G1, Arith, Fwd, false, Comp>(one.data(), tw, q, st1, err)) return 1;
            if (one != pw[p]) {
                err = "polynomial " + std::to_string(p) + " of a job differs from its own transform";
                return 1;
            }
        }
    }
    std::copy(pw[0].begin(), pw[0].end(), limb);
    return 0;
}

// Comp: the direct passes over compressed tables (tw_comp_entries pairs per
// limb instead of N).
template <class G, bool Staged, bool Comp = false>
int run_cfg(int fwd, uint32_t* data, const uint32_t* tw_pairs, const uint32_t* q, int limbs,
            double* stats, std::string& err) {
    Stats st;
    const size_t N = size_t{1} << G::LOGN;
    const size_t TWS = Comp ? tw_comp_entries(G::LOGN) : N;
    for (int l = 0; l < limbs; ++l) {
        const TwPair* tw = reinterpret_cast<const TwPair*>(tw_pairs) + l * TWS;
        int rc;
        if (q[l] < (1u << 30))
            rc = fwd ? run_limb<G, Lazy4, true, Staged, Comp>(data + l * N, tw, q[l], st, err)
                     : run_limb<G, Lazy4, false, Staged, Comp>(data + l * N, tw, q[l], st, err);
        else
            rc = fwd ? run_limb<G, Lazy2, true, Staged, Comp>(data + l * N, tw, q[l], st, err)
                     : run_limb<G, Lazy2, false, Staged, Comp>(data + l * N, tw, q[l], st, err);
        if (rc) return rc;
    }
    if (stats) {
        stats[0] = st.worst;
        stats[1] = st.n ? st.sum / st.n : 0;
    }
    return 0;
}

using RunFn = int (*)(int, uint32_t*, const uint32_t*, const uint32_t*, int, double*,
                      std::string&);
struct Entry {
    int v[7];
    int threads;
    unsigned smem;
    RunFn staged, direct;
    RunFn comp;  // direct, compressed tables (logN >= kTwCompMinLogN; else null)
};

// The compressed-table run of a geometry (none below kTwCompMinLogN).
template <class G>
constexpr RunFn comp_run() {
    if constexpr (G::LOGN >= kTwCompMinLogN) return &run_cfg<G, false, true>;
    else return nullptr;
}

// NP > 1 has no staged form: its staged entry runs the direct passes, as
// the library's does.
#define EMU_G(N, CL, R1, EB, K1A, K2A, NP) Geometry<N, CL, R1, EB, K1A, K2A, NP>
#define EMU_ENTRY(N, CL, R1, EB, K1A, K2A, NP)                                             \
    {{N, CL, R1, EB, K1A, K2A, NP},                                                        \
     EMU_G(N, CL, R1, EB, K1A, K2A, NP)::THREADS,                                          \
     EMU_G(N, CL, R1, EB, K1A, K2A, NP)::SMEM_BYTES,                                       \
     &run_cfg<EMU_G(N, CL, R1, EB, K1A, K2A, NP), (NP) == 1>,                              \
     &run_cfg<EMU_G(N, CL, R1, EB, K1A, K2A, NP), false>,                                  \
     comp_run<EMU_G(N, CL, R1, EB, K1A, K2A, NP)>()},
// ---------------------------------------------------------------------------
// Split configurations (split_geo.cuh): phase 1 straight from and back to
// global memory, the cluster barrier (here: the end of a step over every CTA),
// then the phase-2 passes in the work buffer and the chunked store.  The same
// checks as the cluster kernels: bounds, every work-buffer word of a pass and
// every global word of each phase written exactly once, warp-local reads
// after warp barriers, bank conflicts; bit-exact results against the oracle.
// ---------------------------------------------------------------------------
template <class G, class Arith, bool Fwd, bool Comp>
int run_split_limb(uint32_t* limb, const TwPair* tw, uint32_t q, Stats& st, std::string& err) {
    using Ctx = EmuCtx<false, Comp>;
    constexpr uint32_t N = 1u << G::LOGN;
    constexpr uint32_t kTwLen = Comp ? tw_comp_entries(G::LOGN) : N;
    EmuCluster cl;
    cl.C = G::C;
    cl.smem_words = G::SLAB_WORDS;
    cl.smem.assign(G::C, std::vector<uint32_t>(G::SLAB_WORDS, 0xDEADBEEFu));
    cl.writes.assign(G::C, std::vector<uint32_t>(G::SLAB_WORDS, 0));
    cl.shadow.assign(G::C, std::vector<uint32_t>(G::SLAB_WORDS, 0));
    cl.rwrites.assign(G::C, std::vector<uint32_t>(G::SLAB_WORDS, 0));
    cl.writer.assign(G::C, std::vector<uint32_t>(G::SLAB_WORDS, 0xFFFFFFFFu));
    std::vector<uint32_t> words(limb, limb + N);
    uint32_t* gp[1] = {words.data()};
    std::vector<uint32_t> gw[1] = {std::vector<uint32_t>(N, 0)};
    auto mk = [&](uint32_t rank) {
        Ctx c{&cl, gp, N, tw, kTwLen, q, 2 * q, rank};
        c.gwrites = gw;
        return c;
    };
    auto step = [&](auto fn, bool warp_local) {
        cl.warp_local = warp_local;
        for (auto& w : cl.writes) std::fill(w.begin(), w.end(), 0u);
        for (uint32_t r = 0; r < (uint32_t)G::C; ++r) {
            Ctx c = mk(r);
            for (uint32_t t = 0; t < (uint32_t)G::THREADS; ++t) {
                c.tid = t;
                c.seq = 0;
                fn(c, t);
            }
        }
        account(cl, st);
    };
    auto check_cover = [&](const char* what) {
        for (int r = 0; r < G::C; ++r)
            for (uint32_t lam = 0; lam < G::M; ++lam)
                if (cl.writes[r][G::XW::phys(lam)] != 1) {
                    if (err.empty()) err = std::string(what) + ": word not written exactly once";
                    return;
                }
    };
    auto check_global = [&](const char* what) {
        for (uint32_t i = 0; i < N; ++i)
            if (gw[0][i] != 1) {
                if (err.empty()) err = std::string(what) + ": global word not written exactly once";
                return;
            }
        std::fill(gw[0].begin(), gw[0].end(), 0u);
    };
    if constexpr (Fwd) {
        using F = SplitFwd<G, Arith, Ctx>;
        step([](Ctx& c, uint32_t t) { F::p1(c, t); }, false);
        check_global("phase 1");
        step([](Ctx& c, uint32_t t) { F::p2a(c, t); }, false);
        check_cover("pass 2a");
        step([](Ctx& c, uint32_t t) { F::p2b(c, t); }, G::kABWarp);
        check_cover("pass 2b");
        if constexpr (G::K2C > 0) {
            step([](Ctx& c, uint32_t t) { F::p2c(c, t); }, G::kBCWarp);
            check_cover("pass 2c");
        }
        step([](Ctx& c, uint32_t t) { F::out(c, t); }, G::kChunkWarp);
        check_global("output");
    } else {
        using I = SplitInv<G, Arith, Ctx>;
        step([](Ctx& c, uint32_t t) { I::in(c, t); }, false);
        check_cover("slab in");
        if constexpr (G::K2C > 0) {
            step([](Ctx& c, uint32_t t) { I::p2c(c, t); }, G::kChunkWarp);
            check_cover("pass 2c");
            step([](Ctx& c, uint32_t t) { I::p2b(c, t); }, G::kBCWarp);
        } else {
            step([](Ctx& c, uint32_t t) { I::p2b(c, t); }, G::kChunkWarp);
        }
        check_cover("pass 2b");
        step([](Ctx& c, uint32_t t) { I::p2a(c, t); }, G::kABWarp);
        check_global("phase 2");
        step([](Ctx& c, uint32_t t) { I::p1(c, t); }, false);
        check_global("phase 1");
    }
    if (!cl.err.empty() && err.empty()) err = cl.err;
    if (!err.empty()) return 1;
    std::copy(words.begin(), words.end(), limb);
    return 0;
}

template <class G, bool Comp>
int run_split_cfg(int fwd, uint32_t* data, const uint32_t* tw_pairs, const uint32_t* q, int limbs,
                  double* stats, std::string& err) {
    Stats st;
    const size_t N = size_t{1} << G::LOGN;
    const size_t TWS = Comp ? tw_comp_entries(G::LOGN) : N;
    for (int l = 0; l < limbs; ++l) {
        const TwPair* tw = reinterpret_cast<const TwPair*>(tw_pairs) + l * TWS;
        int rc;
        if (q[l] < (1u << 30))
            rc = fwd ? run_split_limb<G, Lazy4, true, Comp>(data + l * N, tw, q[l], st, err)
                     : run_split_limb<G, Lazy4, false, Comp>(data + l * N, tw, q[l], st, err);
        else
            rc = fwd ? run_split_limb<G, Lazy2, true, Comp>(data + l * N, tw, q[l], st, err)
                     : run_split_limb<G, Lazy2, false, Comp>(data + l * N, tw, q[l], st, err);
        if (rc) return rc;
    }
    if (stats) {
        stats[0] = st.worst;
        stats[1] = st.n ? st.sum / st.n : 0;
    }
    return 0;
}

struct SplitEntry {
    int v[5];
    int threads;
    unsigned smem;
    RunFn full, comp;  // full / compressed twiddle tables
};

#define EMU_SG(N, CL, EB, KA, KB) SplitGeo<N, CL, EB, KA, KB>
#define EMU_SPLIT_ENTRY(N, CL, EB, KA, KB)                                                       \
    {{N, CL, EB, KA, KB}, EMU_SG(N, CL, EB, KA, KB)::THREADS, EMU_SG(N, CL, EB, KA, KB)::SMEM_BYTES, \
     &run_split_cfg<EMU_SG(N, CL, EB, KA, KB), false>,                                            \
     &run_split_cfg<EMU_SG(N, CL, EB, KA, KB), true>},

}  // namespace emu
