// CPU emulator of the fused kernels' register passes (test infrastructure).
//
// Runs the very same pass functions as the device kernels (ntt_core.cuh) on
// the host, thread by thread, with the barriers between passes implied, and
// checks what a GPU run cannot show safely: every global / shared / DSMEM
// access is in bounds, every scatter and store covers its destination
// exactly once, and how many ways each warp-wide shared-memory access is
// bank-conflicted.  Built by tests/emu/Makefile into libntt_emu.so (host
// code only; nothing here runs on a GPU).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../ntt_b200/csrc/configs.h"
#include "../../ntt_b200/csrc/ntt_core.cuh"

using namespace nttb;

namespace {

struct Access {
    uint32_t warp, seq, kind, rank_dst;
    uint32_t addr;
};

struct EmuCluster {
    int C = 1;
    uint32_t smem_words = 0;
    std::vector<std::vector<uint32_t>> smem;
    // DSMEM scatter target: the device orders every CTA's local reads of a
    // step before any remote store lands (cluster arrive/wait), so remote
    // stores go to a shadow copy that is committed when the step ends.
    std::vector<std::vector<uint32_t>> shadow;
    std::vector<std::vector<uint32_t>> writes;  // per word write count in current step
    std::vector<std::vector<uint32_t>> rwrites;
    std::vector<Access> log;
    std::string err;
};

struct EmuCtx {
    EmuCluster* cl;
    uint32_t* g;
    uint32_t glen;
    const TwPair* twp;
    uint32_t twlen;
    uint32_t q, q2, rank;
    uint32_t tid = 0, seq = 0;
    std::vector<uint32_t>* gwrites;

    void fail(const char* what, uint64_t v) {
        if (cl->err.empty()) {
            char b[160];
            snprintf(b, sizeof b, "%s out of range: %llu (rank %u tid %u)", what,
                     (unsigned long long)v, rank, tid);
            cl->err = b;
        }
    }
    uint32_t gload(uint32_t o) {
        if (o >= glen) { fail("gload", o); return 0; }
        return g[o];
    }
    void gload4(uint32_t o, uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d) {
        if (o % 4 || o + 3 >= glen) { fail("gload4", o); a = b = c = d = 0; return; }
        a = g[o]; b = g[o + 1]; c = g[o + 2]; d = g[o + 3];
    }
    void gstore(uint32_t o, uint32_t v) {
        if (o >= glen) { fail("gstore", o); return; }
        g[o] = v;
        (*gwrites)[o]++;
    }
    void gstore4(uint32_t o, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
        if (o % 4 || o + 3 >= glen) { fail("gstore4", o); return; }
        g[o] = a; g[o + 1] = b; g[o + 2] = c; g[o + 3] = d;
        for (int i = 0; i < 4; ++i) (*gwrites)[o + i]++;
    }
    uint32_t sload(uint32_t w) {
        if (w >= cl->smem_words) { fail("sload", w); return 0; }
        cl->log.push_back({tid / 32, seq++, 0, rank, w});
        return cl->smem[rank][w];
    }
    void sstore(uint32_t w, uint32_t v) {
        if (w >= cl->smem_words) { fail("sstore", w); return; }
        cl->log.push_back({tid / 32, seq++, 1, rank, w});
        cl->smem[rank][w] = v;
        cl->writes[rank][w]++;
    }
    void rstore(uint32_t dst, uint32_t w, uint32_t v) {
        if (dst >= (uint32_t)cl->C) { fail("rstore rank", dst); return; }
        if (w >= cl->smem_words) { fail("rstore", w); return; }
        cl->log.push_back({tid / 32, seq++, 2, dst, w});
        cl->shadow[dst][w] = v;
        cl->writes[dst][w]++;
        cl->rwrites[dst][w]++;
    }
    TwPair tw(uint32_t i) {
        if (i >= twlen) { fail("twiddle", i); return TwPair{0, 0}; }
        return twp[i];
    }
    void after_local_reads() {}
    void before_scatter() {}
};

uint32_t* g_dump = nullptr;  // optional: shared state after the scatter

struct Stats {
    double worst = 0, sum = 0;
    long n = 0;
};

// Conflict degree of each warp-wide access = max number of distinct words
// that map to one bank (remote stores are grouped per destination CTA).
void account(EmuCluster& cl, Stats& st) {
    std::map<std::tuple<uint32_t, uint32_t, uint32_t, uint32_t>, std::vector<uint32_t>> groups;
    for (auto& a : cl.log) groups[{a.warp, a.seq, a.kind, a.rank_dst}].push_back(a.addr);
    for (auto& kv : groups) {
        std::map<uint32_t, std::vector<uint32_t>> banks;
        for (uint32_t w : kv.second) {
            auto& v = banks[w % 32];
            bool dup = false;
            for (uint32_t x : v) dup |= (x == w);
            if (!dup) v.push_back(w);
        }
        size_t deg = 0;
        for (auto& b : banks) deg = b.second.size() > deg ? b.second.size() : deg;
        st.worst = deg > st.worst ? deg : st.worst;
        st.sum += deg;
        st.n++;
    }
    cl.log.clear();
}

template <class G, class Arith, bool Fwd>
int run_limb(uint32_t* limb, const TwPair* tw, uint32_t q, Stats& st, std::string& err) {
    EmuCluster cl;
    cl.C = G::C;
    cl.smem_words = G::SMEM_WORDS;
    cl.smem.assign(G::C, std::vector<uint32_t>(G::SMEM_WORDS, 0xDEADBEEFu));
    cl.writes.assign(G::C, std::vector<uint32_t>(G::SMEM_WORDS, 0));
    cl.shadow.assign(G::C, std::vector<uint32_t>(G::SMEM_WORDS, 0));
    cl.rwrites.assign(G::C, std::vector<uint32_t>(G::SMEM_WORDS, 0));
    std::vector<uint32_t> gw(1u << G::LOGN, 0);
    auto mk = [&](uint32_t rank) {
        EmuCtx c{&cl, limb, 1u << G::LOGN, tw, 1u << G::LOGN, q, 2 * q, rank};
        c.gwrites = &gw;
        return c;
    };
    using F = Forward<G, Arith, EmuCtx>;
    using I = Inverse<G, Arith, EmuCtx>;
    // step runner: run fn for every thread of every CTA
    auto step = [&](auto fn) {
        for (auto& w : cl.writes) std::fill(w.begin(), w.end(), 0u);
        for (auto& w : cl.rwrites) std::fill(w.begin(), w.end(), 0u);
        for (uint32_t r = 0; r < (uint32_t)G::C; ++r) {
            EmuCtx c = mk(r);
            for (uint32_t t = 0; t < (uint32_t)G::THREADS; ++t) {
                c.tid = t;
                c.seq = 0;
                fn(c, t);
            }
        }
        for (int r = 0; r < G::C; ++r)
            for (uint32_t w = 0; w < G::SMEM_WORDS; ++w)
                if (cl.rwrites[r][w]) cl.smem[r][w] = cl.shadow[r][w];
        account(cl, st);
    };
    // every non-pad shared word written exactly once by a store step
    auto check_cover = [&](const char* what) {
        for (int r = 0; r < G::C; ++r)
            for (uint32_t lam = 0; lam < G::M; ++lam)
                if (cl.writes[r][smem_phys(lam)] != 1) {
                    if (err.empty())
                        err = std::string(what) + ": shared word not written exactly once";
                    return;
                }
    };
    if (Fwd) {
        step([](EmuCtx& c, uint32_t t) { F::pass1a(c, t); });
        if (G::K1B > 0) {
            check_cover("pass1a");
            step([](EmuCtx& c, uint32_t t) { F::pass1b(c, t); });
        }
        check_cover("scatter");
        if (g_dump)
            for (int r = 0; r < G::C; ++r)
                for (uint32_t lam = 0; lam < G::M; ++lam)
                    g_dump[r * G::M + lam] = cl.smem[r][smem_phys(lam)];
        step([](EmuCtx& c, uint32_t t) { F::pass2a(c, t); });
        if (G::K2B > 0) {
            check_cover("pass2a");
            step([](EmuCtx& c, uint32_t t) { F::pass2b(c, t); });
        }
    } else {
        if (G::K2B > 0) {
            step([](EmuCtx& c, uint32_t t) { I::pass2b(c, t); });
            check_cover("pass2b");
        }
        step([](EmuCtx& c, uint32_t t) { I::pass2a(c, t); });
        check_cover("scatter");
        if (G::K1B > 0) {
            step([](EmuCtx& c, uint32_t t) { I::pass1b(c, t); });
            check_cover("pass1b");
        }
        step([](EmuCtx& c, uint32_t t) { I::pass1a(c, t); });
    }
    for (uint32_t i = 0; i < (1u << G::LOGN); ++i)
        if (gw[i] != 1 && err.empty()) err = "global word not written exactly once";
    if (!cl.err.empty() && err.empty()) err = cl.err;
    return err.empty() ? 0 : 1;
}

template <class G>
int run_cfg(int fwd, uint32_t* data, const uint32_t* tw_pairs, const uint32_t* q, int limbs,
            double* stats, std::string& err) {
    Stats st;
    const size_t N = size_t{1} << G::LOGN;
    for (int l = 0; l < limbs; ++l) {
        const TwPair* tw = reinterpret_cast<const TwPair*>(tw_pairs) + l * N;
        int rc;
        if (q[l] < (1u << 30))
            rc = fwd ? run_limb<G, Lazy4, true>(data + l * N, tw, q[l], st, err)
                     : run_limb<G, Lazy4, false>(data + l * N, tw, q[l], st, err);
        else
            rc = fwd ? run_limb<G, Lazy2, true>(data + l * N, tw, q[l], st, err)
                     : run_limb<G, Lazy2, false>(data + l * N, tw, q[l], st, err);
        if (rc) return rc;
    }
    if (stats) {
        stats[0] = st.worst;
        stats[1] = st.n ? st.sum / st.n : 0;
    }
    return 0;
}

struct Entry {
    int v[6];
    int threads;
    unsigned smem;
    int (*fn)(int, uint32_t*, const uint32_t*, const uint32_t*, int, double*, std::string&);
};

#define EMU_ENTRY(N, CL, R1, EB, K1A, K2A)                                              \
    {{N, CL, R1, EB, K1A, K2A}, Geometry<N, CL, R1, EB, K1A, K2A>::THREADS,             \
     Geometry<N, CL, R1, EB, K1A, K2A>::SMEM_BYTES,                                     \
     &run_cfg<Geometry<N, CL, R1, EB, K1A, K2A>>},
const Entry kEntries[] = {NTTB_CFG_ALL(EMU_ENTRY)};
std::string g_err;

}  // namespace

extern "C" {
int emu_num_configs() { return (int)(sizeof(kEntries) / sizeof(kEntries[0])); }
void emu_config(int i, int* out8) {
    for (int k = 0; k < 6; ++k) out8[k] = kEntries[i].v[k];
    out8[6] = kEntries[i].threads;
    out8[7] = (int)kEntries[i].smem;
}
// data: limbs * N words in place; tw_pairs: limbs * N (w, w') pairs.
int emu_transform(int i, int fwd, uint32_t* data, const uint32_t* tw_pairs, const uint32_t* q,
                  int limbs, double* stats) {
    g_err.clear();
    return kEntries[i].fn(fwd, data, tw_pairs, q, limbs, stats, g_err);
}
const char* emu_last_error() { return g_err.c_str(); }
void emu_set_dump(uint32_t* p) { g_dump = p; }
}
