// CPU emulator of the fused kernels' register passes (test infrastructure):
// the C entry points over every compiled configuration (the instantiations
// live in emu_n*.cu, one file per configuration list, compiled in parallel).
#include "emu_core.h"

namespace emu {

uint32_t* g_dump = nullptr;  // optional: work buffer of every CTA after the forward scatter

// Conflict degree of each warp-wide access = max number of distinct words
// (16-byte chunks for the 128-bit stage reads, per quarter warp) that map
// to one bank.
void account(EmuCluster& cl, Stats& st) {
    static const bool verbose = getenv("NTT_EMU_VERBOSE") != nullptr;
    std::map<std::tuple<uint32_t, uint32_t, uint32_t, uint32_t, uint32_t>, std::vector<uint32_t>>
        groups;
    for (auto& a : cl.log) groups[{a.src, a.warp, a.seq, a.kind, a.rank_dst}].push_back(a.addr);
    double worst_step = 0, sum_step = 0, wk[6] = {0, 0, 0, 0, 0, 0};
    long n_step = 0;
    for (auto& kv : groups) {
        const uint32_t kd = std::get<3>(kv.first);
        // 16-byte pieces (stage reads, kind 3; 128-bit work-buffer accesses,
        // kind 4) in groups of 4 banks, 8-byte pieces (kind 5) in pairs
        const uint32_t vw = (kd == 3 || kd == 4) ? 4u : kd == 5 ? 2u : 1u;
        std::map<uint32_t, std::vector<uint32_t>> banks;
        for (uint32_t w0 : kv.second) {
            const uint32_t w = w0 / vw;
            auto& v = banks[w % (32u / vw)];
            bool dup = false;
            for (uint32_t x : v) dup |= (x == w);
            if (!dup) v.push_back(w);
        }
        size_t deg = 0;
        for (auto& b : banks) deg = b.second.size() > deg ? b.second.size() : deg;
        st.worst = deg > st.worst ? deg : st.worst;
        st.sum += deg;
        st.n++;
        worst_step = deg > worst_step ? deg : worst_step;
        sum_step += deg;
        n_step++;
        wk[kd] = deg > wk[kd] ? deg : wk[kd];
    }
    if (verbose && n_step)
        fprintf(stderr, "  step: worst %.0f avg %.2f (lds %.0f, sts %.0f, dsmem %.0f, stage128 %.0f)\n",
                worst_step, sum_step / n_step, wk[0], wk[1], wk[2], wk[3]);
    cl.log.clear();
}

#define EMU_LIST(n) extern const Entry kEmu##n[]; extern const int kEmu##n##Count;
EMU_LIST(N10) EMU_LIST(N11) EMU_LIST(N12) EMU_LIST(N13) EMU_LIST(N14) EMU_LIST(N15)
EMU_LIST(N16) EMU_LIST(N16B) EMU_LIST(N16M) EMU_LIST(N17)

namespace {
// the same order as NTTB_CFG_ALL (configs.h)
const std::vector<Entry>& entries() {
    static const std::vector<Entry> v = [] {
        std::vector<Entry> r;
#define EMU_ADD(n) r.insert(r.end(), kEmu##n, kEmu##n + kEmu##n##Count);
        EMU_ADD(N10) EMU_ADD(N11) EMU_ADD(N12) EMU_ADD(N13) EMU_ADD(N14) EMU_ADD(N15)
        EMU_ADD(N16) EMU_ADD(N16B) EMU_ADD(N16M) EMU_ADD(N17)
        return r;
    }();
    return v;
}
std::string g_err;
}  // namespace

extern const SplitEntry kEmuSplit[];
extern const int kEmuSplitCount;

}  // namespace emu

using namespace emu;

extern "C" {
int emu_num_configs() { return (int)entries().size(); }
// out9: N, CL, R1, EB, K1A, K2A, NP, threads, shared-memory bytes
void emu_config(int i, int* out9) {
    for (int k = 0; k < 7; ++k) out9[k] = entries()[i].v[k];
    out9[7] = entries()[i].threads;
    out9[8] = (int)entries()[i].smem;
}
// data: limbs * N words in place; tw_pairs: limbs * N (w, w') pairs, or
// limbs * tw_comp_entries(logN) with mode bit 2.
// mode bit 0: forward (else inverse); bit 1: direct input (else staged);
// bit 2: direct input over compressed tables.
int emu_transform(int i, int mode, uint32_t* data, const uint32_t* tw_pairs, const uint32_t* q,
                  int limbs, double* stats) {
    g_err.clear();
    RunFn fn = (mode & 4) ? entries()[i].comp : (mode & 2) ? entries()[i].direct
                                                          : entries()[i].staged;
    if (!fn) {
        g_err = "no compressed-table form below logN 15";
        return 1;
    }
    return fn(mode & 1, data, tw_pairs, q, limbs, stats, g_err);
}
const char* emu_last_error() { return g_err.c_str(); }
// Split configurations (NTTB_SPLIT_ALL order).  out7: N, CL, EB, K2A, K2B,
// threads, shared-memory bytes.
int emu_num_split() { return kEmuSplitCount; }
void emu_split_config(int i, int* out7) {
    for (int k = 0; k < 5; ++k) out7[k] = kEmuSplit[i].v[k];
    out7[5] = kEmuSplit[i].threads;
    out7[6] = (int)kEmuSplit[i].smem;
}
// mode bit 0: forward (else inverse); bit 2: compressed tables.
int emu_split_transform(int i, int mode, uint32_t* data, const uint32_t* tw_pairs,
                        const uint32_t* q, int limbs, double* stats) {
    g_err.clear();
    RunFn fn = (mode & 4) ? kEmuSplit[i].comp : kEmuSplit[i].full;
    return fn(mode & 1, data, tw_pairs, q, limbs, stats, g_err);
}
void emu_set_dump(uint32_t* p) { g_dump = p; }
}
