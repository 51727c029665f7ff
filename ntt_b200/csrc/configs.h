// Compiled fused-kernel configurations.
//
// X(LOGN, CLOG, R1, EB, K1A, K2A, NP):
//   LOGN  log2 N of the limb
//   CLOG  log2 of the thread-block cluster size (CTAs per limb)
//   R1    stages of phase 1 (the reference's NTT-Phase1 radix_stages); phase 2
//         does LOGN - R1 (its NTT-Phase2 radix_stages)
//   EB    log2 words per thread in a register pass (the reference's
//         stage_merging upper bound: a pass merges up to EB radix-2 stages)
//   K1A   stages of the first register pass of phase 1 (rest: second pass)
//   K2A   stages of the first register pass of phase 2
//   NP    polynomials per job: one cluster transforms the same limb of NP
//         polynomials at once, so each twiddle it loads serves NP butterflies
//         (2^EB words per thread per polynomial; direct schedule only)
// Each logN has its own list so the instantiations compile in parallel
// (logN 16 in three: two of one polynomial per job, one of two).
#pragma once

#define NTTB_CFG_N10(X) X(10, 0, 5, 5, 5, 5, 1)
#define NTTB_CFG_N11(X) X(11, 0, 6, 5, 1, 5, 1)
#define NTTB_CFG_N12(X) X(12, 0, 7, 5, 3, 5, 1) X(12, 0, 6, 4, 3, 3, 1)
#define NTTB_CFG_N13(X) X(13, 0, 8, 5, 3, 5, 1)
#define NTTB_CFG_N14(X) X(14, 0, 9, 5, 4, 5, 1) X(14, 1, 9, 5, 4, 5, 1) X(14, 1, 6, 6, 6, 4, 1)
#define NTTB_CFG_N15(X) X(15, 1, 10, 5, 5, 5, 1) X(15, 2, 8, 5, 3, 4, 1) X(15, 2, 6, 6, 6, 5, 1)
#define NTTB_CFG_N16(X) \
    X(16, 3, 8, 5, 3, 4, 1) X(16, 3, 7, 5, 3, 5, 1) X(16, 2, 8, 5, 3, 4, 1) X(16, 4, 8, 5, 3, 4, 1)
#define NTTB_CFG_N16B(X) X(16, 3, 8, 4, 4, 4, 1) X(16, 3, 6, 6, 6, 5, 1) X(16, 4, 6, 6, 6, 4, 1)
#define NTTB_CFG_N16M(X) \
    X(16, 3, 8, 5, 3, 4, 2) X(16, 3, 7, 5, 3, 5, 2) X(16, 4, 8, 5, 3, 4, 2) \
    X(16, 3, 8, 4, 4, 4, 2) X(16, 4, 8, 4, 4, 4, 2)
#define NTTB_CFG_N17(X) X(17, 3, 8, 5, 3, 5, 1) X(17, 4, 8, 5, 3, 5, 1) X(17, 4, 6, 6, 6, 5, 1)

#define NTTB_CFG_ALL(X)                                                                      \
    NTTB_CFG_N10(X) NTTB_CFG_N11(X) NTTB_CFG_N12(X) NTTB_CFG_N13(X) NTTB_CFG_N14(X)      \
    NTTB_CFG_N15(X) NTTB_CFG_N16(X) NTTB_CFG_N16B(X) NTTB_CFG_N16M(X) NTTB_CFG_N17(X)

// Split configurations (split_kernel.cuh): S(LOGN, CLOG, EB, K2A, K2B).
//   Phase 1 = EB row stages, one register pass per column straight from and
//   back to global memory; the limb's CTAs then exchange through L2 (in
//   place) across one cluster barrier; phase 2 = passes of K2A, K2B and
//   LOGN - EB - K2A - K2B (if nonzero) stages over the CTA's contiguous rows.
#define NTTB_SPLIT_N16(S) \
    S(16, 3, 5, 4, 4) S(16, 3, 4, 4, 4) S(16, 3, 5, 3, 4) S(16, 4, 5, 4, 4) S(16, 4, 4, 4, 4)
#define NTTB_SPLIT_REST(S) \
    S(17, 4, 5, 4, 4) S(15, 3, 5, 4, 3) S(15, 2, 5, 5, 5) S(15, 2, 4, 4, 4)
#define NTTB_SPLIT_ALL(S) NTTB_SPLIT_N16(S) NTTB_SPLIT_REST(S)

#include <cstdint>

namespace nttb {

struct FusedConfig {
    int logN, clog, r1, eb, k1a, k2a, np;
    int threads;
    uint32_t smem_bytes;         // staged kernels (work + stage buffer + mbarrier)
    uint32_t smem_bytes_direct;  // direct kernels (work buffer)
    // fused_kernel<G, Fwd, Staged, Arith>: [staged][fwd][lazy2]; NP > 1
    // configurations have no staged form: their staged entries are the
    // direct kernels (run over resident chunks of jobs)
    const void* kern[2][2][2];
    // the direct forward with the product epilogue (fused_kernel<..., Mul>): [lazy2]
    // (nullptr for split configurations: a cluster configuration runs it)
    const void* kern_mul[2];
    int split;  // 1: split configuration (exchange through L2), 0: cluster scatter
    int k2b;    // split: stages of the second phase-2 pass
    // split: the one-launch negacyclic product (split_mul_kernel) [lazy2]
    // and its dynamic shared memory (work buffer + the spectrum of b)
    const void* kern_smul[2];
    uint32_t smem_smul;
    // the direct forward with the subtract-and-scale output (ModDown;
    // FusedArgs.sub): [lazy2]
    const void* kern_sub[2];
    // split: the transforms over compressed twiddle tables (plans created
    // with NTT_PLAN_COMPRESSED_TWIDDLES) [fwd][lazy2]; null for cluster
    // configurations
    const void* kern_comp[2][2];
    // split: the forward whose final store multiplies by a resident spectrum
    // (ntt_multiply_spectrum_many) [lazy2]; null for cluster configurations
    const void* kern_mulspec[2];
    bool has_mul() const { return kern_mul[0] != nullptr; }
    const void* kernel(bool staged, bool fwd, bool lazy2) const {
        return kern[staged ? 1 : 0][fwd ? 1 : 0][lazy2 ? 1 : 0];
    }
};

// All compiled configurations (registry.cu); count via fused_config_count().
const FusedConfig* fused_configs();
int fused_config_count();

}  // namespace nttb
