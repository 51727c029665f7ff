// Internal interfaces shared by the host translation units of libntt_b200.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include "../../include/ntt_b200.h"
#include "../../include/ntt_b200_tune.h"
#include "configs.h"
#include "fused_kernel.cuh"
#include "twiddle.h"

namespace nttb {

ntt_status_t fail(ntt_status_t st, const char* fmt, ...);
ntt_status_t cuda_fail(cudaError_t e, const char* what);

// Untuned default for (logN, direction); config_by_r1 matches a phase split.
const FusedConfig* default_config(int logN, bool fwd = true);
// ... for launches of a single polynomial (one polynomial per job).
const FusedConfig* default_single_config(int logN, bool fwd);
const FusedConfig* config_by_r1(int logN, int r1);
// Untuned cluster (scatter) configuration with np polynomials per job.
const FusedConfig* cluster_config(int logN, int np = 1);
const FusedConfig* config_by_index(int idx);
// Autotuned choice for (logN, limbs, direction) on the current device, or
// nullptr.
const FusedConfig* tuned_config(int logN, int limbs, bool fwd);
// Clusters of this configuration resident at once on the current device.
int config_resident_clusters(const FusedConfig* c, bool fwd, int schedule);
// One launch of a fused configuration under a schedule (NTT_SCHEDULE_*);
// lazy2: some modulus is >= 2^30 (the [0, 2q) range discipline for all).
// mul: the direct forward with the product epilogue (FusedArgs.src).
// Kernel variants of a configuration (FusedConfig's kern_* entries): the
// plain transforms; the direct forward with the product epilogue
// (FusedArgs.src), with the subtract-and-scale output (FusedArgs.sub), with
// the product by a resident spectrum (FusedArgs.spec); the transforms over
// compressed twiddle tables.
enum class KernelVariant { Plain, Mul, SubScale, MulSpec, Compressed };
ntt_status_t launch_fused(const FusedConfig* c, bool fwd, const FusedArgs& a, cudaStream_t s,
                          int schedule, bool lazy2, KernelVariant v = KernelVariant::Plain);
ntt_status_t validate_modulus(int logN, ModulusConfig m, ModulusRuntime* rt);
// Validates m and fills the twiddle-generation inputs of both directions
// (entries 0/1 carry the folded Montgomery / N^{-1} R^{-1} factors).
ntt_status_t twiddle_gen_inputs(int logN, ModulusConfig m, TwGenLimb* fwd, TwGenLimb* inv);
// One launch over `polys` polynomials of `limbs` limbs (cfg == nullptr: the
// single-CTA small-size kernel).  status: optional device error word.
// mul_src (fused forward only): transform mul_src (same shape and stride)
// instead and store the Montgomery product of each output word with the
// spectrum word already at its place in `a`.
// scale (optional, device, one constant per limb): forward of c * x, or
// c * inverse, folded into the limb's stage 0.
// ops (optional): the limb map and the subtract-and-scale output of the
// ModUp / ModDown forwards (FusedArgs), the spectrum of the spectrum
// product, and whether `tw` is a compressed table (tw_comp_* layout);
// `limbs` counts the launch's limbs (the table's limbs minus skip_len).
struct LimbOps {
    uint32_t skip_at = 0, skip_len = 0;
    const uint32_t* sub = nullptr;
    size_t sub_stride = 0;
    uint32_t sub_begin = 0, sub_end = 0;
    const uint32_t* sub_mul = nullptr;
    bool compressed = false;
    const uint32_t* spec = nullptr;  // the spectrum the forward's output is multiplied by
    size_t spec_stride = 0;
    bool small_shared = false;  // logN 6..9: the shared-memory kernel, not the warp one
};
ntt_status_t run_transform(int logN, const FusedConfig* cfg, const TwPair* tw, const uint32_t* q,
                           int limbs, uint32_t* a, size_t polys, size_t stride, bool fwd,
                           cudaStream_t s, uint32_t* status, int schedule, bool lazy2,
                           const uint32_t* mul_src = nullptr, const uint32_t* scale = nullptr,
                           const LimbOps* ops = nullptr);

}  // namespace nttb
