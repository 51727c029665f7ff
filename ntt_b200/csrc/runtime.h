// Internal interfaces shared by the host translation units of libntt_b200.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include "../../include/ntt_b200.h"
#include "configs.h"
#include "fused_kernel.cuh"

namespace nttb {

ntt_status_t fail(ntt_status_t st, const char* fmt, ...);
ntt_status_t cuda_fail(cudaError_t e, const char* what);

const FusedConfig* default_config(int logN);
const FusedConfig* config_by_r1(int logN, int r1);
const FusedConfig* config_by_index(int idx);
// Autotuned choice for (logN, limbs) on the current device, or nullptr.
const FusedConfig* tuned_config(int logN, int limbs);
ntt_status_t launch_fused(const FusedConfig* c, bool fwd, const FusedArgs& a, cudaStream_t s);
ntt_status_t validate_modulus(int logN, ModulusConfig m, ModulusRuntime* rt);
// One launch over `polys` polynomials of `limbs` limbs (cfg == nullptr: the
// single-CTA small-size kernel).
ntt_status_t run_transform(int logN, const FusedConfig* cfg, const TwPair* tw, const uint32_t* q,
                           int limbs, uint32_t* a, size_t polys, size_t stride, bool fwd,
                           cudaStream_t s);

}  // namespace nttb
