#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "arith.cuh"

namespace nttb {
constexpr int kSmallMaxLogN = 9;
struct SmallArgs {
    uint32_t* data;
    const TwPair* tw;
    const uint32_t* q;
    uint32_t limbs;
    uint32_t jobs;
    unsigned long long poly_stride;
    int logN;
    const uint32_t* scale;  // optional per-limb constant folded into stage 0
    // limb map and subtract-and-scale output: as FusedArgs (fused_kernel.cuh)
    uint32_t skip_at, skip_len;
    const uint32_t* sub;
    unsigned long long sub_stride;
    uint32_t sub_begin, sub_end;
    const uint32_t* sub_mul;
};
cudaError_t launch_small(const SmallArgs& a, bool fwd, cudaStream_t s);
// Warp-per-limb kernel (warp.cu) for kWarpMinLogN <= logN <= kSmallMaxLogN:
// registers and shuffles, same results as launch_small.
constexpr int kWarpMinLogN = 6;
cudaError_t launch_warp(const SmallArgs& a, bool fwd, cudaStream_t s);
}  // namespace nttb
