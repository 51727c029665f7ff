// Integer-multiply throughput of the current device, measured (the
// denominator of the transforms' integer roofline).
//
// Every thread runs 8 independent chains of Shoup products -- the
// transforms' multiply mix: one 32-bit multiply-high and two multiply-lows
// per product -- so the measurement is bound by the multiply pipe, not by
// latency.  Result: 32-bit multiplies per second over the whole device.
#include <cuda_runtime.h>

#include "../../include/ntt_b200.h"
#include "arith.cuh"
#include "runtime.h"

namespace nttb {

constexpr int kChains = 8;
constexpr int kMulsPerProduct = 3;

__global__ void __launch_bounds__(256) imad_peak_kernel(uint32_t* out, uint32_t iters,
                                                        uint32_t w, uint32_t wp, uint32_t q) {
    uint32_t x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 7919u + c * 104729u + blockIdx.x;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = shoup_mul(x[c], w, wp, q);
    }
    uint32_t acc = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc ^= x[c];
    if (acc == 0x9E3779B9u) out[0] = acc;  // keeps the chains live
}

}  // namespace nttb

using namespace nttb;

extern "C" ntt_status_t ntt_measure_int_peak(double* muls_per_second) {
    if (!muls_per_second) return fail(NTT_ERR_INVALID_ARGUMENT, "NULL output");
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint32_t* out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t s = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&out, 4);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float ms = 0;
    const uint32_t iters = 4096;
    const unsigned blocks = (unsigned)sms * 8;
    const uint32_t q = 974258177u, w = 123456789u;
    const uint32_t wp = shoup_companion(w, q);
    if (e == cudaSuccess) {
        imad_peak_kernel<<<blocks, 256, 0, s>>>(out, 64, w, wp, q);  // warm-up
        cudaEventRecord(e0, s);
        imad_peak_kernel<<<blocks, 256, 0, s>>>(out, iters, w, wp, q);
        cudaEventRecord(e1, s);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    if (out) cudaFree(out);
    if (e != cudaSuccess) return cuda_fail(e, "integer peak measurement");
    const double muls = (double)blocks * 256 * kChains * iters * kMulsPerProduct;
    *muls_per_second = muls / (ms * 1e-3);
    return NTT_OK;
}
