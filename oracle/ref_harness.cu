// Include-harness around the reference's own v04 source file.
//
// TEST INFRASTRUCTURE ONLY (the checker, never the product).  It compiles the
// reference translation unit unchanged from where it lies (the path comes in
// through -DNTT_REF_SRC, see oracle/Makefile), renames its main(), and exports
// C entry points over its host functions and its launchers, so that:
//   * the C restatement in oracle/ntt_oracle.c is pinned against the
//     reference's own cpu_ntt_butterfly / cpu_intt_butterfly /
//     make_modulus_runtime / make_twiddle_table / fill_random;
//   * the reference CPU path can be timed on the GPU host (bench.py
//     --impl reference, cpu_baseline kind "reference");
//   * the reference's own sm_100a build of launch_ntt / launch_intt
//     (DefaultNTTLaunchConfig<16>) gives a third parity reference on a B200.
// Output goes to oracle/_ref/ only (git-ignored).
#include <cstdint>
#include <cstddef>
#include <thread>
#include <vector>

#define main ntt_reference_main
#include NTT_REF_SRC
#undef main

extern "C" {

// make_modulus_runtime (v04:681-718).  The reference calls std::exit on an
// invalid modulus/root; callers of this harness only pass validated configs.
void ref_modulus_runtime(int logN, uint32_t qi, uint32_t g, uint32_t out[8]) {
    ModulusRuntime r = make_modulus_runtime(logN, ModulusConfig{qi, g});
    out[0] = r.qi; out[1] = r.primitive_root; out[2] = r.q_inv; out[3] = r.r2;
    out[4] = r.psi; out[5] = r.psi_inv; out[6] = r.omega; out[7] = r.degree_inv;
}

void ref_twiddle_table(int logN, uint32_t q, uint32_t psi, uint32_t* out) {
    std::vector<uint32_t> t = make_twiddle_table(logN, q, psi);
    for (size_t i = 0; i < t.size(); ++i) out[i] = t[i];
}

void ref_fill_random(uint32_t* arr, size_t size, uint32_t q) { fill_random(arr, size, q); }

uint32_t ref_to_mont(uint32_t x, uint32_t q) { return to_mont(x, q); }
uint32_t ref_from_mont(uint32_t x, uint32_t q, uint32_t q_inv) { return from_mont(x, q, q_inv); }

void ref_cpu_ntt(uint32_t* a, int logN, uint32_t q, const uint32_t* psi) {
    cpu_ntt_butterfly(a, logN, q, psi);
}

void ref_cpu_intt(uint32_t* a, int logN, uint32_t q, const uint32_t* inv_psi, uint32_t degree_inv) {
    cpu_intt_butterfly(a, logN, q, inv_psi, degree_inv);
}

// Limbs split across `threads` host threads, each calling the reference's
// unchanged cpu_ntt_butterfly / cpu_intt_butterfly (degree_inv == nullptr
// selects the forward transform).
void ref_cpu_transform_limbs(uint32_t* a, int logN, int limbs, const uint32_t* q,
                             const uint32_t* tables, const uint32_t* degree_inv,
                             int threads) {
    size_t N = size_t{1} << logN;
    if (threads < 1) threads = 1;
    if (threads > limbs) threads = limbs;
    auto work = [&](int t) {
        for (int l = t; l < limbs; l += threads) {
            if (degree_inv)
                cpu_intt_butterfly(a + l * N, logN, q[l], tables + l * N, degree_inv[l]);
            else
                cpu_ntt_butterfly(a + l * N, logN, q[l], tables + l * N);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
}

// The reference's own GPU launchers at logN = 16 with its default phase
// triples, on caller-owned device buffers (legacy default stream, as in v04).
int ref_gpu_launch_ntt16(uint32_t* A, const uint32_t* tw, const uint32_t* moduli,
                         const uint32_t* q_inv, const uint32_t* r2, size_t limbs) {
    launch_ntt<DefaultNTTLaunchConfig<16>>(A, tw, moduli, q_inv, r2, limbs);
    return (int)cudaDeviceSynchronize();
}

int ref_gpu_launch_intt16(uint32_t* A, const uint32_t* itw, const uint32_t* moduli,
                          const uint32_t* q_inv, const uint32_t* dinv, size_t limbs) {
    launch_intt<DefaultNTTLaunchConfig<16>>(A, itw, moduli, q_inv, dinv, limbs);
    return (int)cudaDeviceSynchronize();
}

// Device time (CUDA events, legacy default stream, as v04:980-998) of the
// reference's per-call path at logN = 16 over `polys` packed polynomials of
// `limbs` limbs at A: one launch_ntt (then, separately, launch_intt) call per
// polynomial, averaged over `iters` passes after one warm-up pass.  With
// `restore` non-null every call is preceded by the reference's device-to-
// device copy of that polynomial from `restore` (v04:984).  Returns the
// CUDA error code; ms_* receive milliseconds per pass over all polynomials.
int ref_gpu_time16(uint32_t* A, const uint32_t* restore, const uint32_t* tw,
                   const uint32_t* itw, const uint32_t* moduli, const uint32_t* q_inv,
                   const uint32_t* r2, const uint32_t* dinv, size_t limbs, int polys,
                   int iters, float* ms_ntt, float* ms_intt) {
    const size_t words = limbs << 16;
    auto pass = [&](bool fwd) {
        for (int p = 0; p < polys; ++p) {
            uint32_t* a = A + (size_t)p * words;
            if (restore)
                cudaMemcpy(a, restore + (size_t)p * words, words * 4, cudaMemcpyDeviceToDevice);
            if (fwd) launch_ntt<DefaultNTTLaunchConfig<16>>(a, tw, moduli, q_inv, r2, limbs);
            else launch_intt<DefaultNTTLaunchConfig<16>>(a, itw, moduli, q_inv, dinv, limbs);
        }
    };
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float* out[2] = {ms_ntt, ms_intt};
    for (int d = 0; d < 2; ++d) {
        pass(d == 0);
        cudaEventRecord(e0);
        for (int i = 0; i < iters; ++i) pass(d == 0);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        *out[d] = ms / (float)iters;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return (int)cudaDeviceSynchronize();
}

}  // extern "C"
