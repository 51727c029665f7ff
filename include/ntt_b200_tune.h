/*
 * ntt_b200 autotuner and kernel-configuration catalogue (C ABI).
 *
 * Replaces the reference's compile-time phase-triple choice
 * (DefaultNTTLaunchConfig<LogN>, src/ntt_config.h:62-73) with a run-time
 * sweep over the compiled fused-kernel configurations, cached on disk.
 */
#ifndef NTT_B200_TUNE_H
#define NTT_B200_TUNE_H
#include "ntt_b200.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct ntt_kernel_config {
    int logN;
    int cluster_ctas;    /* CTAs per limb (thread-block cluster size)  */
    int r1;              /* phase-1 (column) stages; phase 2 = logN - r1 */
    int words_log2;      /* log2 words per thread per register pass    */
    int k1a;             /* stages of the first phase-1 register pass   */
    int k2a;             /* stages of the first phase-2 register pass   */
    int threads;         /* threads per CTA                             */
    uint32_t smem_bytes; /* dynamic shared memory per CTA               */
} ntt_kernel_config_t;

typedef struct ntt_tune_result {
    int config_index;
    double roundtrip_us; /* forward + inverse over the timed batch      */
    int candidates;
} ntt_tune_result_t;

NTT_API int ntt_config_count(void);
NTT_API ntt_status_t ntt_config_get(int index, ntt_kernel_config_t* out);
/* Time every compiled configuration for logN on `polys` polynomials of
 * `limbs` limbs (forward + inverse, `iters` repetitions), remember the
 * fastest for (device, logN, limb bucket) and write the on-disk cache.
 * Plans created afterwards use it when no phase split is requested. */
NTT_API ntt_status_t ntt_autotune(int logN, int limbs, int polys, int iters, ntt_tune_result_t* out);
/* Pin a plan to compiled configurations (indices into the catalogue above;
 * -1 keeps the current choice).  A tuning / debugging hook: results are
 * identical for every configuration. */
NTT_API ntt_status_t ntt_plan_force_config(ntt_plan_t* plan, int fwd_index, int inv_index);
/* Drop tuned entries for this process (plans fall back to defaults). */
NTT_API void ntt_autotune_forget(void);
/* Re-read the cache file on next use. */
NTT_API void ntt_autotune_reload(void);

#ifdef __cplusplus
}
#endif
#endif
