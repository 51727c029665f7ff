/*
 * ntt_b200 autotuner, schedules and kernel-configuration catalogue (C ABI).
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

/* Work distribution of a plan's transform launches (results never depend on
 * it). */
#define NTT_SCHEDULE_DIRECT 0 /* one limb per cluster, input from global memory  */
#define NTT_SCHEDULE_STAGED 1 /* resident clusters, next input bulk-copied ahead */

typedef struct ntt_kernel_config {
    int logN;
    int cluster_ctas;    /* CTAs per limb (thread-block cluster size)    */
    int r1;              /* phase-1 (column) stages; phase 2 = logN - r1 */
    int words_log2;      /* log2 words per thread per register pass      */
    int k1a;             /* stages of the first phase-1 register pass    */
    int k2a;             /* stages of the first phase-2 register pass    */
    int threads;         /* threads per CTA                              */
    uint32_t smem_bytes; /* dynamic shared memory per CTA (direct)       */
    int polys_per_job;   /* polynomials whose same limb one cluster
                            transforms together, sharing every twiddle
                            load (1, or 2 for the paired configurations) */
    int exchange;        /* how the limb's two phases meet: 0 = scatter into
                            the peers' shared memory (DSMEM), 1 = in place
                            through L2 (split kernels: phase 1 is one register
                            pass per column, phase 2 two or three passes)     */
    int k2b;             /* split kernels: stages of the second phase-2 pass */
} ntt_kernel_config_t;

typedef struct ntt_tune_result {
    int fwd_index;  /* fastest configuration for the forward transform */
    int inv_index;  /* ... and for the inverse                         */
    double fwd_us;  /* its time for one launch over the timed batch    */
    double inv_us;
    int candidates;
} ntt_tune_result_t;

NTT_API int ntt_config_count(void);
NTT_API ntt_status_t ntt_config_get(int index, ntt_kernel_config_t* out);
/* Thread-block clusters of configuration `index` resident at once on the
 * current device under `schedule`; -1 on error. */
NTT_API int ntt_config_resident_clusters(int index, int forward, int schedule);
/* Time every compiled configuration for logN on `polys` polynomials of
 * `limbs` limbs (forward and inverse separately, `iters` launches each),
 * remember the fastest of each direction for (device, logN, limb bucket)
 * and write the on-disk cache.  Plans created afterwards use them when no
 * phase split is requested. */
NTT_API ntt_status_t ntt_autotune(int logN, int limbs, int polys, int iters,
                                  ntt_tune_result_t* out);
/* The setters below (ntt_plan_force_config, ntt_plan_set_schedule,
 * ntt_plan_set_small_kernel, ntt_plan_set_multiply_form) change how later
 * calls on the plan launch; call them before the plan is shared between
 * threads, not while another thread launches through it.
 *
 * Pin a plan to compiled configurations (indices into the catalogue above;
 * -1 keeps the current choice).  A tuning / debugging hook: results are
 * identical for every configuration. */
NTT_API ntt_status_t ntt_plan_force_config(ntt_plan_t* plan, int fwd_index, int inv_index);
/* Work distribution of the plan's launches (NTT_SCHEDULE_*; default
 * NTT_SCHEDULE_DIRECT). */
NTT_API ntt_status_t ntt_plan_set_schedule(ntt_plan_t* plan, int schedule);
/* Kernel of the plan's launches at logN 6..9 (results identical):
 * NTT_SMALL_WARP (default): a warp per limb, the limb in registers, the last
 *   five stages pairing lanes through shfl.xor;
 * NTT_SMALL_SHARED: a CTA per limb, one shared-memory round and one barrier
 *   per stage (the path of logN 1..5). */
#define NTT_SMALL_WARP 0
#define NTT_SMALL_SHARED 1
NTT_API ntt_status_t ntt_plan_set_small_kernel(ntt_plan_t* plan, int kind);
/* Form of ntt_multiply_many on plans whose forward is a split configuration
 * (results identical):
 * NTT_MULTIPLY_ONE_LAUNCH: NTT(b), NTT(a), product and INTT per (pair, limb)
 *   in one launch of the split multiply kernel;
 * NTT_MULTIPLY_THREE_LAUNCHES: NTT(b) (split kernel), NTT(a) with the product
 *   folded into its store into b (a cluster kernel: a is only read), INTT(b)
 *   (split kernel); the default, measured faster on B200 (2.09 against
 *   2.37 ms for 128 pairs of 2^16 x 24 limbs).  Other plans always run the
 *   three-launch form. */
#define NTT_MULTIPLY_ONE_LAUNCH 0
#define NTT_MULTIPLY_THREE_LAUNCHES 1
NTT_API ntt_status_t ntt_plan_set_multiply_form(ntt_plan_t* plan, int form);
/* Self-test of the kernels' failure detection (no reference counterpart):
 * runs, on `stream`, the bounded mbarrier wait the transform kernels use,
 * on a barrier that nothing ever completes, with a limit of `limit` tries
 * (1..65536).  The wait gives up, the kernel returns normally and the
 * expiry is recorded in the plan's status word, so that the following
 * ntt_plan_check returns NTT_ERR_TIMEOUT.  The context stays usable. */
NTT_API ntt_status_t ntt_selftest_wait_expiry(const ntt_plan_t* plan, uint32_t limit,
                                              ntt_stream_t stream);
/* Drop tuned entries for this process (plans fall back to defaults). */
NTT_API void ntt_autotune_forget(void);
/* Re-read the cache file on next use. */
NTT_API void ntt_autotune_reload(void);

#ifdef __cplusplus
}
#endif
#endif
