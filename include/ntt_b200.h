/*
 * ntt_b200 -- RNS negacyclic NTT / INTT for NVIDIA B200 (sm_100a).
 *
 * C ABI of libntt_b200.so.  Plain pointers and sizes only; device pointers
 * are CUDA device addresses, streams are cudaStream_t passed as void*.
 * Every entry point returns an ntt_status_t (never exits the process);
 * ntt_last_error() gives the calling thread's detail string.
 *
 * Reference interfaces replaced (vnny27/NTT):
 *   src/ntt_config.h:6-29     ModulusConfig / PhaseConfig / TransformConfig
 *   src/v04_montgomery.cu:17-26    ModulusRuntime
 *   src/v04_montgomery.cu:660-740  host precompute (make_modulus_runtime,
 *                                  make_twiddle_table, to_mont, ...)
 *   src/v04_montgomery.cu:603-658  launch_ntt<LC> / launch_intt<LC>
 * The C++ drop-in spellings of the templates (DefaultNTTLaunchConfig<LogN>,
 * launch_ntt<LC>, ...) are in ntt_b200_config.hpp.
 *
 * Domain contract (identical to the reference's v04 path):
 *   forward: normal-domain input (any uint32, reduced mod q) -> Montgomery
 *            domain output (x * 2^32 mod q), bit-reversed order, in [0, q);
 *   inverse: Montgomery-domain input in [0, q), bit-reversed order ->
 *            normal-domain output in natural order, N^{-1} applied;
 *   layout:  limb-major, A[limb * N + i], in place.
 */
#ifndef NTT_B200_H
#define NTT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define NTT_API __attribute__((visibility("default")))
#else
#define NTT_API
#endif

#define NTT_B200_VERSION 100 /* 1.0.0 */
#define NTT_MIN_LOGN 1
#define NTT_MAX_LOGN 17

/* src/ntt_config.h:6-9 */
typedef struct ModulusConfig {
    uint32_t qi;
    uint32_t primitive_root;
} ModulusConfig;

/* src/ntt_config.h:12-16 (all log2 values) */
typedef struct PhaseConfig {
    int radix_stages;  /* radix-2 stages handled by this phase            */
    int stage_merging; /* stages merged in one register pass (max)        */
    int warp_batching; /* log2 contiguous words per thread at phase I/O  */
} PhaseConfig;

/* src/ntt_config.h:18-23 */
typedef struct TransformConfig {
    PhaseConfig ntt_phase1;
    PhaseConfig ntt_phase2;
    PhaseConfig intt_phase1;
    PhaseConfig intt_phase2;
} TransformConfig;

/* src/v04_montgomery.cu:17-26 */
typedef struct ModulusRuntime {
    uint32_t qi;
    uint32_t primitive_root;
    uint32_t q_inv;   /* -q^{-1} mod 2^32                 */
    uint32_t r2;      /* 2^64 mod q                       */
    uint32_t psi;     /* primitive 2N-th root of unity    */
    uint32_t psi_inv;
    uint32_t omega;   /* psi^2                            */
    uint32_t degree_inv; /* N^{-1} mod q (normal domain)  */
} ModulusRuntime;

typedef enum ntt_status {
    NTT_OK = 0,
    NTT_ERR_INVALID_ARGUMENT = 1,
    NTT_ERR_MODULUS = 2,          /* q != 1 mod 2N      (reference: exit, v04:685-689) */
    NTT_ERR_ROOT = 3,             /* not a 2N-th root   (reference: exit, v04:703-707) */
    NTT_ERR_MODULUS_RANGE = 4,    /* q even, composite, or >= 2^31                       */
    NTT_ERR_UNSUPPORTED = 5,      /* logN outside [NTT_MIN_LOGN, NTT_MAX_LOGN]           */
    NTT_ERR_MISALIGNED = 6,       /* device pointer not 16-byte aligned                  */
    NTT_ERR_CUDA = 7,             /* a CUDA runtime call failed (see ntt_last_error)    */
    NTT_ERR_OUT_OF_MEMORY = 8,
    NTT_ERR_BUDGET = 9,           /* request does not fit the server's memory budget    */
    NTT_ERR_TIMEOUT = 10,         /* bounded wait expired                               */
    NTT_ERR_CANCELLED = 11,
    NTT_ERR_NOT_READY = 12,
    NTT_ERR_SHUTDOWN = 13
} ntt_status_t;

typedef struct ntt_plan ntt_plan_t;
/* cudaStream_t; NULL = legacy default stream.  Calls run in stream order.
 * The launches of the transforms (except the small kernel of logN <= 5), of
 * ntt_pointwise_mul and of the 64-bit
 * variant use programmatic dependent launch: one may be scheduled while the
 * stream's previous kernel drains, but it touches no memory before that
 * kernel has completed, so the caller's own kernels in the stream need
 * nothing of it. */
typedef void* ntt_stream_t;

NTT_API int ntt_version(void);
NTT_API const char* ntt_status_string(ntt_status_t status);
/* Detail of the calling thread's most recent failure ("" if none). */
NTT_API const char* ntt_last_error(void);

/* ---- host precompute (mirrors of src/v04_montgomery.cu:660-740) -------- */

/* make_modulus_runtime (v04:681-718) with status codes instead of exit. */
NTT_API ntt_status_t ntt_modulus_runtime(int logN, ModulusConfig cfg, ModulusRuntime* out);
/* make_twiddle_table (v04:720-727): out[i] = root^bitrev(i, logN) mod q,
 * out must hold 2^logN words (host memory). */
NTT_API ntt_status_t ntt_twiddle_table_host(int logN, uint32_t q, uint32_t root, uint32_t* out);
/* default_moduli() (src/ntt_config.h:75-94): writes min(cap, 16) entries,
 * returns 16. */
NTT_API int ntt_default_moduli(ModulusConfig* out, int cap);
/* DefaultNTTLaunchConfig<LogN>::runtime_transform() (src/ntt_config.h:62-73). */
NTT_API ntt_status_t ntt_default_transform(int logN, TransformConfig* out);
/* The first `count` primes q >= lower_bound with q == 1 (mod 2N), ascending,
 * each with its smallest primitive root (no reference counterpart: the
 * reference hard-codes its moduli). */
NTT_API ntt_status_t ntt_find_moduli(int logN, int count, uint32_t lower_bound, ModulusConfig* out);

/* ---- plans ------------------------------------------------------------ */

typedef struct ntt_plan_info {
    int logN;
    int limbs;
    int cluster_ctas;       /* CTAs cooperating on one limb (DSMEM cluster)  */
    int threads_per_cta;
    uint32_t smem_bytes;    /* dynamic shared memory per CTA                */
    TransformConfig effective; /* the phase triples the kernels run          */
    size_t device_bytes;    /* twiddle tables + constants held by the plan  */
    int tuned;              /* 1 if the configuration came from the tuner   */
    int fwd_config;         /* catalogue index (ntt_config_get) of the      */
    int inv_config;         /* forward / inverse kernel; -1: small sizes    */
    int twiddle_entries;    /* (w, w') pairs per limb and direction: N, or
                               3N/16 + 16 with compressed tables            */
} ntt_plan_info_t;

/* Validates every (qi, primitive_root) exactly as make_modulus_runtime does
 * (plus q odd, prime and < 2^31), then builds device-resident Shoup twiddle
 * tables on the current CUDA device with a generation kernel.
 * transform: NULL = tuned or default configuration; otherwise its phase
 * split (radix_stages) must add up to logN and selects among the compiled
 * kernel configurations (results do not depend on it). */
NTT_API ntt_status_t ntt_plan_create(int logN, const ModulusConfig* moduli, int limbs,
                             const TransformConfig* transform, ntt_plan_t** out);

/* Plan options (flags of ntt_plan_create_ex). */
/* Compressed twiddle tables (Cheddar's on-the-fly twiddles, an MSB x LSB
 * table product: src/NTT_cheddar.cu:42-43, 80-84, 1283-1289): per limb and
 * direction 3N/16 + 16 pairs instead of N (5.3x fewer table bytes): the
 * entries of the first logN-4 stages, one base entry per run of 16 / 8 / 4 /
 * 2 consecutive entries of each of the last four stages, and 16 unit-step
 * factors; those stages multiply by the two factors in turn (two Shoup
 * products instead of one).  The trade: ~20% more integer multiplies per
 * transform for tables that stay in L2 when many limbs or moduli are in
 * flight.  logN >= 15 (the split kernels); such plans run ntt_forward /
 * ntt_inverse (_many, _scaled, _skip, _scaled_range) and return
 * NTT_ERR_UNSUPPORTED for ntt_forward_sub_scale and ntt_multiply_many.
 * Results are identical to those of a full-table plan. */
#define NTT_PLAN_COMPRESSED_TWIDDLES 1u
/* ntt_plan_create with option flags (0 = ntt_plan_create). */
NTT_API ntt_status_t ntt_plan_create_ex(int logN, const ModulusConfig* moduli, int limbs,
                                        const TransformConfig* transform, uint32_t flags,
                                        ntt_plan_t** out);
NTT_API ntt_status_t ntt_plan_destroy(ntt_plan_t* plan);
NTT_API ntt_status_t ntt_plan_get_info(const ntt_plan_t* plan, ntt_plan_info_t* out);
/* Waits for the device, then reads and clears the plan's device status word
 * (bit 0: a bounded wait inside a transform kernel expired -- returned as
 * NTT_ERR_TIMEOUT).  device_status may be NULL. */
NTT_API ntt_status_t ntt_plan_check(const ntt_plan_t* plan, uint32_t* device_status);
/* Device pointers of the plan's tables: limbs * N (w, w') uint32 pairs, with
 * entries 0 and 1 holding the constants folded into limb stage 0, and for
 * logN >= 10 the last four stages' blocks interleaved for coalesced loads:
 * stage logN-1-p (p = 0..3) starts at H = N / 2^(p+1), and its entry H + j
 * sits at slot H + (j % F) * (N/32) + j / F with F = 16 / 2^p. */
NTT_API ntt_status_t ntt_plan_tables(const ntt_plan_t* plan, const uint32_t** fwd_pairs,
                             const uint32_t** inv_pairs, const uint32_t** moduli);

/* In-place transforms of one polynomial (limbs * N words, 16-byte aligned). */
NTT_API ntt_status_t ntt_forward(const ntt_plan_t* plan, uint32_t* a_dev, ntt_stream_t stream);
NTT_API ntt_status_t ntt_inverse(const ntt_plan_t* plan, uint32_t* a_dev, ntt_stream_t stream);
/* `polys` polynomials, polynomial p at a_dev + p * poly_stride (words,
 * >= limbs * N, multiple of 4); one launch. */
NTT_API ntt_status_t ntt_forward_many(const ntt_plan_t* plan, uint32_t* a_dev, size_t polys,
                              size_t poly_stride, ntt_stream_t stream);
NTT_API ntt_status_t ntt_inverse_many(const ntt_plan_t* plan, uint32_t* a_dev, size_t polys,
                              size_t poly_stride, ntt_stream_t stream);
/* Transforms with a per-limb constant folded in, at no extra launch or pass
 * (Cheddar's NTTHandler multiplies by a per-limb constant inside its
 * transform kernels: the pre-multiply of NTTPhase1, src/NTT_cheddar.cu:286-293,
 * and INTTAndMultConst, src/NTT_cheddar.cu:743-813):
 *   ntt_forward_scaled: a <- NTT(c_l * a) per limb l;
 *   ntt_inverse_scaled: a <- c_l * INTT(a) per limb l.
 * scale: device array of `limbs` uint32 constants, normal domain (reduced
 * mod q_l).  The constant enters through the limb's stage-0 twiddle pair
 * (table entries 0 and 1, which already carry the Montgomery and N^{-1}
 * factors), so the cost is that of the plain transform.  Same layout,
 * alignment and polys / poly_stride rules as ntt_forward_many. */
NTT_API ntt_status_t ntt_forward_scaled(const ntt_plan_t* plan, uint32_t* a_dev, size_t polys,
                                        size_t poly_stride, const uint32_t* scale_dev,
                                        ntt_stream_t stream);
NTT_API ntt_status_t ntt_inverse_scaled(const ntt_plan_t* plan, uint32_t* a_dev, size_t polys,
                                        size_t poly_stride, const uint32_t* scale_dev,
                                        ntt_stream_t stream);
/* The NTT steps of RNS basis conversion (ModUp / ModDown), each one launch of
 * the plan's transform kernels, same layout and alignment rules as
 * ntt_forward_many; limb indices are the plan's.
 *
 * ntt_forward_skip (ModUp's forward; Cheddar's NTTForModUp,
 * src/NTT_cheddar.cu:886-955): the forward of every limb except
 * [skip_begin, skip_end), which the launch neither reads nor writes (the
 * limbs of the decomposition digit that are already in the NTT domain).
 *
 * ntt_forward_sub_scale (ModDown's forward; NTTForModDown and
 * NTTPhase2ForModDown, src/NTT_cheddar.cu:456-601, 957-1027): per limb l
 *   a_l <- (NTT(a_l) - d_k * s_l) * c_l   (mod q_l), canonical,
 * where s_l = sub_dev[p * sub_stride + k * N + i] with k = l - sub_begin
 * for sub_begin <= l < sub_end (s_l = 0 for the other limbs), in the
 * forward's output domain (Montgomery); c_l = scale_dev[l] (NULL: 1) and
 * d_k = sub_mul_dev[k] (NULL: 1, Cheddar's src2_padding) are normal-domain
 * constants.  c enters through stage 0 as in ntt_forward_scaled and the
 * subtraction of (c d) s rides on the final store, so HBM sees a read and
 * written once and s read once.  sub_stride 0 = packed (sub_end - sub_begin)
 * * N; sub_dev 16-byte aligned for logN >= 10 and must not overlap a_dev.
 *
 * ntt_inverse_scaled_range (INTTForModDown / INTTAndMultConst on part of the
 * basis, src/NTT_cheddar.cu:743-813, 1029-1128): a_l <- c_k * INTT(a_l) for
 * the limbs l in [limb_begin, limb_end) only, c_k = scale_dev[l -
 * limb_begin] (NULL: 1); the reference writes a separate buffer, this one
 * transforms in place. */
NTT_API ntt_status_t ntt_forward_skip(const ntt_plan_t* plan, uint32_t* a_dev, size_t polys,
                                      size_t poly_stride, int skip_begin, int skip_end,
                                      ntt_stream_t stream);
NTT_API ntt_status_t ntt_forward_sub_scale(const ntt_plan_t* plan, uint32_t* a_dev, size_t polys,
                                           size_t poly_stride, const uint32_t* sub_dev,
                                           size_t sub_stride, int sub_begin, int sub_end,
                                           const uint32_t* scale_dev, const uint32_t* sub_mul_dev,
                                           ntt_stream_t stream);
NTT_API ntt_status_t ntt_inverse_scaled_range(const ntt_plan_t* plan, uint32_t* a_dev,
                                              size_t polys, size_t poly_stride, int limb_begin,
                                              int limb_end, const uint32_t* scale_dev,
                                              ntt_stream_t stream);
/* c = a (.) b: pointwise Montgomery product of two forward outputs (x*2^32
 * domain) per limb modulus, giving the spectrum of the negacyclic product
 * for ntt_inverse.  Over `polys` polynomials (poly_stride words apart, 0 =
 * packed); 16-byte aligned; c may alias a or b.  No reference counterpart
 * (the middle step of an unfused negacyclic multiply). */
NTT_API ntt_status_t ntt_pointwise_mul(const ntt_plan_t* plan, uint32_t* c_dev,
                                       const uint32_t* a_dev, const uint32_t* b_dev, size_t polys,
                                       size_t poly_stride, ntt_stream_t stream);
/* b <- a * b, the negacyclic product per limb modulus (normal domain in and
 * out, canonical words), for `polys` pairs (poly_stride words apart, 0 =
 * packed; 16-byte aligned; a is read only and must not overlap b).  Three
 * launches: NTT(b) in place; NTT(a) with the pointwise Montgomery product
 * folded into its store into b (a cluster configuration, whose phases meet in
 * shared memory, so a is only read); INTT(b).  Plans whose forward is a split
 * configuration (logN 15..17) run the first and last with the split kernels,
 * and can run the whole product in one launch of the split multiply kernel
 * instead (ntt_plan_set_multiply_form, include/ntt_b200_tune.h; slower on
 * B200: 3 CTAs per SM for its two work buffers).  Either way the same result
 * as ntt_forward_many on both, ntt_pointwise_mul, then ntt_inverse_many.
 * logN >= 10.  No reference counterpart (the reference has no product). */
NTT_API ntt_status_t ntt_multiply_many(const ntt_plan_t* plan, const uint32_t* a_dev,
                                       uint32_t* b_dev, size_t polys, size_t poly_stride,
                                       ntt_stream_t stream);
/* b <- INTT(NTT(b) (.) a_spec) per limb: the negacyclic product of each b
 * with a polynomial whose spectrum a_spec (the plan's forward output:
 * Montgomery domain, bit-reversed, canonical) is already resident -- the
 * plaintext-times-ciphertext pattern of RNS schemes, where one operand is
 * transformed once and used many times.  Split plans (logN 15..17) run two
 * launches: the forward of b with the Montgomery product by the spectrum word
 * on its final store, then the inverse; other plans run forward,
 * ntt_pointwise_mul and inverse.  a_spec has b's shape and stride, is only
 * read and must not overlap b; 16-byte aligned.  No reference counterpart
 * (the reference has no multiply). */
NTT_API ntt_status_t ntt_multiply_spectrum_many(const ntt_plan_t* plan, const uint32_t* a_spec_dev,
                                                uint32_t* b_dev, size_t polys, size_t poly_stride,
                                                ntt_stream_t stream);
/* Diagnostic (no reference counterpart): 32-bit integer multiplies per second
 * the current device sustains on the transforms' multiply mix (Shoup
 * products: one multiply-high and two multiply-lows each), measured by a
 * short kernel -- the denominator of the integer-multiply roofline. */
NTT_API ntt_status_t ntt_measure_int_peak(double* muls_per_second);

/* ---- drop-in launchers (src/v04_montgomery.cu:603-658) -----------------
 * Same arguments and domain contract as launch_ntt<LC> / launch_intt<LC>:
 * caller-owned device buffers, the reference's Montgomery-form tables
 * (twiddle_dev[limb*N + i] = to_mont(psi^bitrev(i))), launched on the legacy
 * default stream.  phase1/phase2: the LC's NTT (or INTT) phase triples, or
 * NULL for DefaultNTTLaunchConfig<logN>.  The reference's kernels read these
 * tables at every launch; here each call first runs a refresh kernel on the
 * same stream that compares the caller's table words and per-limb moduli,
 * q_inv and r2 / degree_inv against shadow copies on the device and re-derives
 * the Shoup-form entries that changed, then the transform: a caller that
 * rewrites its tables in place (new moduli at the same addresses) gets the new
 * results, with no host synchronisation.  The first call with a given set of
 * pointers allocates the converted table and its shadows (cudaMalloc); later
 * calls allocate nothing.  Unlike the reference, errors are returned; a
 * modulus the refresh finds even or not below 2^31 is reported by
 * ntt_shim_check. */
NTT_API ntt_status_t ntt_launch_ntt(uint32_t* A_dev, const uint32_t* twiddle_dev,
                            const uint32_t* moduli_dev, const uint32_t* q_inv_dev,
                            const uint32_t* r2_dev, size_t limb_count, int logN,
                            const PhaseConfig* phase1, const PhaseConfig* phase2);
NTT_API ntt_status_t ntt_launch_intt(uint32_t* A_dev, const uint32_t* inv_twiddle_dev,
                             const uint32_t* moduli_dev, const uint32_t* q_inv_dev,
                             const uint32_t* degree_inv_dev, size_t limb_count, int logN,
                             const PhaseConfig* phase1, const PhaseConfig* phase2);
/* Frees the converted tables and shadows kept by the drop-in launchers. */
NTT_API void ntt_shim_cache_clear(void);
/* Synchronises and reports NTT_ERR_MODULUS_RANGE if a drop-in call since the
 * last check named a modulus that is even or not below 2^31 (the reference's
 * Montgomery range); clears the record. */
NTT_API ntt_status_t ntt_shim_check(void);

#ifdef __cplusplus
}
#endif
#endif /* NTT_B200_H */
