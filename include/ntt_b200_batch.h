/*
 * ntt_b200 ragged batches (C ABI): many polynomials of different sizes,
 * limb counts, modulus chains and operations in ONE persistent launch.
 *
 * No reference counterpart: the reference transforms one polynomial per
 * launch_ntt<LC> / launch_intt<LC> call (src/v04_montgomery.cu:603-658) with
 * a compile-time logN.  A batch replaces a host loop of such calls.  Each
 * (polynomial, limb) becomes a tile; resident thread-block clusters drain a
 * device-side queue of tile groups.  Per tile the results are bit-identical
 * to ntt_forward / ntt_inverse of a plan with the same modulus.
 *
 * Operations (per job, on caller-owned device memory, limb-major
 * data[limb * 2^logN + i], 16-byte aligned):
 *   NTT_OP_FORWARD   data <- NTT(data)              (as ntt_forward)
 *   NTT_OP_INVERSE   data <- INTT(data)             (as ntt_inverse)
 *   NTT_OP_MULTIPLY  data <- a * data  negacyclic, mod each q, normal domain
 *                    in and out: INTT(NTT(a) (.) NTT(data)) with (.) the
 *                    pointwise Montgomery product; a = operand, read only.
 *   NTT_OP_MULTIPLY_SPECTRUM  data <- INTT(A (.) NTT(data)): the same product
 *                    with the operand given as its spectrum A = NTT(a) (a
 *                    forward output, e.g. kept resident), two transforms.
 * Twiddle tables are generated on the device once per (device, logN,
 * modulus) and kept resident in a process-wide registry shared by all
 * batches.  Jobs of one batch must not overlap in memory (operands may be
 * shared).  logN 12..17.
 */
#ifndef NTT_B200_BATCH_H
#define NTT_B200_BATCH_H
#include "ntt_b200.h"
#ifdef __cplusplus
extern "C" {
#endif

#define NTT_OP_FORWARD 0
#define NTT_OP_INVERSE 1
#define NTT_OP_MULTIPLY 2
#define NTT_OP_MULTIPLY_SPECTRUM 3

#define NTT_BATCH_MIN_LOGN 12
#define NTT_BATCH_MAX_LOGN 17

typedef struct ntt_job {
    int op;                        /* NTT_OP_* */
    int logN;                      /* 12..17 */
    int limbs;                     /* >= 1 */
    const ModulusConfig* moduli;   /* host array [limbs]: the job's modulus chain */
    uint32_t* data;                /* device, limbs * 2^logN words, in place */
    const uint32_t* operand;       /* multiplies: the other factor (device, same shape;
                                      its spectrum for NTT_OP_MULTIPLY_SPECTRUM);
                                      otherwise NULL */
} ntt_job_t;

typedef struct ntt_batch_options {
    int cluster_ctas; /* CTAs per cluster: 8, 16, or 0 = automatic (16 when a
                         job has logN 17, else 8) */
    int use_graph;    /* nonzero: ntt_batch_run replays a CUDA graph (default);
                         zero: a plain kernel launch */
    int max_clusters; /* cap on resident clusters (0 = as many as fit) */
} ntt_batch_options_t;

typedef struct ntt_batch_info {
    int jobs;
    int tiles;          /* (polynomial, limb) tiles */
    int groups;         /* tile groups in the device queue */
    int cluster_ctas;
    int clusters;       /* clusters launched (persistent) */
    int multiply;       /* nonzero: the kernel variant with multiply tiles */
    uint32_t smem_bytes;/* dynamic shared memory per CTA */
    size_t device_bytes;/* descriptors owned by the batch */
} ntt_batch_info_t;

typedef struct ntt_batch ntt_batch_t;

/* Validates every job (moduli as ntt_plan_create does), generates missing
 * twiddle tables on the current device, packs the tiles into groups and
 * uploads the descriptors.  Synchronous.  opts may be NULL. */
NTT_API ntt_status_t ntt_batch_create(const ntt_job_t* jobs, int count,
                                      const ntt_batch_options_t* opts, ntt_batch_t** out);
/* One persistent launch over every tile of the batch on `stream` (the
 * descriptors stay valid, so a batch can be run again on new contents of
 * the same buffers).  Runs of one batch must not overlap in time. */
NTT_API ntt_status_t ntt_batch_run(ntt_batch_t* batch, ntt_stream_t stream);
NTT_API ntt_status_t ntt_batch_get_info(const ntt_batch_t* batch, ntt_batch_info_t* out);
/* Frees the batch's descriptors (waits for its launches to finish). */
NTT_API ntt_status_t ntt_batch_destroy(ntt_batch_t* batch);
/* create + run + wait + destroy. */
NTT_API ntt_status_t ntt_batch_submit(const ntt_job_t* jobs, int count, ntt_stream_t stream);

/* Allocation-free variant of ntt_batch_submit (no reference counterpart:
 * the reference allocates nothing per call but also batches nothing).
 * For callers that must not allocate device memory while they run -- code
 * living inside a fixed, pre-sized memory reservation, or a latency-critical
 * loop where cudaMalloc / cudaFree would synchronise the device -- it runs
 * the batch kernel with its descriptors in a fixed 464 KiB scratch array
 * compiled into the library instead of allocated buffers.
 * Limits: at most NTT_NOALLOC_MAX_TILES (polynomial, limb) tiles per call
 * (NTT_ERR_UNSUPPORTED beyond); every modulus's tables must already be
 * resident (ntt_tables_preload beforehand, else NTT_ERR_NOT_READY).  The
 * scratch holds one call, so calls must not overlap on the device: issue
 * them on one stream or wait between them -- overlapping calls race.  The
 * scratch's group counter must be zero at kernel start; each call zeroes it
 * on `stream` itself.  The first call on a device looks up the scratch's
 * address (one-time set-up); make it before any stream capture.  The
 * descriptors are staged through one host area that the next call
 * overwrites, so a call on a stream that is capturing a graph returns
 * NTT_ERR_UNSUPPORTED.  The call keeps pointers to the resident tables
 * without holding them: do not call ntt_tables_trim while calls are in
 * flight.  Does not wait for the kernel. */
#define NTT_NOALLOC_MAX_TILES 4096
NTT_API ntt_status_t ntt_batch_run_noalloc(const ntt_job_t* jobs, int count, ntt_stream_t stream);

/* Resident twiddle-table registry: bytes held on the current device, and a
 * release of every table no live batch or server uses. */
NTT_API size_t ntt_tables_device_bytes(void);
/* Generates (if missing) the tables of `count` moduli for logN on the
 * current device and keeps them in the registry, so that a later batch or
 * request naming them does not pay for their generation. */
NTT_API ntt_status_t ntt_tables_preload(int logN, const ModulusConfig* moduli, int count);
NTT_API void ntt_tables_trim(void);

#ifdef __cplusplus
}
#endif
#endif
