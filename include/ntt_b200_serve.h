/*
 * ntt_b200 serving loop (C ABI): continuous batching of NTT / INTT /
 * negacyclic-multiply requests of mixed sizes under an HBM budget.
 *
 * No reference counterpart (the reference is a single-threaded benchmark
 * driver, src/v04_montgomery.cu main).  Requests carry host buffers; the
 * server copies each request's polynomial into a slot of its device arena,
 * runs every admitted request of a round in ONE persistent batch launch
 * (include/ntt_b200_batch.h: same kernels, same results as the plain path),
 * copies the results back and completes the tickets.  Several rounds are in
 * flight at once on separate streams: requests that arrive while others run
 * are admitted as soon as a stream and arena space are free, and their
 * copies and transforms overlap the running ones on the device.
 *
 * Requests may instead name device-resident buffers (device_buffers): they
 * are transformed where they lie, so only the device's own work counts.
 *
 * Memory: the arena (`hbm_budget_bytes`, reserved at creation) holds the
 * polynomials of admitted requests and the resident operands; a request
 * waits in FIFO order until its bytes fit.  Twiddle tables live in the
 * process-wide registry (ntt_tables_device_bytes) and are generated when a
 * request first names a modulus.  Host buffers should be pinned
 * (cudaHostAlloc / cudaHostRegister) for the copies to be asynchronous; they
 * must stay valid until the ticket completes.  All entry points are
 * thread-safe.
 */
#ifndef NTT_B200_SERVE_H
#define NTT_B200_SERVE_H
#include "ntt_b200_batch.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct ntt_server ntt_server_t;

typedef struct ntt_server_options {
    size_t hbm_budget_bytes; /* device arena; 0 = 80 GB (capped by free memory) */
    int streams;             /* rounds in flight at once; 0 = 4 */
    int max_round_tiles;     /* (polynomial, limb) tiles per launch; 0 = 1024 */
    int cluster_ctas;        /* 0 = automatic per round (8, or 16 with logN 17) */
    int max_round_requests;  /* requests per launch; 0 = no limit (1 with streams = 1
                                turns batching off: one request per launch, in order) */
} ntt_server_options_t;

typedef struct ntt_request {
    int op;                       /* NTT_OP_FORWARD / _INVERSE / _MULTIPLY / _MULTIPLY_SPECTRUM */
    int logN;                     /* 12..17 */
    int limbs;
    const ModulusConfig* moduli;  /* [limbs]; copied at submit */
    const uint32_t* input;        /* host, limbs * 2^logN words */
    const uint32_t* operand;      /* host: multiply's other factor, a spectrum for
                                     _MULTIPLY_SPECTRUM (or use operand_handle) */
    uint64_t operand_handle;      /* resident operand from ntt_server_put (0 = none) */
    uint32_t* output;             /* host, limbs * 2^logN words (may equal input) */
    int device_buffers;           /* nonzero: input, operand and output are device
                                     buffers on the server's device (16-byte aligned);
                                     the request runs on `output` in place (after a
                                     device copy of `input` when they differ), takes no
                                     arena space and moves nothing over PCIe */
} ntt_request_t;

typedef struct ntt_server_stats {
    uint64_t submitted, completed, failed;
    uint64_t rounds;              /* batch launches */
    double mean_round_requests;
    double p50_ms, p99_ms, mean_ms, max_ms; /* submit -> results in the host buffer */
    double elapsed_s;             /* first submit -> last completion */
    double limb_ntt_per_s;        /* completed limb transforms / elapsed (multiply = 3,
                                     spectrum multiply = 2) */
    size_t budget_bytes, arena_peak_bytes, resident_bytes, table_bytes;
} ntt_server_stats_t;

NTT_API ntt_status_t ntt_server_create(const ntt_server_options_t* opts, ntt_server_t** out);
/* Validates the request (moduli, sizes, budget) and queues it; never blocks
 * on the device.  NTT_ERR_BUDGET: the request alone exceeds the arena. */
NTT_API ntt_status_t ntt_server_submit(ntt_server_t* s, const ntt_request_t* req,
                                       uint64_t* ticket);
/* NTT_OK when done (results written), NTT_ERR_NOT_READY while pending, or
 * the request's error. */
NTT_API ntt_status_t ntt_server_poll(ntt_server_t* s, uint64_t ticket);
/* Blocks until done or `timeout_s` (< 0: no limit) passes (NTT_ERR_TIMEOUT). */
NTT_API ntt_status_t ntt_server_wait(ntt_server_t* s, uint64_t ticket, double timeout_s);
/* Latency of a completed ticket in milliseconds (-1 if not complete). */
NTT_API double ntt_server_latency_ms(ntt_server_t* s, uint64_t ticket);
/* Copies `words` host words into the arena as a resident operand. */
NTT_API ntt_status_t ntt_server_put(ntt_server_t* s, const uint32_t* host, size_t words,
                                    uint64_t* handle);
/* Copies a polynomial of `limbs` x 2^logN host words into the arena and
 * replaces it by its spectrum (forward transform), for
 * NTT_OP_MULTIPLY_SPECTRUM requests: each multiply by it then costs two
 * transforms instead of three.  Synchronous. */
NTT_API ntt_status_t ntt_server_put_spectrum(ntt_server_t* s, int logN,
                                             const ModulusConfig* moduli, int limbs,
                                             const uint32_t* host, uint64_t* handle);
NTT_API ntt_status_t ntt_server_drop(ntt_server_t* s, uint64_t handle);
/* reset != 0 clears the latency record and counters after reading. */
NTT_API ntt_status_t ntt_server_stats(ntt_server_t* s, int reset, ntt_server_stats_t* out);
/* Drains every queued and running request, then frees the server. */
NTT_API ntt_status_t ntt_server_destroy(ntt_server_t* s);

#ifdef __cplusplus
}
#endif
#endif
