// Allocation-free entry point of the ragged-batch kernel
// (ntt_batch_run_noalloc, include/ntt_b200_batch.h).
//
// ntt_batch_create allocates the device descriptors of a batch (tiles, tile
// groups, group counter) with cudaMalloc.  This entry point runs the same
// kernel with those descriptors in a fixed scratch array compiled into the
// library, so a call allocates no device memory.  It is meant for callers
// that must not allocate while they run: code that works inside a fixed,
// pre-sized memory reservation (where an allocation may fail or evict
// something), and latency-critical loops, where cudaMalloc / cudaFree can
// synchronise the device and stall unrelated streams.
//
// Limits and rules:
//  * at most kMaxTiles (polynomial, limb) tiles per call; larger job lists
//    are rejected with NTT_ERR_UNSUPPORTED before any device work;
//  * the twiddle tables of every modulus must already be resident (make
//    them so with ntt_tables_preload, which does allocate, beforehand);
//    otherwise NTT_ERR_NOT_READY;
//  * the scratch holds one call's descriptors, so calls must not overlap in
//    time on the device: issue them on one stream (or wait for one before
//    issuing the next on another); overlapping calls race on the scratch;
//  * the group counter at the end of the scratch must be zero when the
//    kernel starts; every call zeroes it with cudaMemsetAsync on its stream;
//  * the first call on each device looks the scratch's device address up
//    (cudaGetSymbolAddress, which may load this file's device code); make
//    that first call before any stream capture;
//  * the descriptors are staged through one static host area that the next
//    call overwrites, so a call on a stream that is being captured into a
//    graph is refused (NTT_ERR_UNSUPPORTED): a captured copy would read that
//    area again at every replay, by then holding another call's descriptors;
//  * the call keeps raw pointers to the registry's tables without holding
//    them, so ntt_tables_trim must not run while calls are in flight;
//  * the descriptors are staged through pageable host memory, so the call
//    returns once earlier work on `stream` has drained far enough for the
//    driver to take the copy.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/ntt_b200_batch.h"
#include "batch_rt.h"
#include "runtime.h"

using namespace nttb;

namespace {

constexpr uint32_t kMaxTiles = NTT_NOALLOC_MAX_TILES;
constexpr uint32_t kMaxCluster = 16;
constexpr size_t kTileBytes = (size_t)kMaxTiles * sizeof(BatchTile);
constexpr size_t kSlotBytes = (size_t)kMaxTiles * kMaxCluster * 4;  // groups <= tiles
constexpr size_t kRoundBytes = (size_t)kMaxTiles * 4;
constexpr size_t kScratchBytes = kTileBytes + kSlotBytes + kRoundBytes + 256;
static_assert(kTileBytes % 256 == 0 && kSlotBytes % 256 == 0 && kRoundBytes % 256 == 0,
              "scratch sections stay 256-byte aligned");

// Device scratch: tiles | group slots | group rounds | group counter (464 KiB).
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Host staging of the same layout (static: no heap either).
struct HostStage {
    BatchTile tiles[kMaxTiles];
    uint32_t order[kMaxTiles];
    uint32_t slots[kMaxTiles * kMaxCluster];
    uint32_t rounds[kMaxTiles];
};
HostStage g_host;
std::mutex g_mu;  // guards g_host and g_scratch_ptr
constexpr int kMaxDevices = 64;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch on `dev` (current device), looked up once.
ntt_status_t scratch_ptr(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kMaxDevices) return fail(NTT_ERR_UNSUPPORTED, "device %d", dev);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "scratch address (cudaGetSymbolAddress)");
        g_scratch_ptr[dev] = (unsigned char*)p;
    }
    *out = g_scratch_ptr[dev];
    return NTT_OK;
}

// Tile order by (rounds, logN) descending, then the same first-fit group
// filling as the allocating path, into the static arrays.  Returns groups.
uint32_t pack_static(uint32_t ntiles, int cl) {
    uint32_t n = 0;
    for (int r = 3; r >= 1; --r)
        for (int lg = kBatchMaxLogN; lg >= kBatchMinLogN; --lg)
            for (uint32_t t = 0; t < ntiles; ++t)
                if ((int)batch_op_rounds(g_host.tiles[t].op) == r && (int)g_host.tiles[t].logn == lg)
                    g_host.order[n++] = t;
    uint32_t groups = 0;
    int pos = cl;
    uint32_t cur = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t t = g_host.order[i];
        const int size = 1 << batch_tile_clog((int)g_host.tiles[t].logn);
        const uint32_t r = batch_op_rounds(g_host.tiles[t].op);
        if (pos + size > cl || r != cur) {
            for (int k = 0; k < cl; ++k) g_host.slots[(size_t)groups * cl + k] = kIdleSlot;
            g_host.rounds[groups++] = r;
            cur = r;
            pos = 0;
        }
        uint32_t* g = g_host.slots + (size_t)(groups - 1) * cl;
        for (int k = 0; k < size; ++k) g[pos + k] = t | ((uint32_t)k << kSlotSubShift);
        pos += size;
    }
    return groups;
}

}  // namespace

extern "C" ntt_status_t ntt_batch_run_noalloc(const ntt_job_t* jobs, int count,
                                              ntt_stream_t stream) {
    if (count < 0 || (count > 0 && !jobs)) return fail(NTT_ERR_INVALID_ARGUMENT, "bad job array");
    uint64_t ntiles = 0;
    int max_logn = 0;
    for (int j = 0; j < count; ++j) {
        const ntt_job_t& J = jobs[j];
        if (J.op != NTT_OP_FORWARD && J.op != NTT_OP_INVERSE && J.op != NTT_OP_MULTIPLY &&
            J.op != NTT_OP_MULTIPLY_SPECTRUM)
            return fail(NTT_ERR_INVALID_ARGUMENT, "job %d: unknown op %d", j, J.op);
        if (J.logN < NTT_BATCH_MIN_LOGN || J.logN > NTT_BATCH_MAX_LOGN)
            return fail(NTT_ERR_UNSUPPORTED, "job %d: logN %d outside [%d, %d]", j, J.logN,
                        NTT_BATCH_MIN_LOGN, NTT_BATCH_MAX_LOGN);
        if (J.limbs < 1 || !J.moduli || !J.data)
            return fail(NTT_ERR_INVALID_ARGUMENT, "job %d: needs limbs, moduli and data", j);
        if ((uintptr_t)J.data % 16)
            return fail(NTT_ERR_MISALIGNED, "job %d: data must be 16-byte aligned", j);
        if (batch_op_is_multiply((uint32_t)J.op)) {
            if (!J.operand) return fail(NTT_ERR_INVALID_ARGUMENT, "job %d: multiply needs an operand", j);
            if ((uintptr_t)J.operand % 16)
                return fail(NTT_ERR_MISALIGNED, "job %d: operand must be 16-byte aligned", j);
        }
        if (J.logN > max_logn) max_logn = J.logN;
        ntiles += (uint64_t)J.limbs;
    }
    if (ntiles > kMaxTiles)
        return fail(NTT_ERR_UNSUPPORTED, "%llu tiles: the allocation-free entry point takes at most %u",
                    (unsigned long long)ntiles, kMaxTiles);
    if (ntiles == 0) return NTT_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return cuda_fail(cudaGetLastError(), "cudaGetDevice");
    const int cl = max_logn >= 17 ? 16 : 8;
    const cudaStream_t s = (cudaStream_t)stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaError_t e = cudaStreamIsCapturing(s, &cap); e != cudaSuccess)
        return cuda_fail(e, "cudaStreamIsCapturing");
    if (cap != cudaStreamCaptureStatusNone)
        return fail(NTT_ERR_UNSUPPORTED,
                    "the allocation-free entry point stages its descriptors in one host area "
                    "that the next call overwrites; it cannot run on a capturing stream");

    std::lock_guard<std::mutex> lk(g_mu);
    unsigned char* scratch = nullptr;
    if (ntt_status_t st = scratch_ptr(dev, &scratch)) return st;
    uint32_t t = 0;
    for (int j = 0; j < count; ++j) {
        const ntt_job_t& J = jobs[j];
        const size_t N = size_t{1} << J.logN;
        for (int l = 0; l < J.limbs; ++l, ++t) {
            const TwPair *fwd = nullptr, *inv = nullptr;
            uint32_t nqinv = 0;
            if (!find_resident_table(dev, J.logN, J.moduli[l], &fwd, &inv, &nqinv))
                return fail(NTT_ERR_NOT_READY,
                            "job %d limb %d: tables of q=%u (logN %d) are not resident; "
                            "preload them with ntt_tables_preload",
                            j, l, J.moduli[l].qi, J.logN);
            BatchTile& b = g_host.tiles[t];
            b.data = J.data + (size_t)l * N;
            b.operand = batch_op_is_multiply((uint32_t)J.op) ? J.operand + (size_t)l * N : nullptr;
            b.tw_fwd = fwd;
            b.tw_inv = inv;
            b.q = J.moduli[l].qi;
            b.qinv = nqinv;
            b.logn = (uint32_t)J.logN;
            b.op = (uint32_t)J.op;
        }
    }
    const uint32_t groups = pack_static((uint32_t)ntiles, cl);
    BatchArgs a;
    a.tiles = (const BatchTile*)scratch;
    a.slots = (const uint32_t*)(scratch + kTileBytes);
    a.rounds = (const uint32_t*)(scratch + kTileBytes + kSlotBytes);
    a.counter = (uint32_t*)(scratch + kTileBytes + kSlotBytes + kRoundBytes);
    a.groups = groups;
    cudaError_t e = cudaMemcpyAsync(scratch, g_host.tiles, ntiles * sizeof(BatchTile),
                                    cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync((void*)a.slots, g_host.slots, (size_t)groups * cl * 4,
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync((void*)a.rounds, g_host.rounds, (size_t)groups * 4,
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.counter, 0, 4, s);
    if (e != cudaSuccess) return cuda_fail(e, "scratch upload");
    const BatchVariant v = batch_variant(g_host.tiles, (size_t)ntiles, cl);
    const int resident = batch_resident_clusters(v);
    if (resident <= 0) return fail(NTT_ERR_CUDA, "batch kernel: no resident clusters of %d CTAs", cl);
    return batch_launch(a, v, resident < (int)groups ? resident : (int)groups, s);
}
