// Ragged batches: twiddle-table registry, tile packing, persistent launch
// and CUDA-graph replay (include/ntt_b200_batch.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <tuple>
#include <vector>

#include "../../include/ntt_b200_batch.h"
#include "batch_kernel.cuh"
#include "batch_rt.h"
#include "host_math.h"
#include "runtime.h"

namespace nttb {
extern const void* const kBatchKernel_c16[2];
extern const void* const kBatchKernel_c16m[2];
extern const void* const kBatchKernel_c8[2];
extern const void* const kBatchKernel_c8m[2];

#define NTT_CUDA_TRY(expr, what)                         \
    do {                                                 \
        cudaError_t e_ = (expr);                         \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

// ---------------------------------------------------------------------------
// Twiddle-table registry.  Tables are generated in slabs (all moduli of one
// logN missing at one request); a slab is freed when neither the registry
// nor any batch refers to it.
// ---------------------------------------------------------------------------
TableSlab::~TableSlab() {
    if (!block) return;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != device) cudaSetDevice(device);
    cudaFree(block);
    if (cur != device) cudaSetDevice(cur);
}

namespace {
std::mutex g_tab_mu;
// (device, logN, q, root) -> tables
std::map<std::tuple<int, int, uint32_t, uint32_t>, TableRef> g_tables;
}  // namespace

ntt_status_t acquire_tables(int logN, const ModulusConfig* mods, int count,
                            std::vector<TableRef>& out) {
    int dev = 0;
    NTT_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lk(g_tab_mu);
    out.assign(count, TableRef{});
    std::vector<int> miss;
    std::map<std::pair<uint32_t, uint32_t>, int> miss_idx;
    for (int i = 0; i < count; ++i) {
        auto it = g_tables.find({dev, logN, mods[i].qi, mods[i].primitive_root});
        if (it != g_tables.end()) {
            out[i] = it->second;
        } else if (!miss_idx.count({mods[i].qi, mods[i].primitive_root})) {
            miss_idx[{mods[i].qi, mods[i].primitive_root}] = (int)miss.size();
            miss.push_back(i);
        }
    }
    if (!miss.empty()) {
        const int m = (int)miss.size();
        std::vector<TwGenLimb> gen(2 * m);
        for (int j = 0; j < m; ++j)
            if (ntt_status_t st = twiddle_gen_inputs(logN, mods[miss[j]], &gen[j], &gen[m + j]))
                return st;
        const size_t N = size_t{1} << logN;
        auto slab = std::make_shared<TableSlab>();
        slab->device = dev;
        const size_t tab_bytes = 2 * (size_t)m * N * sizeof(TwPair);
        slab->bytes = tab_bytes + gen.size() * sizeof(TwGenLimb);
        // generation on a private non-blocking stream, synchronised alone:
        // no device-wide synchronisation, so running batches (a serving
        // loop's rounds) are not stalled; the generator inputs stay in the
        // slab (no cudaFree, which would synchronise the device)
        cudaStream_t gs = nullptr;
        cudaError_t e = cudaStreamCreateWithFlags(&gs, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaMalloc(&slab->block, slab->bytes);
        TwPair* fwd = (TwPair*)slab->block;
        TwPair* inv = fwd + (size_t)m * N;
        TwGenLimb* gdev = (TwGenLimb*)((char*)slab->block + tab_bytes);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(gdev, gen.data(), gen.size() * sizeof(TwGenLimb),
                                cudaMemcpyHostToDevice, gs);
        if (e == cudaSuccess) e = launch_twiddle_gen(fwd, gdev, m, logN, gs);
        if (e == cudaSuccess) e = launch_twiddle_gen(inv, gdev + m, m, logN, gs);
        if (e == cudaSuccess) e = cudaStreamSynchronize(gs);
        if (gs) cudaStreamDestroy(gs);
        if (e != cudaSuccess) {
            if (e == cudaErrorMemoryAllocation) {
                cudaGetLastError();
                return fail(NTT_ERR_OUT_OF_MEMORY, "twiddle tables: out of device memory");
            }
            return cuda_fail(e, "twiddle table generation");
        }
        for (int j = 0; j < m; ++j) {
            TableRef r{slab, fwd + (size_t)j * N, inv + (size_t)j * N, gen[j].q,
                       gen[j].nqinv};
            g_tables[{dev, logN, mods[miss[j]].qi, mods[miss[j]].primitive_root}] = r;
        }
        for (int i = 0; i < count; ++i)
            if (!out[i].slab) out[i] = g_tables[{dev, logN, mods[i].qi, mods[i].primitive_root}];
    }
    return NTT_OK;
}

bool find_resident_table(int dev, int logN, ModulusConfig m, const TwPair** fwd,
                         const TwPair** inv, uint32_t* nqinv) {
    std::lock_guard<std::mutex> lk(g_tab_mu);
    auto it = g_tables.find({dev, logN, m.qi, m.primitive_root});
    if (it == g_tables.end()) return false;
    *fwd = it->second.fwd;
    *inv = it->second.inv;
    *nqinv = it->second.nqinv;
    return true;
}

size_t tables_device_bytes(int dev) {
    std::lock_guard<std::mutex> lk(g_tab_mu);
    std::set<const TableSlab*> seen;
    size_t b = 0;
    for (auto& kv : g_tables)
        if (std::get<0>(kv.first) == dev && seen.insert(kv.second.slab.get()).second)
            b += kv.second.slab->bytes;
    return b;
}

void tables_trim() {
    std::lock_guard<std::mutex> lk(g_tab_mu);
    // keep slabs that a batch or server still holds (use_count > registry refs)
    std::map<const TableSlab*, long> reg_refs;
    for (auto& kv : g_tables) reg_refs[kv.second.slab.get()]++;
    for (auto it = g_tables.begin(); it != g_tables.end();) {
        const TableSlab* s = it->second.slab.get();
        if (it->second.slab.use_count() <= reg_refs[s]) it = g_tables.erase(it);
        else ++it;
    }
}

// ---------------------------------------------------------------------------
// Kernel variants.
// ---------------------------------------------------------------------------
BatchVariant batch_variant(const BatchTile* tiles, size_t n, int cluster_ctas) {
    BatchVariant v{cluster_ctas, false, false};
    uint32_t max_logn = 0;
    for (size_t i = 0; i < n; ++i) {
        v.mul |= batch_op_is_multiply(tiles[i].op);
        v.lazy2 |= tiles[i].q >= (1u << 30);
        max_logn = tiles[i].logn > max_logn ? tiles[i].logn : max_logn;
    }
    if (!v.cluster_ctas) v.cluster_ctas = max_logn >= 17 ? 16 : 8;
    return v;
}

const void* batch_kernel_fn(const BatchVariant& v) {
    const int k = v.lazy2 ? 1 : 0;
    if (v.cluster_ctas == 16) return v.mul ? kBatchKernel_c16m[k] : kBatchKernel_c16[k];
    return v.mul ? kBatchKernel_c8m[k] : kBatchKernel_c8[k];
}
uint32_t batch_kernel_smem(bool mul) {
    return mul ? batch_smem_bytes<true>() : batch_smem_bytes<false>();
}

namespace {
std::mutex g_bk_mu;
std::set<std::pair<int, const void*>> g_bk_ready;
std::map<std::pair<int, const void*>, int> g_bk_occ;
}  // namespace

// Resident clusters of a batch-kernel variant on the current device (sets
// the function attributes on first use).
int batch_resident_clusters(const BatchVariant& v) {
    const int cl = v.cluster_ctas;
    const void* fn = batch_kernel_fn(v);
    const uint32_t smem = batch_kernel_smem(v.mul);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    std::lock_guard<std::mutex> lk(g_bk_mu);
    auto key = std::make_pair(dev, fn);
    if (!g_bk_ready.count(key)) {
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return -1;
        if (cl > 8 &&
            cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                cudaSuccess)
            return -1;
        g_bk_ready.insert(key);
    }
    auto it = g_bk_occ.find(key);
    if (it != g_bk_occ.end()) return it->second;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(cl, 1, 1);
    lc.blockDim = dim3(kBatchThreads, 1, 1);
    lc.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, fn, &lc) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    g_bk_occ[key] = n;
    return n;
}

ntt_status_t batch_launch(const BatchArgs& a, const BatchVariant& v, int clusters, cudaStream_t s) {
    const int cl = v.cluster_ctas;
    const bool mul = v.mul;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(cl * clusters, 1, 1);
    lc.blockDim = dim3(kBatchThreads, 1, 1);
    lc.dynamicSmemBytes = batch_kernel_smem(mul);
    lc.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    BatchArgs copy = a;
    void* params[] = {&copy};
    NTT_CUDA_TRY(cudaLaunchKernelExC(&lc, batch_kernel_fn(v), params), "batch kernel launch");
    return NTT_OK;
}

// ---------------------------------------------------------------------------
// Packing: tiles sorted by (rounds, logN) descending, placed first-fit in
// aligned power-of-two CTA ranges.  With non-increasing sizes the fill
// position is always aligned, so a group is filled before the next opens;
// tiles of different round counts never share a group.
// ---------------------------------------------------------------------------
void pack_tiles(const std::vector<BatchTile>& tiles, int cl, std::vector<uint32_t>& slots,
                std::vector<uint32_t>& rounds) {
    std::vector<uint32_t> order(tiles.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (uint32_t)i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
        const uint32_t rx = batch_op_rounds(tiles[x].op), ry = batch_op_rounds(tiles[y].op);
        if (rx != ry) return rx > ry;
        return tiles[x].logn > tiles[y].logn;
    });
    slots.clear();
    rounds.clear();
    int pos = cl;  // no open group
    uint32_t cur_rounds = 0;
    for (uint32_t t : order) {
        const int size = 1 << batch_tile_clog((int)tiles[t].logn);
        const uint32_t r = batch_op_rounds(tiles[t].op);
        if (pos + size > cl || r != cur_rounds) {
            slots.insert(slots.end(), (size_t)cl, kIdleSlot);
            rounds.push_back(r);
            cur_rounds = r;
            pos = 0;
        }
        uint32_t* g = slots.data() + slots.size() - cl;
        for (int k = 0; k < size; ++k) g[pos + k] = t | ((uint32_t)k << kSlotSubShift);
        pos += size;
    }
}

}  // namespace nttb

using namespace nttb;

struct ntt_batch {
    int device = 0;
    int jobs = 0, cl = 8, clusters = 0;
    bool mul = false;
    BatchVariant variant{8, false, false};
    bool use_graph = true;
    std::vector<BatchTile> tiles;
    std::vector<uint32_t> slots, rounds;
    std::vector<std::shared_ptr<TableSlab>> slabs;
    void* block = nullptr;
    size_t bytes = 0;
    BatchArgs args{};
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap = nullptr;
};

static ntt_status_t batch_build(const ntt_job_t* jobs, int count, const ntt_batch_options_t* o,
                                ntt_batch_t** out) {
    if (!out) return fail(NTT_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (count < 0 || (count > 0 && !jobs)) return fail(NTT_ERR_INVALID_ARGUMENT, "bad job array");
    ntt_batch_options_t opt{0, 1, 0};
    if (o) opt = *o;
    if (opt.cluster_ctas != 0 && opt.cluster_ctas != 8 && opt.cluster_ctas != 16)
        return fail(NTT_ERR_INVALID_ARGUMENT, "cluster_ctas must be 0, 8 or 16");
    if (opt.max_clusters < 0) return fail(NTT_ERR_INVALID_ARGUMENT, "max_clusters < 0");
    int max_logn = 0;
    bool mul = false;
    size_t ntiles = 0;
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
            mul = true;
        }
        max_logn = std::max(max_logn, J.logN);
        ntiles += (size_t)J.limbs;
    }
    if (ntiles > kSlotTileMask) return fail(NTT_ERR_UNSUPPORTED, "more than 2^24 tiles");
    const int cl = opt.cluster_ctas ? opt.cluster_ctas : (max_logn >= 17 ? 16 : 8);
    if (max_logn >= 17 && cl < 16)
        return fail(NTT_ERR_UNSUPPORTED, "logN 17 tiles need 16-CTA clusters");
    auto* b = new ntt_batch();
    std::unique_ptr<ntt_batch> guard(b);
    NTT_CUDA_TRY(cudaGetDevice(&b->device), "cudaGetDevice");
    b->jobs = count;
    b->cl = cl;
    b->mul = mul;
    b->use_graph = opt.use_graph != 0;
    b->tiles.reserve(ntiles);
    std::set<const TableSlab*> held;
    std::vector<TableRef> refs;
    for (int j = 0; j < count; ++j) {
        const ntt_job_t& J = jobs[j];
        if (ntt_status_t st = acquire_tables(J.logN, J.moduli, J.limbs, refs)) return st;
        const size_t N = size_t{1} << J.logN;
        for (int l = 0; l < J.limbs; ++l) {
            BatchTile t;
            t.data = J.data + (size_t)l * N;
            t.operand = batch_op_is_multiply((uint32_t)J.op) ? J.operand + (size_t)l * N : nullptr;
            t.tw_fwd = refs[l].fwd;
            t.tw_inv = refs[l].inv;
            t.q = refs[l].q;
            t.qinv = refs[l].nqinv;
            t.logn = (uint32_t)J.logN;
            t.op = (uint32_t)J.op;
            b->tiles.push_back(t);
            if (held.insert(refs[l].slab.get()).second) b->slabs.push_back(refs[l].slab);
        }
    }
    pack_tiles(b->tiles, cl, b->slots, b->rounds);
    const size_t groups = b->rounds.size();
    const size_t t_bytes = (b->tiles.size() * sizeof(BatchTile) + 255) & ~size_t{255};
    const size_t s_bytes = (b->slots.size() * 4 + 255) & ~size_t{255};
    const size_t r_bytes = (groups * 4 + 255) & ~size_t{255};
    b->bytes = t_bytes + s_bytes + r_bytes + 256;
    NTT_CUDA_TRY(cudaMalloc(&b->block, b->bytes), "batch descriptors");
    char* base = (char*)b->block;
    b->args.tiles = (const BatchTile*)base;
    b->args.slots = (const uint32_t*)(base + t_bytes);
    b->args.rounds = (const uint32_t*)(base + t_bytes + s_bytes);
    b->args.counter = (uint32_t*)(base + t_bytes + s_bytes + r_bytes);
    b->args.groups = (uint32_t)groups;
    if (!b->tiles.empty()) {
        NTT_CUDA_TRY(cudaMemcpy(base, b->tiles.data(), b->tiles.size() * sizeof(BatchTile),
                                cudaMemcpyHostToDevice), "batch upload");
        NTT_CUDA_TRY(cudaMemcpy((void*)b->args.slots, b->slots.data(), b->slots.size() * 4,
                                cudaMemcpyHostToDevice), "batch upload");
        NTT_CUDA_TRY(cudaMemcpy((void*)b->args.rounds, b->rounds.data(), groups * 4,
                                cudaMemcpyHostToDevice), "batch upload");
    }
    b->variant = batch_variant(b->tiles.data(), b->tiles.size(), cl);
    const int resident = batch_resident_clusters(b->variant);
    if (resident <= 0) return fail(NTT_ERR_CUDA, "batch kernel: no resident clusters of %d CTAs", cl);
    int clusters = std::min<int>(resident, (int)groups);
    if (opt.max_clusters > 0) clusters = std::min(clusters, opt.max_clusters);
    b->clusters = clusters;
    *out = guard.release();
    return NTT_OK;
}

static ntt_status_t batch_enqueue(ntt_batch_t* b, cudaStream_t s) {
    NTT_CUDA_TRY(cudaMemsetAsync(b->args.counter, 0, 4, s), "batch counter reset");
    return batch_launch(b->args, b->variant, b->clusters, s);
}

extern "C" {

ntt_status_t ntt_batch_create(const ntt_job_t* jobs, int count, const ntt_batch_options_t* opts,
                              ntt_batch_t** out) {
    return batch_build(jobs, count, opts, out);
}

ntt_status_t ntt_batch_run(ntt_batch_t* b, ntt_stream_t stream) {
    if (!b) return fail(NTT_ERR_INVALID_ARGUMENT, "NULL batch");
    if (b->args.groups == 0) return NTT_OK;
    int dev = 0;
    NTT_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev != b->device)
        return fail(NTT_ERR_INVALID_ARGUMENT, "batch belongs to device %d (current %d)", b->device, dev);
    cudaStream_t s = (cudaStream_t)stream;
    if (!b->use_graph) return batch_enqueue(b, s);
    if (!b->exec) {
        // captured on a private stream (the caller's may be the legacy
        // default stream, which cannot be captured), replayed on any stream
        if (!b->cap)
            NTT_CUDA_TRY(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking), "capture stream");
        NTT_CUDA_TRY(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "begin capture");
        ntt_status_t st = batch_enqueue(b, b->cap);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->cap, &g);
        if (st != NTT_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return cuda_fail(e, "end capture");
        e = cudaGraphInstantiate(&b->exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            b->exec = nullptr;
            return cuda_fail(e, "graph instantiate");
        }
    }
    NTT_CUDA_TRY(cudaGraphLaunch(b->exec, s), "graph launch");
    return NTT_OK;
}

ntt_status_t ntt_batch_get_info(const ntt_batch_t* b, ntt_batch_info_t* out) {
    if (!b || !out) return fail(NTT_ERR_INVALID_ARGUMENT, "NULL argument");
    std::memset(out, 0, sizeof *out);
    out->jobs = b->jobs;
    out->tiles = (int)b->tiles.size();
    out->groups = (int)b->rounds.size();
    out->cluster_ctas = b->cl;
    out->clusters = b->clusters;
    out->multiply = b->mul ? 1 : 0;
    out->smem_bytes = batch_kernel_smem(b->mul);
    out->device_bytes = b->bytes;
    return NTT_OK;
}

ntt_status_t ntt_batch_destroy(ntt_batch_t* b) {
    if (!b) return NTT_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != b->device) cudaSetDevice(b->device);
    cudaDeviceSynchronize();  // launches of this batch may still be queued on any stream
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->cap) cudaStreamDestroy(b->cap);
    if (b->block) cudaFree(b->block);
    if (cur != b->device) cudaSetDevice(cur);
    delete b;
    return NTT_OK;
}

ntt_status_t ntt_batch_submit(const ntt_job_t* jobs, int count, ntt_stream_t stream) {
    ntt_batch_options_t o{0, 0, 0};
    ntt_batch_t* b = nullptr;
    if (ntt_status_t st = batch_build(jobs, count, &o, &b)) return st;
    ntt_status_t st = ntt_batch_run(b, stream);
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    ntt_batch_destroy(b);
    if (st != NTT_OK) return st;
    if (e != cudaSuccess) return cuda_fail(e, "batch submit");
    return NTT_OK;
}

size_t ntt_tables_device_bytes(void) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    return tables_device_bytes(dev);
}

void ntt_tables_trim(void) { tables_trim(); }

ntt_status_t ntt_tables_preload(int logN, const ModulusConfig* moduli, int count) {
    if (count < 1 || !moduli) return fail(NTT_ERR_INVALID_ARGUMENT, "need at least one modulus");
    if (logN < NTT_BATCH_MIN_LOGN || logN > NTT_BATCH_MAX_LOGN)
        return fail(NTT_ERR_UNSUPPORTED, "logN %d outside [%d, %d]", logN, NTT_BATCH_MIN_LOGN,
                    NTT_BATCH_MAX_LOGN);
    std::vector<TableRef> refs;
    return acquire_tables(logN, moduli, count, refs);
}

}  // extern "C"
