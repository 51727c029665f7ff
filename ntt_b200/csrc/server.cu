// Serving loop: continuous batching of transform / multiply requests over
// the persistent batch kernel (include/ntt_b200_serve.h).
//
// Threads: the caller's (submit / poll / wait / put), one scheduler that
// admits queued requests into rounds, and one completion thread per stream
// slot.  A round = the H2D copies of its requests, one persistent batch
// launch, the D2H copies and an event, all on the slot's stream; up to
// `streams` rounds are in flight, so a round's copies overlap the others'
// transforms.  Device memory comes from one arena reserved at creation
// (first-fit with coalescing); a request is admitted, in FIFO order, once
// its polynomials fit.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/ntt_b200_serve.h"
#include "batch_rt.h"
#include "runtime.h"

using namespace nttb;
using Clock = std::chrono::steady_clock;

namespace {

constexpr size_t kAlign = 256;
constexpr size_t kNone = ~size_t{0};

// First-fit allocator over [0, size) with coalescing frees.
struct Arena {
    std::map<size_t, size_t> free_;  // offset -> length
    size_t used = 0, peak = 0;
    void init(size_t size) { free_[0] = size; }
    size_t alloc(size_t bytes) {
        bytes = (bytes + kAlign - 1) & ~(kAlign - 1);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            const size_t off = it->first, len = it->second;
            free_.erase(it);
            if (len > bytes) free_[off + bytes] = len - bytes;
            used += bytes;
            peak = std::max(peak, used);
            return off;
        }
        return kNone;
    }
    void release(size_t off, size_t bytes) {
        bytes = (bytes + kAlign - 1) & ~(kAlign - 1);
        used -= bytes;
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + bytes == next->first) {
            bytes += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += bytes;
                return;
            }
        }
        free_[off] = bytes;
    }
};

struct Req {
    uint64_t id = 0;
    int op = 0, logN = 0, limbs = 0;
    const uint32_t* input = nullptr;
    const uint32_t* operand = nullptr;
    uint64_t operand_handle = 0;
    uint32_t* output = nullptr;
    bool dev = false;                       // device-resident buffers (no arena, no PCIe)
    size_t bytes = 0;                       // one polynomial
    size_t off_data = kNone, off_op = kNone;  // arena slots owned by the request
    size_t res_off = kNone;                     // resident operand (owned by its handle)
    std::vector<TableRef> tables;
    Clock::time_point t_submit, t_done;
    ntt_status_t status = NTT_ERR_NOT_READY;
    size_t arena_need() const {
        if (dev) return 0;
        return bytes + (batch_op_is_multiply((uint32_t)op) && !operand_handle ? bytes : 0);
    }
};
using ReqP = std::shared_ptr<Req>;

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    void* dev_desc = nullptr;   // tiles | slots | rounds | counter
    void* host_desc = nullptr;  // pinned staging of the same
    size_t desc_bytes = 0;
    std::vector<ReqP> reqs;     // the round in flight
    bool busy = false;
    bool launched = false;      // the completion thread has work
    std::thread waiter;
};

}  // namespace

struct ntt_server {
    ntt_server_options_t opt{};
    int device = 0;
    char* arena_base = nullptr;
    size_t arena_size = 0;
    Arena arena;
    std::mutex mu;
    std::condition_variable cv_sched, cv_done, cv_slot;
    std::deque<ReqP> pending;
    std::unordered_map<uint64_t, ReqP> reqs;
    std::unordered_map<uint64_t, std::pair<size_t, size_t>> resident;  // handle -> (off, bytes)
    size_t resident_bytes = 0;
    std::vector<std::unique_ptr<Slot>> slots;
    std::thread sched;
    bool stop = false;
    uint64_t next_id = 1, next_handle = 1;
    // statistics
    uint64_t submitted = 0, completed = 0, failed = 0, rounds = 0, round_reqs = 0;
    double limb_ntts = 0;
    std::vector<double> lat_ms;
    bool have_first = false;
    Clock::time_point first_submit, last_done;
};

namespace {

size_t desc_capacity(int max_tiles) {
    const size_t t = ((size_t)max_tiles * sizeof(BatchTile) + 255) & ~size_t{255};
    const size_t s = ((size_t)max_tiles * 16 * 4 + 255) & ~size_t{255};
    const size_t r = ((size_t)max_tiles * 4 + 255) & ~size_t{255};
    return t + s + r + 256;
}

void finish_round(ntt_server* S, Slot& sl, ntt_status_t st) {
    const Clock::time_point now = Clock::now();
    std::lock_guard<std::mutex> lk(S->mu);
    for (auto& r : sl.reqs) {
        if (r->off_data != kNone) S->arena.release(r->off_data, r->bytes);
        if (r->off_op != kNone) S->arena.release(r->off_op, r->bytes);
        r->off_data = r->off_op = kNone;
        r->tables.clear();
        r->t_done = now;
        r->status = st;
        if (st == NTT_OK) {
            ++S->completed;
            S->lat_ms.push_back(std::chrono::duration<double, std::milli>(now - r->t_submit).count());
            S->limb_ntts += (double)r->limbs * batch_op_rounds((uint32_t)r->op);
        } else {
            ++S->failed;
        }
    }
    S->last_done = now;
    sl.reqs.clear();
    sl.busy = false;
    sl.launched = false;
    S->cv_sched.notify_all();
    S->cv_done.notify_all();
}

// Issues one round on a slot (called without the lock; the requests are
// owned by the slot).  Returns the first error.
ntt_status_t issue_round(ntt_server* S, Slot& sl) {
    cudaStream_t s = sl.stream;
    std::vector<BatchTile> tiles;
    int max_logn = 0;
    for (auto& r : sl.reqs) {
        char* data = r->dev ? (char*)r->output : S->arena_base + r->off_data;
        if (r->dev) {
            if (r->input != r->output &&
                cudaMemcpyAsync(data, r->input, r->bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
                return cuda_fail(cudaGetLastError(), "round input copy (device)");
        } else if (cudaMemcpyAsync(data, r->input, r->bytes, cudaMemcpyHostToDevice, s) !=
                   cudaSuccess) {
            return cuda_fail(cudaGetLastError(), "round input copy");
        }
        const uint32_t* opnd = nullptr;
        if (batch_op_is_multiply((uint32_t)r->op)) {
            if (r->dev && !r->operand_handle) {
                opnd = r->operand;
            } else if (r->operand_handle) {
                opnd = (const uint32_t*)(S->arena_base + r->res_off);
            } else {
                if (cudaMemcpyAsync(S->arena_base + r->off_op, r->operand, r->bytes,
                                    cudaMemcpyHostToDevice, s) != cudaSuccess)
                    return cuda_fail(cudaGetLastError(), "round operand copy");
                opnd = (const uint32_t*)(S->arena_base + r->off_op);
            }
        }
        const size_t N = size_t{1} << r->logN;
        max_logn = std::max(max_logn, r->logN);
        for (int l = 0; l < r->limbs; ++l) {
            BatchTile t;
            t.data = (uint32_t*)data + (size_t)l * N;
            t.operand = opnd ? opnd + (size_t)l * N : nullptr;
            t.tw_fwd = r->tables[l].fwd;
            t.tw_inv = r->tables[l].inv;
            t.q = r->tables[l].q;
            t.qinv = r->tables[l].nqinv;
            t.logn = (uint32_t)r->logN;
            t.op = (uint32_t)r->op;
            tiles.push_back(t);
        }
    }
    const int cl = S->opt.cluster_ctas ? S->opt.cluster_ctas : (max_logn >= 17 ? 16 : 8);
    std::vector<uint32_t> slots, rounds;
    pack_tiles(tiles, cl, slots, rounds);
    const size_t t_bytes = (tiles.size() * sizeof(BatchTile) + 255) & ~size_t{255};
    const size_t s_bytes = (slots.size() * 4 + 255) & ~size_t{255};
    const size_t r_bytes = (rounds.size() * 4 + 255) & ~size_t{255};
    const size_t need = t_bytes + s_bytes + r_bytes + 256;
    if (need > sl.desc_bytes) return fail(NTT_ERR_INVALID_ARGUMENT, "round descriptors overflow");
    char* h = (char*)sl.host_desc;
    std::memcpy(h, tiles.data(), tiles.size() * sizeof(BatchTile));
    std::memcpy(h + t_bytes, slots.data(), slots.size() * 4);
    std::memcpy(h + t_bytes + s_bytes, rounds.data(), rounds.size() * 4);
    std::memset(h + t_bytes + s_bytes + r_bytes, 0, 4);  // the group counter starts at zero
    if (cudaMemcpyAsync(sl.dev_desc, h, need, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "round descriptor copy");
    char* d = (char*)sl.dev_desc;
    BatchArgs a;
    a.tiles = (const BatchTile*)d;
    a.slots = (const uint32_t*)(d + t_bytes);
    a.rounds = (const uint32_t*)(d + t_bytes + s_bytes);
    a.counter = (uint32_t*)(d + t_bytes + s_bytes + r_bytes);
    a.groups = (uint32_t)rounds.size();
    const BatchVariant v = batch_variant(tiles.data(), tiles.size(), cl);
    const int resident = batch_resident_clusters(v);
    if (resident <= 0) return fail(NTT_ERR_CUDA, "batch kernel: no resident clusters");
    if (ntt_status_t st = batch_launch(a, v, std::min<int>(resident, (int)rounds.size()), s))
        return st;
    for (auto& r : sl.reqs)
        if (!r->dev && cudaMemcpyAsync(r->output, S->arena_base + r->off_data, r->bytes,
                                       cudaMemcpyDeviceToHost, s) != cudaSuccess)
            return cuda_fail(cudaGetLastError(), "round output copy");
    if (cudaEventRecord(sl.done, s) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "round event");
    return NTT_OK;
}

void waiter_main(ntt_server* S, Slot* sl) {
    cudaSetDevice(S->device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_slot.wait(lk, [&] { return sl->launched || (S->stop && !sl->busy); });
            if (!sl->launched) return;
        }
        const cudaError_t e = cudaEventSynchronize(sl->done);
        finish_round(S, *sl, e == cudaSuccess ? NTT_OK : cuda_fail(e, "round"));
    }
}

void scheduler_main(ntt_server* S) {
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        Slot* free_slot = nullptr;
        S->cv_sched.wait(lk, [&] {
            free_slot = nullptr;
            for (auto& s : S->slots)
                if (!s->busy) {
                    free_slot = s.get();
                    break;
                }
            return (S->stop && S->pending.empty()) || (!S->pending.empty() && free_slot);
        });
        if (S->pending.empty()) return;  // stop requested and drained
        // admit in FIFO order while the polynomials fit
        std::vector<ReqP> take;
        size_t tiles = 0;
        while (!S->pending.empty()) {
            ReqP r = S->pending.front();
            if (!take.empty() && tiles + (size_t)r->limbs > (size_t)S->opt.max_round_tiles) break;
            if (S->opt.max_round_requests && take.size() >= (size_t)S->opt.max_round_requests)
                break;
            if (r->dev) {  // runs where it lies: no arena space
                if (r->operand_handle) {
                    auto it = S->resident.find(r->operand_handle);
                    if (it == S->resident.end() || it->second.second < r->bytes) {
                        S->pending.pop_front();
                        r->status = fail(NTT_ERR_INVALID_ARGUMENT, "unknown or short operand handle");
                        ++S->failed;
                        S->cv_done.notify_all();
                        continue;
                    }
                    r->res_off = it->second.first;
                }
                take.push_back(r);
                tiles += (size_t)r->limbs;
                S->pending.pop_front();
                continue;
            }
            const size_t od = S->arena.alloc(r->bytes);
            if (od == kNone) break;
            size_t oo = kNone;
            if (batch_op_is_multiply((uint32_t)r->op)) {
                if (r->operand_handle) {
                    auto it = S->resident.find(r->operand_handle);
                    if (it == S->resident.end() || it->second.second < r->bytes) {
                        S->arena.release(od, r->bytes);
                        S->pending.pop_front();
                        r->status = fail(NTT_ERR_INVALID_ARGUMENT, "unknown or short operand handle");
                        ++S->failed;
                        S->cv_done.notify_all();
                        continue;
                    }
                    r->res_off = it->second.first;
                } else {
                    oo = S->arena.alloc(r->bytes);
                    if (oo == kNone) {
                        S->arena.release(od, r->bytes);
                        break;
                    }
                    r->off_op = oo;
                }
            }
            r->off_data = od;
            take.push_back(r);
            tiles += (size_t)r->limbs;
            S->pending.pop_front();
        }
        if (take.empty()) {
            bool any_busy = false;
            for (auto& s : S->slots) any_busy |= s->busy;
            if (!any_busy) {
                // nothing in flight will free memory: the head cannot fit
                ReqP r = S->pending.front();
                S->pending.pop_front();
                r->status = fail(NTT_ERR_BUDGET, "request does not fit the arena next to the "
                                 "resident operands");
                ++S->failed;
                S->cv_done.notify_all();
            } else {
                S->cv_sched.wait(lk);  // until a round completes
            }
            continue;
        }
        Slot& sl = *free_slot;
        sl.busy = true;
        sl.reqs = take;
        ++S->rounds;
        S->round_reqs += take.size();
        lk.unlock();
        ntt_status_t st = issue_round(S, sl);
        if (st != NTT_OK) {
            cudaStreamSynchronize(sl.stream);
            finish_round(S, sl, st);
            lk.lock();
            continue;
        }
        lk.lock();
        sl.launched = true;
        S->cv_slot.notify_all();
    }
}

}  // namespace

extern "C" {

ntt_status_t ntt_server_create(const ntt_server_options_t* opts, ntt_server_t** out) {
    if (!out) return fail(NTT_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    ntt_server_options_t o{};
    if (opts) o = *opts;
    if (o.streams < 0 || o.max_round_tiles < 0 || o.max_round_requests < 0 ||
        (o.cluster_ctas != 0 && o.cluster_ctas != 8 && o.cluster_ctas != 16))
        return fail(NTT_ERR_INVALID_ARGUMENT, "bad server options");
    if (!o.hbm_budget_bytes) o.hbm_budget_bytes = size_t{80} << 30;
    // defaults from a sweep on B200 at saturating load: the PCIe copies
    // pipeline once rounds hold ~1k tiles and 3-4 rounds are in flight
    if (!o.streams) o.streams = 4;
    if (!o.max_round_tiles) o.max_round_tiles = 1024;
    auto S = std::make_unique<ntt_server>();
    if (cudaGetDevice(&S->device) != cudaSuccess) return cuda_fail(cudaGetLastError(), "cudaGetDevice");
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "cudaMemGetInfo");
    const size_t margin = size_t{4} << 30;
    size_t size = (o.hbm_budget_bytes + kAlign - 1) & ~(kAlign - 1);
    if (size + margin > free_b) size = free_b > margin ? ((free_b - margin) & ~(kAlign - 1)) : 0;
    if (size == 0) return fail(NTT_ERR_OUT_OF_MEMORY, "no device memory for the server arena");
    o.hbm_budget_bytes = size;
    S->opt = o;
    if (cudaMalloc((void**)&S->arena_base, size) != cudaSuccess) {
        cudaGetLastError();
        return fail(NTT_ERR_OUT_OF_MEMORY, "server arena of %zu bytes", size);
    }
    S->arena_size = size;
    S->arena.init(size);
    const size_t desc = desc_capacity(o.max_round_tiles);
    for (int i = 0; i < o.streams; ++i) {
        auto sl = std::make_unique<Slot>();
        sl->desc_bytes = desc;
        cudaError_t e = cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking);
        // completion threads sleep in cudaEventSynchronize instead of
        // spinning: on a shared host, four spinning threads next to the
        // caller's submit loop showed up as multi-millisecond latency tails
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming | cudaEventBlockingSync);
        if (e == cudaSuccess) e = cudaMalloc(&sl->dev_desc, desc);
        if (e == cudaSuccess) e = cudaHostAlloc(&sl->host_desc, desc, cudaHostAllocDefault);
        S->slots.push_back(std::move(sl));
        if (e != cudaSuccess) {
            ntt_server_t* tmp = S.release();
            ntt_server_destroy(tmp);
            return cuda_fail(e, "server stream slot");
        }
    }
    ntt_server* raw = S.get();
    for (auto& sl : S->slots) sl->waiter = std::thread(waiter_main, raw, sl.get());
    S->sched = std::thread(scheduler_main, raw);
    *out = S.release();
    return NTT_OK;
}

ntt_status_t ntt_server_submit(ntt_server_t* S, const ntt_request_t* q, uint64_t* ticket) {
    if (!S || !q || !ticket) return fail(NTT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (q->op != NTT_OP_FORWARD && q->op != NTT_OP_INVERSE && q->op != NTT_OP_MULTIPLY &&
        q->op != NTT_OP_MULTIPLY_SPECTRUM)
        return fail(NTT_ERR_INVALID_ARGUMENT, "unknown op %d", q->op);
    if (q->logN < NTT_BATCH_MIN_LOGN || q->logN > NTT_BATCH_MAX_LOGN)
        return fail(NTT_ERR_UNSUPPORTED, "logN %d outside [%d, %d]", q->logN, NTT_BATCH_MIN_LOGN,
                    NTT_BATCH_MAX_LOGN);
    if (q->logN > 16 && S->opt.cluster_ctas == 8)
        return fail(NTT_ERR_UNSUPPORTED, "logN 17 needs 16-CTA clusters");
    if (q->limbs < 1 || !q->moduli || !q->input || !q->output)
        return fail(NTT_ERR_INVALID_ARGUMENT, "request needs limbs, moduli, input and output");
    if (q->limbs > S->opt.max_round_tiles)
        return fail(NTT_ERR_UNSUPPORTED, "more limbs than a round holds (%d)", S->opt.max_round_tiles);
    if (batch_op_is_multiply((uint32_t)q->op) && !q->operand && !q->operand_handle)
        return fail(NTT_ERR_INVALID_ARGUMENT, "multiply needs an operand");
    if (q->device_buffers &&
        (((uintptr_t)q->input | (uintptr_t)q->output | (uintptr_t)q->operand) & 15u) != 0)
        return fail(NTT_ERR_MISALIGNED, "device buffers must be 16-byte aligned");
    auto r = std::make_shared<Req>();
    r->op = q->op;
    r->logN = q->logN;
    r->limbs = q->limbs;
    r->input = q->input;
    r->operand = q->operand;
    r->operand_handle = batch_op_is_multiply((uint32_t)q->op) ? q->operand_handle : 0;
    r->output = q->output;
    r->dev = q->device_buffers != 0;
    r->bytes = ((size_t)q->limbs << q->logN) * 4;
    if (r->arena_need() > S->arena_size)
        return fail(NTT_ERR_BUDGET, "request needs %zu bytes, arena holds %zu", r->arena_need(),
                    S->arena_size);
    {
        int cur = 0;
        cudaGetDevice(&cur);
        if (cur != S->device) cudaSetDevice(S->device);
        ntt_status_t st = acquire_tables(q->logN, q->moduli, q->limbs, r->tables);
        if (cur != S->device) cudaSetDevice(cur);
        if (st != NTT_OK) return st;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return fail(NTT_ERR_SHUTDOWN, "server is shutting down");
    r->id = S->next_id++;
    r->t_submit = Clock::now();
    if (!S->have_first) {
        S->have_first = true;
        S->first_submit = r->t_submit;
    }
    ++S->submitted;
    S->reqs[r->id] = r;
    S->pending.push_back(r);
    *ticket = r->id;
    S->cv_sched.notify_all();
    return NTT_OK;
}

ntt_status_t ntt_server_poll(ntt_server_t* S, uint64_t ticket) {
    if (!S) return fail(NTT_ERR_INVALID_ARGUMENT, "NULL server");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return fail(NTT_ERR_INVALID_ARGUMENT, "unknown ticket");
    return it->second->status;
}

ntt_status_t ntt_server_wait(ntt_server_t* S, uint64_t ticket, double timeout_s) {
    if (!S) return fail(NTT_ERR_INVALID_ARGUMENT, "NULL server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return fail(NTT_ERR_INVALID_ARGUMENT, "unknown ticket");
    ReqP r = it->second;
    auto ready = [&] { return r->status != NTT_ERR_NOT_READY; };
    if (timeout_s < 0) {
        S->cv_done.wait(lk, ready);
    } else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
        return fail(NTT_ERR_TIMEOUT, "ticket %llu still pending", (unsigned long long)ticket);
    }
    return r->status;
}

double ntt_server_latency_ms(ntt_server_t* S, uint64_t ticket) {
    if (!S) return -1.0;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end() || it->second->status != NTT_OK) return -1.0;
    return std::chrono::duration<double, std::milli>(it->second->t_done - it->second->t_submit)
        .count();
}

ntt_status_t ntt_server_put(ntt_server_t* S, const uint32_t* host, size_t words, uint64_t* handle) {
    if (!S || !host || !handle || words == 0) return fail(NTT_ERR_INVALID_ARGUMENT, "bad arguments");
    size_t off;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        off = S->arena.alloc(words * 4);
        if (off == kNone) return fail(NTT_ERR_BUDGET, "no arena space for %zu words", words);
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != S->device) cudaSetDevice(S->device);
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(S->arena_base + off, host, words * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (s) cudaStreamDestroy(s);
    if (cur != S->device) cudaSetDevice(cur);
    std::lock_guard<std::mutex> lk(S->mu);
    if (e != cudaSuccess) {
        S->arena.release(off, words * 4);
        return cuda_fail(e, "resident operand copy");
    }
    *handle = S->next_handle++;
    S->resident[*handle] = {off, words * 4};
    S->resident_bytes += (words * 4 + kAlign - 1) & ~(kAlign - 1);
    return NTT_OK;
}

ntt_status_t ntt_server_put_spectrum(ntt_server_t* S, int logN, const ModulusConfig* moduli,
                                     int limbs, const uint32_t* host, uint64_t* handle) {
    if (!S || !moduli || !host || !handle || limbs < 1)
        return fail(NTT_ERR_INVALID_ARGUMENT, "bad arguments");
    if (logN < NTT_BATCH_MIN_LOGN || logN > NTT_BATCH_MAX_LOGN)
        return fail(NTT_ERR_UNSUPPORTED, "logN %d outside [%d, %d]", logN, NTT_BATCH_MIN_LOGN,
                    NTT_BATCH_MAX_LOGN);
    uint64_t h = 0;
    if (ntt_status_t st = ntt_server_put(S, host, (size_t)limbs << logN, &h)) return st;
    size_t off;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        off = S->resident[h].first;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != S->device) cudaSetDevice(S->device);
    ntt_job_t job{NTT_OP_FORWARD, logN, limbs, moduli, (uint32_t*)(S->arena_base + off), nullptr};
    ntt_batch_options_t o{0, 0, 0};
    ntt_batch_t* b = nullptr;
    ntt_status_t st = ntt_batch_create(&job, 1, &o, &b);
    cudaStream_t s = nullptr;
    if (st == NTT_OK && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
        st = cuda_fail(cudaGetLastError(), "spectrum stream");
    if (st == NTT_OK) st = ntt_batch_run(b, s);
    if (st == NTT_OK && cudaStreamSynchronize(s) != cudaSuccess)
        st = cuda_fail(cudaGetLastError(), "spectrum transform");
    if (s) cudaStreamDestroy(s);
    if (b) ntt_batch_destroy(b);
    if (cur != S->device) cudaSetDevice(cur);
    if (st != NTT_OK) {
        ntt_server_drop(S, h);
        return st;
    }
    *handle = h;
    return NTT_OK;
}

ntt_status_t ntt_server_drop(ntt_server_t* S, uint64_t handle) {
    if (!S) return fail(NTT_ERR_INVALID_ARGUMENT, "NULL server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->resident.find(handle);
    if (it == S->resident.end()) return fail(NTT_ERR_INVALID_ARGUMENT, "unknown handle");
    // wait until no queued or running request names the handle
    auto in_use = [&] {
        for (auto& r : S->pending)
            if (r->operand_handle == handle) return true;
        for (auto& s : S->slots)
            for (auto& r : s->reqs)
                if (r->operand_handle == handle) return true;
        return false;
    };
    S->cv_done.wait(lk, [&] { return !in_use(); });
    S->arena.release(it->second.first, it->second.second);
    S->resident_bytes -= (it->second.second + kAlign - 1) & ~(kAlign - 1);
    S->resident.erase(it);
    S->cv_sched.notify_all();
    return NTT_OK;
}

ntt_status_t ntt_server_stats(ntt_server_t* S, int reset, ntt_server_stats_t* out) {
    if (!S || !out) return fail(NTT_ERR_INVALID_ARGUMENT, "NULL argument");
    std::lock_guard<std::mutex> lk(S->mu);
    std::memset(out, 0, sizeof *out);
    out->submitted = S->submitted;
    out->completed = S->completed;
    out->failed = S->failed;
    out->rounds = S->rounds;
    out->mean_round_requests = S->rounds ? (double)S->round_reqs / S->rounds : 0.0;
    if (!S->lat_ms.empty()) {
        std::vector<double> v = S->lat_ms;
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) {
            const size_t i = (size_t)std::min<double>(v.size() - 1, std::ceil(p * v.size()) - 1);
            return v[i];
        };
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        out->max_ms = v.back();
        double sum = 0;
        for (double x : v) sum += x;
        out->mean_ms = sum / v.size();
    }
    if (S->have_first && S->completed)
        out->elapsed_s = std::chrono::duration<double>(S->last_done - S->first_submit).count();
    out->limb_ntt_per_s = out->elapsed_s > 0 ? S->limb_ntts / out->elapsed_s : 0.0;
    out->budget_bytes = S->arena_size;
    out->arena_peak_bytes = S->arena.peak;
    out->resident_bytes = S->resident_bytes;
    out->table_bytes = tables_device_bytes(S->device);
    if (reset) {
        S->submitted = S->completed = S->failed = S->rounds = S->round_reqs = 0;
        S->limb_ntts = 0;
        S->lat_ms.clear();
        S->have_first = false;
        S->arena.peak = S->arena.used;
        // completed tickets are forgotten; pending ones stay
        for (auto it = S->reqs.begin(); it != S->reqs.end();)
            it = it->second->status != NTT_ERR_NOT_READY ? S->reqs.erase(it) : std::next(it);
    }
    return NTT_OK;
}

ntt_status_t ntt_server_destroy(ntt_server_t* S) {
    if (!S) return NTT_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv_sched.notify_all();
    }
    if (S->sched.joinable()) S->sched.join();
    {
        // every round issued by the scheduler is now owned by a waiter
        std::unique_lock<std::mutex> lk(S->mu);
        S->cv_done.wait(lk, [&] {
            for (auto& s : S->slots)
                if (s->busy) return false;
            return true;
        });
        S->cv_slot.notify_all();
    }
    for (auto& sl : S->slots)
        if (sl->waiter.joinable()) sl->waiter.join();
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != S->device) cudaSetDevice(S->device);
    for (auto& sl : S->slots) {
        if (sl->done) cudaEventDestroy(sl->done);
        if (sl->stream) cudaStreamDestroy(sl->stream);
        if (sl->dev_desc) cudaFree(sl->dev_desc);
        if (sl->host_desc) cudaFreeHost(sl->host_desc);
    }
    if (S->arena_base) cudaFree(S->arena_base);
    if (cur != S->device) cudaSetDevice(cur);
    delete S;
    return NTT_OK;
}

}  // extern "C"
