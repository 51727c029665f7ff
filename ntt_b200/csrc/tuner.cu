// Autotuner: sweep the compiled configurations for (logN, limbs), time the
// forward and the inverse launch of each on the device, keep the fastest per
// direction (in memory and in an on-disk cache).
//
// Replaces the reference's compile-time choice of phase triples
// (DefaultNTTLaunchConfig<LogN>, src/ntt_config.h:62-73): the triple is now
// picked per (logN, limb count, direction) at run time, "sweep, then cache".
// Cache file: $NTT_B200_TUNE_CACHE, else $HOME/.cache/ntt_b200/tune.txt;
// one line per entry:
//   "<device-name>|<sm-count> <logN> <limb-bucket> <fwd|inv> <config> <us>",
// <config> the configuration's parameters (config_signature), not its
// catalogue index, so that a cache written by another build of the library
// never selects a different kernel: entries whose configuration is not
// compiled here are ignored.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <sys/stat.h>
#include <tuple>
#include <vector>

#include "runtime.h"

using namespace nttb;

namespace {

std::mutex g_mu;
bool g_loaded = false;
// key: device id, logN, limb bucket, direction (1 = forward)
std::map<std::tuple<std::string, int, int, int>, std::pair<int, double>> g_table;

int limb_bucket(int limbs) {  // 1, 2-4, 5-16, 17-64, 65+
    if (limbs <= 1) return 0;
    if (limbs <= 4) return 1;
    if (limbs <= 16) return 2;
    if (limbs <= 64) return 3;
    return 4;
}

std::string device_key() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return "?";
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return "?";
    std::string n = p.name;
    for (auto& ch : n)
        if (ch == ' ' || ch == '|') ch = '_';
    return n + "|" + std::to_string(p.multiProcessorCount);
}

std::string cache_path() {
    if (const char* e = getenv("NTT_B200_TUNE_CACHE")) return e;
    const char* h = getenv("HOME");
    return std::string(h ? h : "/tmp") + "/.cache/ntt_b200/tune.txt";
}

// "logN,CTAs,r1,eb,k1a,k2a,polys-per-job,exchange,k2b" (ntt_kernel_config_t's fields).
std::string config_signature(const FusedConfig* c) {
    char b[96];
    snprintf(b, sizeof b, "%d,%d,%d,%d,%d,%d,%d,%d,%d", c->logN, 1 << c->clog, c->r1, c->eb, c->k1a,
             c->k2a, c->np, c->split, c->split ? c->k2b : 0);
    return b;
}

int config_by_signature(const std::string& sig) {
    for (int i = 0; i < fused_config_count(); ++i)
        if (config_signature(config_by_index(i)) == sig) return i;
    return -1;
}

void load_locked() {
    if (g_loaded) return;
    g_loaded = true;
    FILE* f = fopen(cache_path().c_str(), "r");
    if (!f) return;
    char dev[256], dir[8], sig[96];
    int logN, bucket;
    double us;
    while (fscanf(f, "%255s %d %d %7s %95s %lf", dev, &logN, &bucket, dir, sig, &us) == 6) {
        const int idx = config_by_signature(sig);
        if (idx >= 0 && config_by_index(idx)->logN == logN)
            g_table[{dev, logN, bucket, std::string(dir) == "fwd" ? 1 : 0}] = {idx, us};
    }
    fclose(f);
}

void save_locked() {
    std::string path = cache_path();
    std::string dir = path.substr(0, path.find_last_of('/'));
    for (size_t i = 1; i <= dir.size(); ++i)  // parent directories, best effort
        if (i == dir.size() || dir[i] == '/') mkdir(dir.substr(0, i).c_str(), 0755);
    FILE* f = fopen(path.c_str(), "w");
    if (!f) return;
    for (auto& kv : g_table)
        fprintf(f, "%s %d %d %s %s %.3f\n", std::get<0>(kv.first).c_str(), std::get<1>(kv.first),
                std::get<2>(kv.first), std::get<3>(kv.first) ? "fwd" : "inv",
                config_signature(config_by_index(kv.second.first)).c_str(), kv.second.second);
    fclose(f);
}

// Deterministic filler below every supported modulus (the timed transforms
// do not depend on the values).
__global__ void fill_kernel(uint32_t* a, size_t n, uint32_t seed) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) {
        uint32_t x = (uint32_t)i * 2654435761u ^ seed;
        x ^= x >> 13;
        x *= 0x5bd1e995u;
        a[i] = (x ^ (x >> 15)) & 0x1fffffffu;
    }
}

}  // namespace

namespace nttb {
const FusedConfig* tuned_config(int logN, int limbs, bool fwd) {
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    auto it = g_table.find({device_key(), logN, limb_bucket(limbs), fwd ? 1 : 0});
    if (it == g_table.end()) return nullptr;
    return config_by_index(it->second.first);
}
}  // namespace nttb

extern "C" {

int ntt_config_count(void) { return fused_config_count(); }

ntt_status_t ntt_config_get(int index, ntt_kernel_config_t* out) {
    const FusedConfig* c = config_by_index(index);
    if (!c || !out) return fail(NTT_ERR_INVALID_ARGUMENT, "bad config index %d", index);
    *out = ntt_kernel_config_t{c->logN, 1 << c->clog, c->r1,      c->eb,
                               c->k1a,  c->k2a,       c->threads, c->smem_bytes_direct,
                               c->np,   c->split,     c->split ? c->k2b : 0};
    return NTT_OK;
}

int ntt_config_resident_clusters(int index, int forward, int schedule) {
    const FusedConfig* c = config_by_index(index);
    if (!c) return -1;
    return config_resident_clusters(c, forward != 0, schedule);
}

ntt_status_t ntt_autotune(int logN, int limbs, int polys, int iters, ntt_tune_result_t* out) {
    if (limbs < 1 || polys < 1 || iters < 1)
        return fail(NTT_ERR_INVALID_ARGUMENT, "limbs, polys and iters must be positive");
    std::vector<int> cand;
    for (int i = 0; i < fused_config_count(); ++i)
        if (config_by_index(i)->logN == logN) cand.push_back(i);
    if (cand.empty()) return fail(NTT_ERR_UNSUPPORTED, "no fused configurations for logN %d", logN);
    std::vector<ModulusConfig> mods(limbs);
    if (ntt_status_t st = ntt_find_moduli(logN, limbs, 1u << 29, mods.data())) return st;
    ntt_plan_t* plan = nullptr;
    if (ntt_status_t st = ntt_plan_create(logN, mods.data(), limbs, nullptr, &plan)) return st;
    const uint32_t *tw_f = nullptr, *tw_i = nullptr, *qd = nullptr;
    ntt_plan_tables(plan, &tw_f, &tw_i, &qd);
    const size_t words = (size_t)polys * limbs << logN;
    uint32_t* data = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t s = nullptr;
    ntt_status_t st = NTT_OK;
    double best[2] = {1e30, 1e30};
    int best_idx[2] = {-1, -1};
    cudaError_t ce = cudaMalloc(&data, words * 4);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
    if (ce != cudaSuccess) st = cuda_fail(ce, "autotune setup");
    if (st == NTT_OK) {
        fill_kernel<<<(unsigned)((words + 255) / 256), 256, 0, s>>>(data, words, 1234u);
        for (int idx : cand) {
            const FusedConfig* c = config_by_index(idx);
            for (int dir = 1; dir >= 0 && st == NTT_OK; --dir) {  // 1 = forward
                float ms = 0;
                for (int rep = 0; rep < 2 && st == NTT_OK; ++rep) {  // rep 0 = warm-up
                    cudaEventRecord(e0, s);
                    for (int it = 0; it < iters && st == NTT_OK; ++it)
                        st = run_transform(logN, c, (const TwPair*)(dir ? tw_f : tw_i), qd, limbs,
                                           data, polys, (size_t)limbs << logN, dir == 1, s,
                                           nullptr, NTT_SCHEDULE_DIRECT, false);
                    cudaEventRecord(e1, s);
                    ce = cudaEventSynchronize(e1);
                    if (ce != cudaSuccess) st = cuda_fail(ce, "autotune timing");
                    cudaEventElapsedTime(&ms, e0, e1);
                }
                const double us = 1000.0 * ms / iters;
                if (st == NTT_OK && us < best[dir]) {
                    best[dir] = us;
                    best_idx[dir] = idx;
                }
            }
            if (st != NTT_OK) break;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    if (data) cudaFree(data);
    ntt_plan_destroy(plan);
    if (st != NTT_OK) return st;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        load_locked();
        g_table[{device_key(), logN, limb_bucket(limbs), 1}] = {best_idx[1], best[1]};
        g_table[{device_key(), logN, limb_bucket(limbs), 0}] = {best_idx[0], best[0]};
        save_locked();
    }
    if (out) {
        out->fwd_index = best_idx[1];
        out->inv_index = best_idx[0];
        out->fwd_us = best[1];
        out->inv_us = best[0];
        out->candidates = (int)cand.size();
    }
    return NTT_OK;
}

void ntt_autotune_forget(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_table.clear();
    g_loaded = true;  // do not reload the file until ntt_autotune_reload
}

void ntt_autotune_reload(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_table.clear();
    g_loaded = false;
}

}  // extern "C"
