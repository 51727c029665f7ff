// Host-side pieces of the batch runtime shared with the serving loop.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <memory>
#include <vector>

#include "../../include/ntt_b200.h"
#include "arith.cuh"
#include "batch_geo.h"

namespace nttb {

// One device allocation of twiddle tables (several moduli of one logN).
struct TableSlab {
    int device = 0;
    void* block = nullptr;
    size_t bytes = 0;
    ~TableSlab();
};

// The resident tables of one (logN, modulus).
struct TableRef {
    std::shared_ptr<TableSlab> slab;
    const TwPair* fwd = nullptr;
    const TwPair* inv = nullptr;
    uint32_t q = 0;
    uint32_t nqinv = 0;  // -q^{-1} mod 2^32
};

// Tables of `count` moduli for logN on the current device, generating the
// missing ones (validated as plan creation does).
ntt_status_t acquire_tables(int logN, const ModulusConfig* mods, int count,
                            std::vector<TableRef>& out);
size_t tables_device_bytes(int device);
// Registry lookup only (never generates or allocates): false when the
// tables of (logN, m) are not resident on `device`.
bool find_resident_table(int device, int logN, ModulusConfig m, const TwPair** fwd,
                         const TwPair** inv, uint32_t* nqinv);
void tables_trim();

// Which instantiation of the batch kernel a launch needs.
struct BatchVariant {
    int cluster_ctas;  // 8 or 16 (16 when a tile has logN 17)
    bool mul;          // multiply tiles present
    bool lazy2;        // a modulus >= 2^30: [0, 2q) range discipline for every tile
};
BatchVariant batch_variant(const BatchTile* tiles, size_t n, int cluster_ctas);
const void* batch_kernel_fn(const BatchVariant& v);
uint32_t batch_kernel_smem(bool mul);
int batch_resident_clusters(const BatchVariant& v);
// One persistent launch (the counter must be zero, e.g. a memset ahead of it).
ntt_status_t batch_launch(const BatchArgs& a, const BatchVariant& v, int clusters, cudaStream_t s);
// Groups of cluster_ctas slots for the tiles (see batch.cu).
void pack_tiles(const std::vector<BatchTile>& tiles, int cluster_ctas,
                std::vector<uint32_t>& slots, std::vector<uint32_t>& rounds);

}  // namespace nttb
