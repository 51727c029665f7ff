// Shapes of the persistent ragged-batch kernel, shared by host and device.
//
// Every CTA of the batch kernel has 256 threads and handles 8192 words of a
// limb (4096 for logN 12), so a limb of 2^logN words occupies 2^(logN-13)
// CTAs of a cluster (one CTA below logN 14).  A cluster of kBatchCluster
// CTAs takes one "group" of tiles at a time: tiles of different limbs (and
// of different polynomials, sizes, moduli and operations) sit side by side
// in aligned power-of-two CTA ranges of the cluster.
#pragma once
#include <cstdint>

namespace nttb {

constexpr int kBatchThreads = 256;
constexpr int kBatchMinLogN = 12;
constexpr int kBatchMaxLogN = 17;
// tile operations
constexpr uint32_t kOpForward = 0;   // forward NTT in place
constexpr uint32_t kOpInverse = 1;   // inverse NTT in place
constexpr uint32_t kOpMultiply = 2;  // data = INTT(NTT(operand) . NTT(data))
constexpr uint32_t kOpMultiplySpectrum = 3;  // data = INTT(operand . NTT(data)), operand a spectrum
constexpr bool batch_op_is_multiply(uint32_t op) {
    return op == kOpMultiply || op == kOpMultiplySpectrum;
}
// cluster barrier rounds a tile of each operation takes (one per transform)
constexpr uint32_t batch_op_rounds(uint32_t op) {
    return op == kOpMultiply ? 3u : op == kOpMultiplySpectrum ? 2u : 1u;
}
// log2 CTAs per limb tile
constexpr int batch_tile_clog(int logN) { return logN >= 14 ? logN - 13 : 0; }
// slot word of a group: tile index | sub-rank << 24, or idle
constexpr uint32_t kIdleSlot = 0xFFFFFFFFu;
constexpr uint32_t kSlotTileMask = 0x00FFFFFFu;
constexpr int kSlotSubShift = 24;

// One (polynomial, limb) tile.  48 bytes.
struct BatchTile {
    uint32_t* data;           // limb start: input, output in place
    const uint32_t* operand;  // multiplies: the other factor's limb (read only)
    const void* tw_fwd;       // [2^logN] forward Shoup twiddle pairs of this modulus
    const void* tw_inv;       // [2^logN] inverse pairs
    uint32_t q;               // modulus
    uint32_t qinv;            // -q^{-1} mod 2^32 (multiplies)
    uint32_t logn;
    uint32_t op;
};

struct BatchArgs {
    const BatchTile* tiles;
    const uint32_t* slots;   // [groups][cluster]
    const uint32_t* rounds;  // [groups]: max rounds of the group's tiles
    uint32_t groups;
    uint32_t* counter;       // next group to take; zero when the launch starts
};

}  // namespace nttb
