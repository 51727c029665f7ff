// Instantiation of the persistent batch kernel: cluster of 8 CTAs,
// multiply tiles included.
#include "../batch_kernel.cuh"

namespace nttb {
extern const void* const kBatchKernel_c8m = (const void*)&batch_kernel<8, true>;
}  // namespace nttb
