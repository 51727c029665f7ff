// Instantiation of the persistent batch kernel: cluster of 8 CTAs,
// multiply tiles excluded.
#include "../batch_kernel.cuh"

namespace nttb {
extern const void* const kBatchKernel_c8 = (const void*)&batch_kernel<8, false>;
}  // namespace nttb
