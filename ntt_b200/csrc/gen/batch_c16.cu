// Instantiation of the persistent batch kernel: cluster of 16 CTAs,
// multiply tiles excluded.
#include "../batch_kernel.cuh"

namespace nttb {
extern const void* const kBatchKernel_c16 = (const void*)&batch_kernel<16, false>;
}  // namespace nttb
