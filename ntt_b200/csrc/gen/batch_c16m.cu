// Instantiation of the persistent batch kernel: cluster of 16 CTAs,
// multiply tiles included.
#include "../batch_kernel.cuh"

namespace nttb {
extern const void* const kBatchKernel_c16m = (const void*)&batch_kernel<16, true>;
}  // namespace nttb
