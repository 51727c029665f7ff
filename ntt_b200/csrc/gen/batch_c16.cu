// Instantiations of the persistent batch kernel: cluster of 16 CTAs,
// multiply tiles excluded, both range disciplines.
#include "../batch_kernel.cuh"

namespace nttb {
extern const void* const kBatchKernel_c16[2] = {(const void*)&batch_kernel<16, false, Lazy4>,
                                               (const void*)&batch_kernel<16, false, Lazy2>};
}  // namespace nttb
