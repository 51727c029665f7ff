// Instantiations of the persistent batch kernel: cluster of 8 CTAs,
// multiply tiles excluded, both range disciplines.
#include "../batch_kernel.cuh"

namespace nttb {
extern const void* const kBatchKernel_c8[2] = {(const void*)&batch_kernel<8, false, Lazy4>,
                                               (const void*)&batch_kernel<8, false, Lazy2>};
}  // namespace nttb
