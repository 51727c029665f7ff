// Instantiations of the persistent batch kernel: cluster of 8 CTAs,
// multiply tiles included, both range disciplines.
#include "../batch_kernel.cuh"

namespace nttb {
extern const void* const kBatchKernel_c8m[2] = {(const void*)&batch_kernel<8, true, Lazy4>,
                                               (const void*)&batch_kernel<8, true, Lazy2>};
}  // namespace nttb
