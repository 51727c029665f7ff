// Instantiations of the persistent batch kernel: cluster of 16 CTAs,
// multiply tiles included, both range disciplines.
#include "../batch_kernel.cuh"

namespace nttb {
extern const void* const kBatchKernel_c16m[2] = {(const void*)&batch_kernel<16, true, Lazy4>,
                                               (const void*)&batch_kernel<16, true, Lazy2>};
}  // namespace nttb
