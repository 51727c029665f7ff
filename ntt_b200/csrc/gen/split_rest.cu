// Instantiations of the split kernels for the other sizes (configs.h).
#include "split_entry.h"

namespace nttb {
extern const FusedConfig kFusedNSplitRest[] = {NTTB_SPLIT_REST(NTTB_SPLIT_ENTRY)};
extern const int kFusedNSplitRestCount = sizeof(kFusedNSplitRest) / sizeof(kFusedNSplitRest[0]);
}  // namespace nttb
