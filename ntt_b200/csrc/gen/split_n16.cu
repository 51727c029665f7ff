// Instantiations of the split kernels for logN = 16 (configs.h).
#include "split_entry.h"

namespace nttb {
extern const FusedConfig kFusedNSplit16[] = {NTTB_SPLIT_N16(NTTB_SPLIT_ENTRY)};
extern const int kFusedNSplit16Count = sizeof(kFusedNSplit16) / sizeof(kFusedNSplit16[0]);
}  // namespace nttb
