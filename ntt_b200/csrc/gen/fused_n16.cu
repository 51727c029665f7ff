// Instantiations of the fused kernel for logN = 16 (see configs.h).
#include "fused_entry.h"

namespace nttb {
extern const FusedConfig kFusedN16[] = {NTTB_CFG_N16(NTTB_ENTRY)};
extern const int kFusedN16Count = sizeof(kFusedN16) / sizeof(kFusedN16[0]);
}  // namespace nttb
