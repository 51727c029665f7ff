// Instantiations of the fused kernel for logN = 17 (see configs.h).
#include "fused_entry.h"

namespace nttb {
extern const FusedConfig kFusedN17[] = {NTTB_CFG_N17(NTTB_ENTRY)};
extern const int kFusedN17Count = sizeof(kFusedN17) / sizeof(kFusedN17[0]);
}  // namespace nttb
