// Instantiations of the fused kernel for logN = 14 (see configs.h).
#include "fused_entry.h"

namespace nttb {
extern const FusedConfig kFusedN14[] = {NTTB_CFG_N14(NTTB_ENTRY)};
extern const int kFusedN14Count = sizeof(kFusedN14) / sizeof(kFusedN14[0]);
}  // namespace nttb
