// Instantiations of the fused kernel for logN = 11 (see configs.h).
#include "fused_entry.h"

namespace nttb {
extern const FusedConfig kFusedN11[] = {NTTB_CFG_N11(NTTB_ENTRY)};
extern const int kFusedN11Count = sizeof(kFusedN11) / sizeof(kFusedN11[0]);
}  // namespace nttb
