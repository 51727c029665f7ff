// Instantiations of the fused kernel for logN = 12 (see configs.h).
#include "fused_entry.h"

namespace nttb {
extern const FusedConfig kFusedN12[] = {NTTB_CFG_N12(NTTB_ENTRY)};
extern const int kFusedN12Count = sizeof(kFusedN12) / sizeof(kFusedN12[0]);
}  // namespace nttb
