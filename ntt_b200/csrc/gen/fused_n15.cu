// Instantiations of the fused kernel for logN = 15 (see configs.h).
#include "fused_entry.h"

namespace nttb {
extern const FusedConfig kFusedN15[] = {NTTB_CFG_N15(NTTB_ENTRY)};
extern const int kFusedN15Count = sizeof(kFusedN15) / sizeof(kFusedN15[0]);
}  // namespace nttb
