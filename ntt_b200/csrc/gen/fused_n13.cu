// Instantiations of the fused kernel for logN = 13 (see configs.h).
#include "fused_entry.h"

namespace nttb {
extern const FusedConfig kFusedN13[] = {NTTB_CFG_N13(NTTB_ENTRY)};
extern const int kFusedN13Count = sizeof(kFusedN13) / sizeof(kFusedN13[0]);
}  // namespace nttb
