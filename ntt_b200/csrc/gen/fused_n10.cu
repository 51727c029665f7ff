// Instantiations of the fused kernel for logN = 10 (see configs.h).
#include "fused_entry.h"

namespace nttb {
extern const FusedConfig kFusedN10[] = {NTTB_CFG_N10(NTTB_ENTRY)};
extern const int kFusedN10Count = sizeof(kFusedN10) / sizeof(kFusedN10[0]);
}  // namespace nttb
