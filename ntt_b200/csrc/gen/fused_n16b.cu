// Instantiations of the fused kernel for logN = 16, second list (see
// configs.h).
#include "fused_entry.h"

namespace nttb {
extern const FusedConfig kFusedN16B[] = {NTTB_CFG_N16B(NTTB_ENTRY)};
extern const int kFusedN16BCount = sizeof(kFusedN16B) / sizeof(kFusedN16B[0]);
}  // namespace nttb
