// Instantiations of the fused kernel for logN = 16 with several polynomials
// per job (see configs.h).
#include "fused_entry.h"

namespace nttb {
extern const FusedConfig kFusedN16M[] = {NTTB_CFG_N16M(NTTB_ENTRY)};
extern const int kFusedN16MCount = sizeof(kFusedN16M) / sizeof(kFusedN16M[0]);
}  // namespace nttb
