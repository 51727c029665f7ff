// Gathers the per-logN instantiation tables into one registry.
#include <vector>
#include "configs.h"

namespace nttb {
#define NTTB_DECL(n)                    \
    extern const FusedConfig kFusedN##n[]; \
    extern const int kFusedN##n##Count;
NTTB_DECL(10) NTTB_DECL(11) NTTB_DECL(12) NTTB_DECL(13)
NTTB_DECL(14) NTTB_DECL(15) NTTB_DECL(16) NTTB_DECL(16B) NTTB_DECL(16M) NTTB_DECL(17)
NTTB_DECL(Split16) NTTB_DECL(SplitRest)

static const std::vector<FusedConfig>& all() {
    static const std::vector<FusedConfig> v = [] {
        std::vector<FusedConfig> r;
#define NTTB_ADD(n) r.insert(r.end(), kFusedN##n, kFusedN##n + kFusedN##n##Count);
        NTTB_ADD(10) NTTB_ADD(11) NTTB_ADD(12) NTTB_ADD(13)
        NTTB_ADD(14) NTTB_ADD(15) NTTB_ADD(16) NTTB_ADD(16B) NTTB_ADD(16M) NTTB_ADD(17)
        NTTB_ADD(Split16) NTTB_ADD(SplitRest)
        return r;
    }();
    return v;
}
const FusedConfig* fused_configs() { return all().data(); }
int fused_config_count() { return (int)all().size(); }
}  // namespace nttb
