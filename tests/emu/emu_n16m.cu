// Emulator instantiations of configuration list N16M (configs.h).
#include "emu_core.h"

namespace emu {
extern const Entry kEmuN16M[] = {NTTB_CFG_N16M(EMU_ENTRY)};
extern const int kEmuN16MCount = sizeof(kEmuN16M) / sizeof(kEmuN16M[0]);
}  // namespace emu
