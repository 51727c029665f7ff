// Emulator instantiations of configuration list N16 (configs.h).
#include "emu_core.h"

namespace emu {
extern const Entry kEmuN16[] = {NTTB_CFG_N16(EMU_ENTRY)};
extern const int kEmuN16Count = sizeof(kEmuN16) / sizeof(kEmuN16[0]);
}  // namespace emu
