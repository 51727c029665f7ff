// Emulator instantiations of configuration list N11 (configs.h).
#include "emu_core.h"

namespace emu {
extern const Entry kEmuN11[] = {NTTB_CFG_N11(EMU_ENTRY)};
extern const int kEmuN11Count = sizeof(kEmuN11) / sizeof(kEmuN11[0]);
}  // namespace emu
