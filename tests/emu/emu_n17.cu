// Emulator instantiations of configuration list N17 (configs.h).
#include "emu_core.h"

namespace emu {
extern const Entry kEmuN17[] = {NTTB_CFG_N17(EMU_ENTRY)};
extern const int kEmuN17Count = sizeof(kEmuN17) / sizeof(kEmuN17[0]);
}  // namespace emu
