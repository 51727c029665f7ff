// Emulator instantiations of configuration list N12 (configs.h).
#include "emu_core.h"

namespace emu {
extern const Entry kEmuN12[] = {NTTB_CFG_N12(EMU_ENTRY)};
extern const int kEmuN12Count = sizeof(kEmuN12) / sizeof(kEmuN12[0]);
}  // namespace emu
