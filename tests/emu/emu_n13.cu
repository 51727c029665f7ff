// Emulator instantiations of configuration list N13 (configs.h).
#include "emu_core.h"

namespace emu {
extern const Entry kEmuN13[] = {NTTB_CFG_N13(EMU_ENTRY)};
extern const int kEmuN13Count = sizeof(kEmuN13) / sizeof(kEmuN13[0]);
}  // namespace emu
