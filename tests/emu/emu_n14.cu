// Emulator instantiations of configuration list N14 (configs.h).
#include "emu_core.h"

namespace emu {
extern const Entry kEmuN14[] = {NTTB_CFG_N14(EMU_ENTRY)};
extern const int kEmuN14Count = sizeof(kEmuN14) / sizeof(kEmuN14[0]);
}  // namespace emu
