// Emulator instantiations of configuration list N10 (configs.h).
#include "emu_core.h"

namespace emu {
extern const Entry kEmuN10[] = {NTTB_CFG_N10(EMU_ENTRY)};
extern const int kEmuN10Count = sizeof(kEmuN10) / sizeof(kEmuN10[0]);
}  // namespace emu
