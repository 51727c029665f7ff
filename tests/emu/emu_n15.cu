// Emulator instantiations of configuration list N15 (configs.h).
#include "emu_core.h"

namespace emu {
extern const Entry kEmuN15[] = {NTTB_CFG_N15(EMU_ENTRY)};
extern const int kEmuN15Count = sizeof(kEmuN15) / sizeof(kEmuN15[0]);
}  // namespace emu
