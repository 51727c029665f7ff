// Emulator instantiations of configuration list N16B (configs.h).
#include "emu_core.h"

namespace emu {
extern const Entry kEmuN16B[] = {NTTB_CFG_N16B(EMU_ENTRY)};
extern const int kEmuN16BCount = sizeof(kEmuN16B) / sizeof(kEmuN16B[0]);
}  // namespace emu
