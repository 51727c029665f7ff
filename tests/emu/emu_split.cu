// Emulator instantiations of the split configurations (configs.h).
#include "emu_core.h"

namespace emu {
extern const SplitEntry kEmuSplit[] = {NTTB_SPLIT_ALL(EMU_SPLIT_ENTRY)};
extern const int kEmuSplitCount = sizeof(kEmuSplit) / sizeof(kEmuSplit[0]);
}  // namespace emu
