// Logging stub used only when compiling the reference's CPU coefficient
// generator (core/fft/utils/rotate.cpp + core/utils wten) into oracle/_ref.
// The reference's logger lives in the Mki runtime, which is not available;
// its call sites only stream diagnostic text, so stderr stands in for it.
#pragma once
#include <iostream>
#define ASDSIP_LOG(level) std::cerr
#define ASDSIP_ELOG(code) std::cerr
