// Stand-in for the CUDA runtime header when device sources are compiled by
// the host warp emulator.
#pragma once
#include "emu.h"
