/* Stand-in for <cuda.h> when the reference kernels are compiled as host C++ (cuda_emu.h). */
#pragma once
#include "../cuda_emu.h"
