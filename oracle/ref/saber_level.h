/*
 * Selects the Saber level when the reference's Saber kernels are compiled as host C++
 * (force-included before them; TEST INFRASTRUCTURE ONLY).  The reference fixes its level in
 * SABER-GPU/include/params.h:6 (SABER_L 3) and derives mu and eT from it there (:10-19);
 * this header includes that file once and then redefines the three level parameters for
 * REF_SABER_L, so that every size macro of params.h (all defined in terms of them) follows.
 * The values are the Saber specification's: LightSaber l=2 mu=10 eT=3, Saber l=3 mu=8
 * eT=4, FireSaber l=4 mu=6 eT=6 (the same table as params.h:10-19).
 */
#pragma once
#include "cuda_emu.h"
#include "include/params.h"
#undef SABER_L
#undef SABER_MU
#undef SABER_ET
#if REF_SABER_L == 2
#define SABER_L 2
#define SABER_MU 10
#define SABER_ET 3
#elif REF_SABER_L == 3
#define SABER_L 3
#define SABER_MU 8
#define SABER_ET 4
#elif REF_SABER_L == 4
#define SABER_L 4
#define SABER_MU 6
#define SABER_ET 6
#else
#error "REF_SABER_L must be 2, 3 or 4"
#endif
