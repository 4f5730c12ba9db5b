// Launch shapes of the hot kernels, chosen by teal_b200/autotune.py on a B200 (fastest
// measured RK step, TGV 96^3 FP64: 1.411 ms vs 1.455 ms for 256 / 2 / 256); a value given with -D
// at build time wins.
#pragma once

#ifndef TG_FACE_BLOCK
#define TG_FACE_BLOCK 128  // threads per face-flux block
#endif
#ifndef TG_FACE_MINB
#define TG_FACE_MINB 4  // face-flux blocks kept resident per SM (caps registers per thread)
#endif
#ifndef TG_CELL_BLOCK
#define TG_CELL_BLOCK 256  // threads per cell-gather block
#endif
