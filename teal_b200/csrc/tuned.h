// Launch shapes of the hot kernels. Defaults below; teal_b200/autotune.py times variants on the
// GPU and rewrites this file with the fastest (a value given with -D at build time wins).
#pragma once

#ifndef TG_FACE_BLOCK
#define TG_FACE_BLOCK 256  // threads per face-flux block
#endif
#ifndef TG_FACE_MINB
#define TG_FACE_MINB 2  // face-flux blocks kept resident per SM (caps registers per thread)
#endif
#ifndef TG_CELL_BLOCK
#define TG_CELL_BLOCK 256  // threads per cell-gather block
#endif
