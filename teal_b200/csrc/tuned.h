// Launch shapes of the hot kernels, chosen by teal_b200/autotune.py on a B200 (fastest measured RK
// step: TGV for the face, cell and gradient shapes and the Navier-Stokes staging switch, the ramp
// for the Euler staging switch and the Euler face occupancy; times within 0.5 % of the fastest
// count as ties, resolved to fewer resident face blocks, i.e. more registers per thread). From the
// later sweeps: cell 0.113 vs 0.133 ms per TGV 128^3 launch, gradient 0.264 vs 0.280 ms, Euler face
// 0.271 ms at 28 blocks against 0.290 at 24 and 0.318 at 20 (ramp 80^3), FP32-flux face 0.309 ms at
// 32 blocks against 0.326 at 20 (TGV 128^3). A value given with -D at build time wins.
#pragma once

#ifndef TG_FACE_BLOCK
#define TG_FACE_BLOCK 32  // threads per face-flux block
#endif
#ifndef TG_FACE_MINB
#define TG_FACE_MINB 20  // Navier-Stokes face-flux blocks kept resident per SM (caps registers per thread)
#endif
#ifndef TG_FACE_MINB_FP32
#define TG_FACE_MINB_FP32 32  // FP32-flux face-flux blocks kept resident per SM (caps registers per thread)
#endif
#ifndef TG_FACE_MINB_EULER
#define TG_FACE_MINB_EULER 28  // Euler face-flux blocks kept resident per SM (caps registers per thread)
#endif
#ifndef TG_CELL_BLOCK
#define TG_CELL_BLOCK 128  // threads per cell-gather block
#endif
#ifndef TG_FACE_STAGED_NS
#define TG_FACE_STAGED_NS 0  // Navier-Stokes face kernel: geometry staged by bulk copies (1) or loaded (0)
#endif
#ifndef TG_FACE_STAGED_EULER
#define TG_FACE_STAGED_EULER 1  // Euler face kernel: geometry staged by bulk copies (1) or loaded (0)
#endif
#ifndef TG_CELL_MINB
#define TG_CELL_MINB 12  // cell-gather blocks kept resident per SM (caps registers per thread)
#endif
#ifndef TG_GRAD_MINB
#define TG_GRAD_MINB 12  // gradient blocks (160 threads) kept resident per SM (caps registers per thread)
#endif
