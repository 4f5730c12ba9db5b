// Face-flux kernels for the ausmd convective flux with teal's exact FP64 arithmetic (TG_EXACT_TU=1,
// -fmad=false; see physics.cuh).
#include "launch.cuh"

namespace tg {
TG_INSTANTIATE_FACE_EXACT(FK_AUSMD)
}  // namespace tg
