// Face-flux kernel variants for the none convective flux (see kernels.cuh k_face).
#include "launch.cuh"

namespace tg {
TG_INSTANTIATE_FACE(FK_NONE)
}  // namespace tg
