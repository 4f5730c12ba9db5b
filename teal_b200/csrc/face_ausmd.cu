// Face-flux kernel variants for the ausmd convective flux (see kernels.cuh k_face).
#include "launch.cuh"

namespace tg {
TG_INSTANTIATE_FACE(FK_AUSMD)
}  // namespace tg
