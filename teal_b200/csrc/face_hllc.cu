// Face-flux kernel variants for the hllc convective flux (see kernels.cuh k_face).
#include "launch.cuh"

namespace tg {
TG_INSTANTIATE_FACE(FK_HLLC)
}  // namespace tg
