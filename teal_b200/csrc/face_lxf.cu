// Face-flux kernel variants for the lxf convective flux (see kernels.cuh k_face).
#include "launch.cuh"

namespace tg {
TG_INSTANTIATE_FACE(FK_LXF)
}  // namespace tg
