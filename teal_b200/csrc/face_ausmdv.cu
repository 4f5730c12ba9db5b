// Face-flux kernel variants for the ausmdv convective flux (see kernels.cuh k_face).
#include "launch.cuh"

namespace tg {
TG_INSTANTIATE_FACE(FK_AUSMDV)
}  // namespace tg
