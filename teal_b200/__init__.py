"""teal_b200: the residual / time-integration path of the teal finite-volume solver on B200 GPUs.

Hand-written sm_100a CUDA kernels behind a C ABI (include/teal_b200.h); this package is the host
mirror of teal's API over that ABI. Importing it loads the CUDA library and fails when it is not
built: there is no CPU path.
"""

from ._lib import TealError, lib  # noqa: F401  (loads libteal_b200.so or raises ImportError)
from ._lib import (  # noqa: F401
    TG_ADVANCE_EULER,
    TG_ADVANCE_IMPLICIT_EULER,
    TG_ADVANCE_LSERK,
    TG_EULER,
    TG_NAVIERSTOKES,
    TG_PRECISION_FP32_FLUX,
    TG_PRECISION_FP64,
    TG_PRECISION_FP64_EXACT,
)
from .api import (  # noqa: F401
    Batch,
    Context,
    Equations,
    Mesh,
    Simulation,
    euler_create,
    mesh_create,
    navierstokes_create,
    register_function,
)
