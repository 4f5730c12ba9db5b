"""ctypes bindings of the C ABI declared in include/teal_b200.h.

The shared library is built in-tree (teal_b200/libteal_b200.so, `python -c "import __graft_entry__;
__graft_entry__.build()"` or `make -C teal_b200/csrc`). Importing this module fails loudly when the
library is missing: there is no CPU fallback.
"""

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# TEAL_B200_LIBRARY selects another build of the same library (autotuning variants)
LIB_PATH = os.environ.get("TEAL_B200_LIBRARY") or os.path.join(_HERE, "libteal_b200.so")

TG_OK = 0
TG_ERR_INVALID = 1
TG_ERR_CUDA = 2
TG_ERR_OOM = 3
TG_ERR_NONFINITE = 4
TG_ERR_TIMEOUT = 5
TG_ERR_NO_DEVICE = 6

TG_EULER, TG_NAVIERSTOKES = 0, 1
TG_VISCOUS_NONE, TG_VISCOUS_CENTRAL = 0, 1
TG_LIMITER_NONE, TG_LIMITER_BARTH_JESPERSEN, TG_LIMITER_VENKATAKRISHNAN = 0, 1, 2
TG_ADVANCE_EULER, TG_ADVANCE_LSERK, TG_ADVANCE_IMPLICIT_EULER = 0, 1, 2
TG_PRECISION_FP64, TG_PRECISION_FP32_FLUX, TG_PRECISION_FP64_EXACT = 0, 1, 2
TG_WAIT_POLLS = 1 << 20  # default (and maximum) tries of a device-side bounded wait
TG_SOURCE_NONE, TG_SOURCE_BODY_FORCE, TG_SOURCE_BULK_FORCING, TG_SOURCE_DEVICE = 0, 1, 2, 3
TG_BC_CUSTOM = 9
TG_FUNCTION_BOUNDARY, TG_FUNCTION_SOURCE = 1, 2
TG_PREPARE_NONE, TG_PREPARE_AVERAGE = 0, 1
TG_NOALLOC_MAX_CELLS = 67108864  # cell limit of tg_residual_noalloc (its fixed scratch array)

_int_p = ctypes.POINTER(ctypes.c_int)
_dbl_p = ctypes.POINTER(ctypes.c_double)


class TgMesh(ctypes.Structure):
    """`tg_mesh`: teal's Mesh arrays (src/mesh.h:13-72)."""

    _fields_ = [
        ("num_cells", ctypes.c_int),
        ("num_inner_cells", ctypes.c_int),
        ("off_boundary_cells", ctypes.c_int),
        ("off_periodic_cells", ctypes.c_int),
        ("cell_cell_off", _int_p),
        ("cell_cell_idx", _int_p),
        ("cell_volume", _dbl_p),
        ("cell_center", _dbl_p),
        ("cell_projection", _dbl_p),
        ("cell_offset", _dbl_p),
        ("sum_volume", ctypes.c_double),
        ("num_faces", ctypes.c_int),
        ("num_inner_faces", ctypes.c_int),
        ("off_boundary_faces", ctypes.c_int),
        ("face_cell", _int_p),
        ("face_area", _dbl_p),
        ("face_basis", _dbl_p),
        ("face_weight", _dbl_p),
        ("face_offset", _dbl_p),
        ("face_correction", _dbl_p),
        ("num_entities", ctypes.c_int),
        ("num_inner_entities", ctypes.c_int),
        ("off_boundary_entities", ctypes.c_int),
        ("entity_face_off", _int_p),
        ("num_neighbors", ctypes.c_int),
        ("neighbor_tag", _int_p),
        ("neighbor_recv_off", _int_p),
        ("neighbor_send_off", _int_p),
        ("neighbor_send_idx", _int_p),
    ]


class TgEquations(ctypes.Structure):
    """`tg_equations`: the Equations plugin table by kind (src/equations.h:97-111)."""

    _fields_ = [
        ("physics", ctypes.c_int),
        ("space_order", ctypes.c_int),
        ("convective", ctypes.c_int),
        ("viscous", ctypes.c_int),
        ("limiter", ctypes.c_int),
        ("limiter_parameter", _dbl_p),
        ("limiter_coefficient", ctypes.c_double),
        ("property", ctypes.c_double * 3),
        ("num_boundaries", ctypes.c_int),
        ("boundary_kind", _int_p),
        ("boundary_context", _dbl_p),
        ("source", ctypes.c_int),
        ("source_parameter", ctypes.c_double * 4),
    ]


class TgRungeKutta(ctypes.Structure):
    _fields_ = [("time_order", ctypes.c_int), ("num_stages", ctypes.c_int)]


class TgNewtonKrylov(ctypes.Structure):
    _fields_ = [
        ("newton_tolerance", ctypes.c_double),
        ("krylov_tolerance", ctypes.c_double),
        ("krylov_dimension", ctypes.c_int),
    ]


# every exported entry point of include/teal_b200.h: (name, restype, argtypes)
_vp = ctypes.c_void_p
SIGNATURES = [
    ("tg_convective_select", ctypes.c_int, [ctypes.c_char_p]),
    ("tg_viscous_select", ctypes.c_int, [ctypes.c_char_p]),
    ("tg_limiter_select", ctypes.c_int, [ctypes.c_char_p]),
    ("tg_boundary_select", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int]),
    ("tg_advance_select", ctypes.c_int, [ctypes.c_char_p]),
    ("tg_source_select", ctypes.c_int, [ctypes.c_char_p]),
    ("tg_create", ctypes.c_int, [ctypes.POINTER(TgMesh), ctypes.POINTER(TgEquations), ctypes.c_int,
                                 ctypes.POINTER(_vp)]),
    ("tg_destroy", ctypes.c_int, [_vp]),
    ("tg_last_error", ctypes.c_char_p, []),
    ("tg_set_stream", ctypes.c_int, [_vp, _vp]),
    ("tg_set_wait_limit", ctypes.c_int, [_vp, ctypes.c_int]),
    ("tg_set_primitive", ctypes.c_int, [_vp, _vp]),
    ("tg_get_primitive", ctypes.c_int, [_vp, _vp]),
    ("tg_derivative", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double]),
    ("tg_gradient", ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int, _vp]),
    ("tg_timestep", ctypes.c_int, [_vp, _dbl_p]),
    ("tg_residual", ctypes.c_int, [_vp, _vp, _vp]),
    ("tg_advance", ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_double, _dbl_p, ctypes.c_double,
                                  _vp, _dbl_p]),
    ("tg_advance_host", ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_double, _dbl_p, ctypes.c_double,
                                       _vp, _vp, _vp, _dbl_p]),
    ("tg_run", ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                              ctypes.c_int, ctypes.c_double, _dbl_p, _int_p, _vp]),
    ("tg_last_step", ctypes.c_int, [_vp, ctypes.c_int, _dbl_p]),
    ("tg_batch_create", ctypes.c_int, [ctypes.POINTER(TgMesh), ctypes.POINTER(TgEquations), ctypes.c_int,
                                       ctypes.c_int, ctypes.POINTER(_vp)]),
    ("tg_batch_size", ctypes.c_int, [_vp, _int_p]),
    ("tg_batch_set_primitive", ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    ("tg_batch_get_primitive", ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    ("tg_batch_run", ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_double, _vp, _vp, _vp, _vp, _vp, _vp,
                                    _vp]),
    ("tg_batch_status", ctypes.c_int, [_vp, _vp]),
    ("tg_create_partition", ctypes.c_int, [ctypes.POINTER(TgMesh), ctypes.POINTER(TgEquations), ctypes.c_int, _vp,
                                           ctypes.c_int, _vp, ctypes.c_int, ctypes.POINTER(_vp)]),
    ("tg_part_buffers", ctypes.c_int, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                       ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_long)]),
    ("tg_part_step_begin", ctypes.c_int, [_vp, _dbl_p]),
    ("tg_part_set_step", ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double]),
    ("tg_part_phase", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int]),
    ("tg_part_residual_sums", ctypes.c_int, [_vp, _vp]),
    ("tg_stream_of", ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    ("tg_lserk_alpha", ctypes.c_int, [ctypes.c_int, ctypes.c_int, _dbl_p]),
    ("tg_bind", ctypes.c_int, [_vp, _vp, _vp]),
    ("tg_unbind", ctypes.c_int, [_vp]),
    ("tg_teal_euler", ctypes.c_double, [_vp, _dbl_p, _vp, ctypes.c_double, ctypes.c_double, _vp]),
    ("tg_teal_lserk", ctypes.c_double, [_vp, _dbl_p, _vp, ctypes.c_double, ctypes.c_double, _vp]),
    ("tg_teal_implicit_euler", ctypes.c_double, [_vp, _dbl_p, _vp, ctypes.c_double, ctypes.c_double,
                                                 _vp]),
    ("tg_host_mesh_cartesian", ctypes.c_int, [_dbl_p, _dbl_p, _int_p, _int_p, _dbl_p, ctypes.POINTER(_vp)]),
    ("tg_host_mesh_cells", ctypes.c_int, [ctypes.c_int, _dbl_p, ctypes.c_int, ctypes.c_int, _int_p, _int_p,
                                          ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), _int_p,
                                          ctypes.POINTER(_vp)]),
    ("tg_host_mesh_cells_periodic", ctypes.c_int,
     [ctypes.c_int, _dbl_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _int_p, _int_p, ctypes.c_int, ctypes.c_int,
      ctypes.POINTER(ctypes.c_char_p), _int_p, _dbl_p, _dbl_p, ctypes.c_int, _int_p, _int_p, _int_p, _int_p,
      ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), _dbl_p, _dbl_p, ctypes.POINTER(_vp)]),
    ("tg_host_mesh_cartesian_split", ctypes.c_int,
     [_dbl_p, _dbl_p, _int_p, _int_p, _dbl_p, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), _dbl_p, _dbl_p,
      ctypes.POINTER(_vp)]),
    ("tg_host_mesh_view", ctypes.c_int, [_vp, ctypes.POINTER(TgMesh)]),
    ("tg_host_mesh_entity", ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), _int_p,
                                           _int_p]),
    ("tg_host_mesh_nodes", ctypes.c_int, [_vp, _int_p, ctypes.POINTER(_dbl_p), ctypes.POINTER(_int_p),
                                          ctypes.POINTER(_int_p)]),
    ("tg_host_mesh_destroy", ctypes.c_int, [_vp]),
    ("tg_profile", ctypes.c_int, [_vp, ctypes.c_int]),
    ("tg_profile_read", ctypes.c_int, [_vp, _vp, _vp]),
    ("tg_launch_count", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_long)]),
    ("tg_layout", ctypes.c_int, [_vp, ctypes.c_char_p, _vp, ctypes.c_long]),
    ("tg_residual_noalloc", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_double, _vp, _vp]),
    ("tg_function_register", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p,
                                            ctypes.c_long]),
    ("tg_bind_boundary_function", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_char_p]),
    ("tg_bind_source_function", ctypes.c_int, [_vp, ctypes.c_char_p]),
    ("tg_bind_source_prepare", ctypes.c_int, [_vp, ctypes.c_int]),
    ("tg_build_info", ctypes.c_char_p, []),
]


def load(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(
            f"teal_b200: the CUDA library {path} is not built; run "
            "`python -c 'import __graft_entry__ as g; g.build()'` (no CPU fallback exists)")
    lib = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load()


class TealError(RuntimeError):
    """A nonzero status of the C ABI (teal itself would exit through teal_error)."""

    def __init__(self, code, message):
        super().__init__(f"[{code}] {message}")
        self.code = code


def check(status):
    if status != TG_OK:
        raise TealError(status, lib.tg_last_error().decode(errors="replace"))
    return status
