"""ctypes binding of the dsmc_b200 C ABI (include/dsmc_b200.h).

The shared library is built in-tree (cudadsmc_b200/libdsmc_b200.so) by
``cudadsmc_b200.build.build()``.  Importing this module without it raises:
there is no CPU or Python fallback for the timestep.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdsmc_b200.so")

DSMC_OK = 0
STATUS = {
    0: "ok", 1: "invalid argument", 2: "configuration error", 3: "CUDA error",
    4: "out of device memory", 5: "call out of order", 6: "particle capacity exceeded",
    7: "I/O error", 8: "device error flag",
}
FACE = {"specular": 0, "diffuse": 1, "outflow": 2, "periodic": 3, "inflow": 4}
RNG = {"taus": 0, "philox": 1}
INIT = {"reference": 0, "maxwell": 1, "bimodal": 2}

c_float3 = ctypes.c_float * 3
c_int3 = ctypes.c_int * 3
c_uint3 = ctypes.c_uint32 * 3


class Config(ctypes.Structure):
    """dsmc_config: the reference's settings_t plus the extensions."""
    _fields_ = [
        ("grid_min", c_float3), ("grid_max", c_float3), ("grid_dim", c_int3),
        ("density", ctypes.c_float), ("fnum", ctypes.c_float), ("temp", ctypes.c_float),
        ("stream_vel", c_float3), ("periodic", ctypes.c_char),
        ("gas_mass", ctypes.c_float), ("gas_diam", ctypes.c_float), ("gas_tref", ctypes.c_float),
        ("dt", ctypes.c_float), ("geometry", ctypes.c_int), ("benchmark", ctypes.c_int),
        ("gas_omega", ctypes.c_float), ("ntc_local", ctypes.c_int), ("rng", ctypes.c_int),
        ("seed", ctypes.c_uint64), ("face_mode", ctypes.c_int),
        ("face_kind", ctypes.c_int * 6), ("face_temp", ctypes.c_float * 6),
        ("wall_diffuse", ctypes.c_int), ("wall_temp", ctypes.c_float),
        ("init_kind", ctypes.c_int), ("init_temp2", ctypes.c_float),
        ("sample_every", ctypes.c_int), ("capacity_factor", ctypes.c_float),
        ("part_per_cell", ctypes.c_uint32), ("geom_nearest", ctypes.c_int),
    ]


class Info(ctypes.Structure):
    _fields_ = [
        ("part_per_cell", ctypes.c_uint32), ("cells", ctypes.c_uint32),
        ("capacity", ctypes.c_uint32), ("num_particles", ctypes.c_uint32),
        ("cell_size", c_float3), ("cell_volume", ctypes.c_float),
        ("cross_section", ctypes.c_float), ("max_rel_vel", ctypes.c_float),
        ("step", ctypes.c_uint64), ("samples", ctypes.c_uint32), ("sim_time", ctypes.c_double),
        ("particle_steps", ctypes.c_uint64), ("injected", ctypes.c_uint32),
        ("removed", ctypes.c_uint32), ("giant_cells", ctypes.c_uint32),
        ("mesh_flights", ctypes.c_uint32),
    ]


class Grid(ctypes.Structure):
    _fields_ = [("gmin", c_float3), ("gmax", c_float3), ("cell", c_float3), ("dim", c_uint3)]


class CollideParams(ctypes.Structure):
    _fields_ = [
        ("ncells", ctypes.c_uint32), ("cell_volume", ctypes.c_float),
        ("cross_section", ctypes.c_float), ("fnum", ctypes.c_float),
        ("avg_conc", ctypes.c_float), ("dt", ctypes.c_float), ("omega", ctypes.c_float),
        ("vhs_gref", ctypes.c_float), ("ntc_local", ctypes.c_int), ("rng", ctypes.c_int),
        ("seed", ctypes.c_uint64), ("step", ctypes.c_uint32),
    ]


class MoveParams(ctypes.Structure):
    _fields_ = [
        ("grid", Grid), ("dt", ctypes.c_float), ("periodic", ctypes.c_char),
        ("face_mode", ctypes.c_int), ("face_kind", ctypes.c_int * 6),
        ("face_vstd", ctypes.c_float * 6), ("seed", ctypes.c_uint64), ("step", ctypes.c_uint32),
    ]


# (name, restype, argtypes) of every exported entry point.
_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_I = ctypes.c_int
SIGNATURES = [
    ("dsmc_config_default", _I, [ctypes.POINTER(Config)]),
    ("dsmc_config_read_xml", _I, [ctypes.c_char_p, ctypes.POINTER(Config)]),
    ("dsmc_config_from_args", _I, [_I, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(Config),
                                   ctypes.POINTER(ctypes.c_float)]),
    ("dsmc_create", _I, [ctypes.POINTER(Config), ctypes.POINTER(_P)]),
    ("dsmc_destroy", _I, [_P]),
    ("dsmc_last_error", ctypes.c_char_p, [_P]),
    ("dsmc_status_string", ctypes.c_char_p, [_I]),
    ("dsmc_set_stream", _I, [_P, _P]),
    ("dsmc_sync", _I, [_P]),
    ("dsmc_get_info", _I, [_P, ctypes.POINTER(Info)]),
    ("dsmc_profile", _I, [_P, _I]),
    ("dsmc_profile_read", _I, [_P, _P, _P]),
    ("dsmc_set_mesh", _I, [_P, _P, _U32, _P, _U32, _P, _P]),
    ("dsmc_set_geometry_grid", _I, [_P, _P, _P, _P, _P, _P, _P, _P, _U32, _P, _U32, _P]),
    ("dsmc_build_geometry_grid", _I, [_P, _U32, _P, _U32, _P, _P, _P, _P, _P, ctypes.c_uint64,
                                      _P, ctypes.POINTER(ctypes.c_uint64)]),
    ("dsmc_get_geometry_grid", _I, [_P, _P, _P, _P, _P, _P, _P, ctypes.c_uint64, _P,
                                    ctypes.POINTER(ctypes.c_uint64)]),
    ("dsmc_get_entry_reach", _I, [_P, _P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    ("dsmc_get_cell_slabs", _I, [_P, _P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    ("dsmc_read_raw_mesh", _I, [ctypes.c_char_p, _P, ctypes.POINTER(_U32), _P,
                                ctypes.POINTER(_U32), _P]),
    ("dsmc_mesh_icosphere", _I, [_I, ctypes.c_float, _P, _P, ctypes.POINTER(_U32), _P,
                                 ctypes.POINTER(_U32)]),
    ("dsmc_mesh_capsule", _I, [ctypes.c_float, ctypes.c_float, ctypes.c_float, _P, _U32,
                               ctypes.c_uint64, _P, ctypes.POINTER(_U32), _P,
                               ctypes.POINTER(_U32)]),
    ("dsmc_init_state", _I, [_P, _P, ctypes.POINTER(_U32)]),
    ("dsmc_upload_state", _I, [_P, _P, _P, _U32, _I]),
    ("dsmc_download_state", _I, [_P, _P, _P, ctypes.POINTER(_U32), _I]),
    ("dsmc_read_keys", _I, [_P, _P, ctypes.POINTER(_U32)]),
    ("dsmc_set_cell_state", _I, [_P, _P, _P]),
    ("dsmc_get_cell_state", _I, [_P, _P, _P]),
    ("dsmc_set_twisters", _I, [_P, _P, _P, _I]),
    ("dsmc_get_twisters", _I, [_P, _P]),
    ("dsmc_read_twisters", _I, [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, _P]),
    ("dsmc_step", _I, [_P, ctypes.c_float, _I]),
    ("dsmc_step_graph", _I, [_P, ctypes.c_float, _I]),
    ("dsmc_init_from_fields", _I, [_P, _P, _P]),
    ("dsmc_init_from_fields_two_stream", _I, [_P, _P, ctypes.c_float, _P]),
    ("dsmc_gemm_bf16", _I, [_I, _I, _I, _P, _I, _I, _P, _I, _I, _P, _I, ctypes.c_float, _P, _I, _P,
                            _I, _I, _P]),
    ("dsmc_gemm_check", _I, [_P]),
    ("dsmc_gelu_backward", _I, [_P, _P, _P, _P, ctypes.c_size_t, _P]),
    ("dsmc_colsum", _I, [_P, _I, _I, _I, _P, _P]),
    ("dsmc_mse_grad", _I, [_P, _P, ctypes.c_size_t, ctypes.c_float, _P, _P, _P, _P, _P]),
    ("dsmc_adam_step", _I, [_P, _P, _P, _P, _P, ctypes.c_size_t, ctypes.c_float, ctypes.c_float,
                            ctypes.c_float, ctypes.c_float, _I, ctypes.c_float, _P]),
    ("dsmc_to_bf16", _I, [_P, _P, ctypes.c_size_t, _P]),
    ("dsmc_set_kernel_variant", _I, [_P, _I]),
    ("dsmc_get_kernel_variant", _I, [_P, _P, _P]),
    ("dsmc_profile_read_kernels", _I, [_P, _I, _P, _P]),
    ("dsmc_profile_mask", _I, [_P, ctypes.c_uint32]),
    ("dsmc_clearance_at", _I, [_P, _P, _U32, _P, _P]),
    ("dsmc_kernel_variant_count", _I, []),
    ("dsmc_autotune", _I, [_P, ctypes.c_float, _I, _P, _P]),
    ("dsmc_batch_create", _I, [_P, _U32, _P]),
    ("dsmc_batch_destroy", _I, [_P]),
    ("dsmc_batch_last_error", ctypes.c_char_p, [_P]),
    ("dsmc_batch_set_stream", _I, [_P, _P]),
    ("dsmc_batch_step", _I, [_P, _P, _I]),
    ("dsmc_batch_sync", _I, [_P]),
    ("dsmc_batch_autotune", _I, [_P, _P, _I, _P]),
    ("dsmc_sample", _I, [_P]),
    ("dsmc_reset_samples", _I, [_P]),
    ("dsmc_read_cell_sums", _I, [_P, _P, ctypes.POINTER(_U32)]),
    ("dsmc_read_fields", _I, [_P, _P]),
    ("dsmc_get_totals", _I, [_P, _P]),
    ("dsmc_totals_async", _I, [_P, _P]),
    ("dsmc_dump_statistics", _I, [_P, ctypes.c_char_p]),
    ("dsmc_snapshot", _I, [_P, ctypes.c_char_p]),
    ("dsmc_restore", _I, [_P, ctypes.c_char_p]),
    ("dsmc_stage_cell_index", _I, [ctypes.POINTER(Grid), _P, _P, _P, _U32, _P, _P, _P]),
    ("dsmc_stage_sort_workspace", _I, [_U32, _U32, ctypes.POINTER(ctypes.c_size_t)]),
    ("dsmc_stage_sort", _I, [_P, _P, _U32, _U32, _P, _P, ctypes.c_size_t, _P]),
    ("dsmc_stage_sort_static", _I, [_P, _P, _U32, _U32, _P, _P]),
    ("dsmc_stage_bounds_reorder", _I, [_P, _P, _U32, _U32, _P, _P, _P, _P]),
    ("dsmc_stage_collide", _I, [ctypes.POINTER(CollideParams), _P, _P, _P, _P, _P, _P, _P, _P]),
    ("dsmc_stage_move", _I, [_P, ctypes.POINTER(MoveParams), _P, _P, _P, _P, _P, _P, _U32, _P]),
    ("dsmc_stage_sample", _I, [_P, _P, _P, _P, _U32, _P, _P]),
]

_lib = None


def lib():
    """Loads libdsmc_b200.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -c 'import cudadsmc_b200.build as b; "
                "b.build()'` (the DSMC step has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class DsmcError(RuntimeError):
    def __init__(self, status, where, detail=""):
        msg = f"{where}: {STATUS.get(status, status)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)
        self.status = status


def check(status, where, handle=None):
    if status != DSMC_OK:
        detail = lib().dsmc_last_error(handle)
        raise DsmcError(status, where, detail.decode() if detail else "")
