"""Python binding of libstable-fluids.so, the B200 build of the stable-fluids
C ABI (include/stable-fluids-3d.h, include/stable-fluids-b200.h).

The binding is ctypes over the C ABI -- the same entry points a C/C++ caller
such as the reference's benchmark.cu uses -- plus a small `Simulation` helper
that owns a CUDA stream and moves fields between numpy / torch and the
library. torch is used only for device buffers and streams.

The package directory name contains a hyphen; import it with
``importlib.import_module("stable-fluids_b200")``.

The same `Simulation` class can drive any library that exports the seven
upstream symbols (stable-fluids-3d.h:112-154), which is how the tests run the
reference backend side by side with this one.
"""

from __future__ import annotations

import ctypes
import os
import pathlib
from ctypes import POINTER, byref, c_double, c_float, c_int32, c_uint32, c_uint64, c_void_p

_HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = _HERE / "libstable-fluids.so"

# ----------------------------------------------------------------- enums --
RESULT_OK, RESULT_OUT_OF_MEMORY, RESULT_BACKEND_FAILURE = 0, 1, 2

FLOW_NO_SLIP_WALL, FLOW_FREE_SLIP_WALL, FLOW_OUTFLOW, FLOW_PERIODIC = 0, 1, 2, 3
SCALAR_FIXED_VALUE, SCALAR_ZERO_FLUX, SCALAR_PERIODIC = 0, 1, 2
VECTOR_FIELD_FORCE = 0

VIEW_SCALAR_FIELD_DATA = 0
VIEW_SCALAR_FIELD_SOURCE = 1
VIEW_VECTOR_FIELD = 2
VIEW_FLOW_VELOCITY = 3
VIEW_FLOW_VELOCITY_MAGNITUDE = 4
VIEW_FLOW_PRESSURE = 5
VIEW_FLOW_DIVERGENCE = 6
VIEW_LAYOUT_F32_3D, VIEW_LAYOUT_F32_3D_SOA3 = 0, 1

SCHEME_RBGS, SCHEME_JACOBI = 0, 1
WARM_START_ZERO, WARM_START_PREVIOUS, WARM_START_LEARNED = 0, 1, 2
STORAGE_FP32, STORAGE_BF16 = 0, 1


# -------------------------------------------------------------- structs --
class FlowFace(ctypes.Structure):
    _fields_ = [("type", c_uint32), ("velocity_x", c_float), ("velocity_y", c_float), ("velocity_z", c_float), ("pressure", c_float)]


class FlowBoundary(ctypes.Structure):
    _fields_ = [(n, FlowFace) for n in ("x_minus", "x_plus", "y_minus", "y_plus", "z_minus", "z_plus")]


class ScalarFace(ctypes.Structure):
    _fields_ = [("type", c_uint32), ("value", c_float)]


class ScalarBoundary(ctypes.Structure):
    _fields_ = [(n, ScalarFace) for n in ("x_minus", "x_plus", "y_minus", "y_plus", "z_minus", "z_plus")]


class SimulationConfig(ctypes.Structure):
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32),
        ("cell_size", c_float), ("dt", c_float), ("viscosity", c_float),
        ("diffuse_iterations", c_int32), ("pressure_iterations", c_int32),
        ("flow_boundary", FlowBoundary),
    ]


class ScalarFieldDesc(ctypes.Structure):
    _fields_ = [("diffusion", c_float), ("dissipation", c_float), ("initial_value", c_float), ("boundary", ScalarBoundary)]


class VectorFieldDesc(ctypes.Structure):
    _fields_ = [("usage", c_uint32), ("initial_value_x", c_float), ("initial_value_y", c_float), ("initial_value_z", c_float)]


class ContextCreateDesc(ctypes.Structure):
    _fields_ = [
        ("config", SimulationConfig), ("stream", c_void_p),
        ("scalar_fields", POINTER(ScalarFieldDesc)), ("scalar_field_count", c_uint32),
        ("vector_fields", POINTER(VectorFieldDesc)), ("vector_field_count", c_uint32),
    ]


class ViewRequest(ctypes.Structure):
    _fields_ = [("kind", c_uint32), ("scalar_field", c_uint32), ("vector_field", c_uint32), ("consumer_stream", c_void_p)]


class View(ctypes.Structure):
    _fields_ = [
        ("layout", c_uint32), ("nx", c_int32), ("ny", c_int32), ("nz", c_int32),
        ("row_stride_bytes", c_uint64), ("slice_stride_bytes", c_uint64),
        ("data0", c_void_p), ("data1", c_void_p), ("data2", c_void_p),
    ]


class B200Options(ctypes.Structure):
    _fields_ = [
        ("scheme", c_uint32), ("warm_start", c_uint32), ("iterations_per_pass", c_int32),
        ("residual_tolerance", c_float), ("max_pressure_iterations", c_int32),
        ("residual_check_interval", c_int32), ("compute_residual", c_uint32),
        ("warm_start_trial_iterations", c_int32), ("storage", c_uint32), ("warm_start_coarsening", c_uint32), ("reserved", c_uint32 * 6),
    ]


class B200StepStats(ctypes.Structure):
    _fields_ = [
        ("rel_residual", c_double), ("rhs_norm", c_double), ("pressure_iterations", c_int32),
        ("hit_cap", c_int32), ("used_fallback", c_int32), ("reserved", c_int32),
    ]


ABI_SYMBOLS = (
    "stable_fluids_create_context_cuda",
    "stable_fluids_destroy_context_cuda",
    "stable_fluids_update_scalar_field_cuda",
    "stable_fluids_update_scalar_field_source_cuda",
    "stable_fluids_update_vector_field_cuda",
    "stable_fluids_step_cuda",
    "stable_fluids_get_view_cuda",
)
B200_SYMBOLS = (
    "stable_fluids_b200_default_options",
    "stable_fluids_b200_create_context",
    "stable_fluids_b200_get_step_stats",
    "stable_fluids_b200_stage_vector_field",
    "stable_fluids_b200_read_view_async",
    "stable_fluids_b200_enqueue_stage",
    "stable_fluids_b200_get_step_info",
    "stable_fluids_b200_pressure_residual_noalloc",
    "stable_fluids_b200_network_create",
    "stable_fluids_b200_network_destroy",
    "stable_fluids_b200_network_parameters",
    "stable_fluids_b200_network_set_parameters",
    "stable_fluids_b200_network_predict",
    "stable_fluids_b200_network_gradients",
    "stable_fluids_b200_network_train_step",
    "stable_fluids_b200_attach_network",
    "stable_fluids_b200_render_volume",
    "stable_fluids_b200_plume_scene_setup",
    "stable_fluids_b200_plume_scene_forces",
    "stable_fluids_b200_batch_create",
    "stable_fluids_b200_batch_create_ex",
    "stable_fluids_b200_batch_layout",
    "stable_fluids_b200_batch_step",
    "stable_fluids_b200_batch_info",
    "stable_fluids_b200_batch_destroy",
)

(STAGE_FORCES, STAGE_VELOCITY_ADVECTION, STAGE_VELOCITY_DIFFUSION, STAGE_DIVERGENCE, STAGE_PRESSURE,
 STAGE_PROJECTION, STAGE_SCALARS, STAGE_DIAGNOSTICS, STAGE_STEP) = range(9)


BATCH_GRAPHS, BATCH_WORK_TABLE = 0, 1


class B200BatchOptions(ctypes.Structure):
    _fields_ = [("mode", c_uint32), ("autotune", c_uint32), ("tile_cache", ctypes.c_char_p), ("chains", c_uint32), ("reserved", c_uint32 * 3)]


class B200VolumeRender(ctypes.Structure):
    _fields_ = [
        ("eye", c_float * 3), ("right", c_float * 3), ("up", c_float * 3), ("forward", c_float * 3),
        ("volume_min", c_float * 3), ("volume_max", c_float * 3), ("color_a", c_float * 3), ("color_b", c_float * 3),
        ("aspect", c_float), ("tan_half_fov", c_float), ("value_scale", c_float), ("density", c_float),
        ("value_min", c_float), ("value_max", c_float), ("ortho_height", c_float),
        ("steps", c_uint32), ("projection", c_uint32), ("width", c_int32), ("height", c_int32), ("reserved", c_uint32 * 4),
    ]


class B200StepInfo(ctypes.Structure):
    _fields_ = [("kernels_per_step", c_int32), ("scheme", c_uint32), ("iterations_per_pass", c_int32), ("blocked", c_int32), ("device_bytes", c_uint64), ("kernels_per_check", c_int32), ("reserved", c_int32)]


def _bind(lib: ctypes.CDLL, extended: bool) -> ctypes.CDLL:
    P = c_void_p
    lib.stable_fluids_create_context_cuda.argtypes = [POINTER(ContextCreateDesc), POINTER(c_void_p), POINTER(c_uint32), c_uint32, POINTER(c_uint32), c_uint32]
    lib.stable_fluids_destroy_context_cuda.argtypes = [P]
    lib.stable_fluids_update_scalar_field_cuda.argtypes = [P, c_uint32, P]
    lib.stable_fluids_update_scalar_field_source_cuda.argtypes = [P, c_uint32, P]
    lib.stable_fluids_update_vector_field_cuda.argtypes = [P, c_uint32, P, P, P]
    lib.stable_fluids_step_cuda.argtypes = [P]
    lib.stable_fluids_get_view_cuda.argtypes = [P, POINTER(ViewRequest), POINTER(View)]
    for name in ABI_SYMBOLS:
        getattr(lib, name).restype = c_int32
    if extended:
        lib.stable_fluids_b200_default_options.argtypes = [POINTER(B200Options)]
        lib.stable_fluids_b200_create_context.argtypes = [POINTER(ContextCreateDesc), POINTER(B200Options), POINTER(c_void_p), POINTER(c_uint32), c_uint32, POINTER(c_uint32), c_uint32]
        lib.stable_fluids_b200_get_step_stats.argtypes = [P, POINTER(B200StepStats)]
        lib.stable_fluids_b200_stage_vector_field.argtypes = [P, c_uint32, P, P, P, P]
        lib.stable_fluids_b200_read_view_async.argtypes = [P, POINTER(ViewRequest), P, P, P, P]
        lib.stable_fluids_b200_enqueue_stage.argtypes = [P, c_uint32, POINTER(c_int32)]
        lib.stable_fluids_b200_get_step_info.argtypes = [P, POINTER(B200StepInfo)]
        lib.stable_fluids_b200_pressure_residual_noalloc.argtypes = [P, P, c_int32, c_int32, c_int32, c_float, POINTER(FlowBoundary), P, P]
        lib.stable_fluids_b200_network_create.argtypes = [c_uint32, POINTER(c_void_p)]
        lib.stable_fluids_b200_network_destroy.argtypes = [P]
        lib.stable_fluids_b200_network_parameters.argtypes = [P, POINTER(c_uint64), P]
        lib.stable_fluids_b200_network_set_parameters.argtypes = [P, P]
        lib.stable_fluids_b200_network_predict.argtypes = [P, P, P, c_int32, c_int32, c_int32, c_float, P, P]
        lib.stable_fluids_b200_network_gradients.argtypes = [P, P, P, P, c_int32, c_int32, c_int32, c_float, POINTER(c_double), P, P]
        lib.stable_fluids_b200_network_train_step.argtypes = [P, P, P, P, c_int32, c_int32, c_int32, c_float, c_float, POINTER(c_double), P]
        lib.stable_fluids_b200_attach_network.argtypes = [P, P]
        lib.stable_fluids_b200_render_volume.argtypes = [P, POINTER(ViewRequest), POINTER(B200VolumeRender), P]
        lib.stable_fluids_b200_plume_scene_setup.argtypes = [P, c_uint32, c_uint32]
        lib.stable_fluids_b200_plume_scene_forces.argtypes = [P, c_uint32, c_int32]
        lib.stable_fluids_b200_batch_create.argtypes = [POINTER(c_void_p), c_uint32, POINTER(c_void_p)]
        lib.stable_fluids_b200_batch_create_ex.argtypes = [POINTER(c_void_p), c_uint32, POINTER(B200BatchOptions), POINTER(c_void_p)]
        lib.stable_fluids_b200_batch_layout.argtypes = [P, POINTER(c_uint32), POINTER(c_uint32), POINTER(c_int32), c_uint32]
        lib.stable_fluids_b200_batch_step.argtypes = [P]
        lib.stable_fluids_b200_batch_info.argtypes = [P, POINTER(c_uint32), POINTER(c_int32), POINTER(c_void_p)]
        lib.stable_fluids_b200_batch_destroy.argtypes = [P]
        for name in B200_SYMBOLS:
            getattr(lib, name).restype = c_int32
    return lib


def load_library(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    """Loads libstable-fluids.so (this project's build by default). Raises if
    the library has not been built: there is no fallback implementation."""
    p = pathlib.Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing; build it with `make -C {p.parent}` (or __graft_entry__.build())")
    lib = ctypes.CDLL(str(p))
    extended = hasattr(lib, "stable_fluids_b200_create_context")
    lib._sf_extended = extended
    return _bind(lib, extended)


def default_options(lib: ctypes.CDLL | None = None) -> B200Options:
    lib = lib or load_library()
    o = B200Options()
    rc = lib.stable_fluids_b200_default_options(byref(o))
    if rc != RESULT_OK:
        raise RuntimeError(f"stable_fluids_b200_default_options failed ({rc})")
    return o


from .simulation import Batch, Simulation, StableFluidsError  # noqa: E402  (needs the structs above)
from . import scenes  # noqa: E402
from .warmstart import WarmStartNetwork, LAYERS as NETWORK_LAYERS  # noqa: E402

__all__ = [
    "Simulation", "Batch", "StableFluidsError", "load_library", "default_options", "scenes", "WarmStartNetwork", "NETWORK_LAYERS",
    "SimulationConfig", "ScalarFieldDesc", "VectorFieldDesc", "ContextCreateDesc", "FlowBoundary", "FlowFace",
    "ScalarBoundary", "ScalarFace", "ViewRequest", "View", "B200Options", "B200StepStats", "B200StepInfo",
]
