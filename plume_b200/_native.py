"""ctypes binding of libplume_b200.so (include/plume_b200.h).

There is no fallback: importing a kernel wrapper without the built library, or calling one without a CUDA
device, raises. Device arrays are torch tensors (float32, contiguous, on the current CUDA device); every call
is enqueued on torch's current stream.
"""

import ctypes
from pathlib import Path

import torch

LIBRARY = Path(__file__).resolve().parent / "libplume_b200.so"

c_float3 = ctypes.c_float * 3
c_int3 = ctypes.c_int32 * 3


class PlumeGridInfo(ctypes.Structure):
    _fields_ = [("dims", c_int3), ("cell_m", ctypes.c_float), ("origin_m", c_float3), ("open_lo", c_int3),
                ("open_hi", c_int3), ("fill_hi", c_float3), ("ghost_gap", ctypes.c_float)]


class PlumeEmitter(ctypes.Structure):
    _fields_ = [("shape", ctypes.c_int32), ("center_m", c_float3), ("radius_m", ctypes.c_float),
                ("half_size_m", c_float3), ("edge_softness", ctypes.c_float), ("start_s", ctypes.c_float),
                ("end_s", ctypes.c_float), ("smoke_per_s", ctypes.c_float), ("temperature_k", ctypes.c_float),
                ("velocity_mps", c_float3), ("outward", ctypes.c_int32), ("noise_scale_m", ctypes.c_float),
                ("noise_strength", ctypes.c_float), ("stream", ctypes.c_int32)]


class PlumeViewParams(ctypes.Structure):
    _fields_ = [("right", c_float3), ("up", c_float3), ("toward", c_float3), ("left_m", ctypes.c_float),
                ("top_m", ctypes.c_float), ("pixel_m", ctypes.c_float), ("perspective", ctypes.c_int32),
                ("eye", c_float3)]


class PlumeLookParams(ctypes.Structure):
    _fields_ = [("opacity_per_density", ctypes.c_float), ("glow_start_k", ctypes.c_float),
                ("smoke_hides_heat", ctypes.c_float), ("normal_fade_thickness", ctypes.c_float),
                ("shade_layout", ctypes.c_int32), ("shade_fill", ctypes.c_float)]


class PlumeLookInputs(ctypes.Structure):
    _fields_ = [("view", ctypes.c_int32), ("shade_layout", ctypes.c_int32), ("heat_divisor", ctypes.c_float),
                ("shade_divisor", ctypes.c_float), ("shade_depth", ctypes.c_float), ("ambient", ctypes.c_float),
                ("toward_light", c_float3), ("background", c_float3)]


class PlumeField(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("hat", ctypes.c_void_p), ("next", ctypes.c_void_p)]


class PlumeLevel(ctypes.Structure):
    _fields_ = [("info", PlumeGridInfo), ("q", ctypes.c_void_p), ("rhs", ctypes.c_void_p),
                ("residual", ctypes.c_void_p)]


class PlumeStepState(ctypes.Structure):
    _fields_ = [("info", PlumeGridInfo), ("u", PlumeField), ("v", PlumeField), ("w", PlumeField),
                ("smoke", PlumeField), ("temperature", PlumeField), ("pressure", ctypes.c_void_p),
                ("divergence", ctypes.c_void_p), ("curl", ctypes.c_void_p * 3), ("push", ctypes.c_void_p * 3),
                ("sums", ctypes.c_void_p), ("factor", ctypes.c_void_p), ("advect_scratch", ctypes.c_void_p),
                ("levels", ctypes.POINTER(PlumeLevel)),
                ("level_count", ctypes.c_int32), ("storage", ctypes.c_int32)]


# Storage codes of the velocity, smoke and temperature arrays (PLUME_STORAGE_*): float32, bfloat16, float16.
STORAGE = {torch.float32: 0, torch.bfloat16: 1, torch.float16: 2}


def storage_of(tensor: torch.Tensor) -> int:
    if tensor.dtype not in STORAGE:
        raise TypeError(f"fields are stored as float32, bfloat16 or float16, not {tensor.dtype}")
    return STORAGE[tensor.dtype]


class PlumeStepParams(ctypes.Structure):
    _fields_ = [("time_s", ctypes.c_float), ("dt", ctypes.c_float), ("dt_over_cell", ctypes.c_float),
                ("seed", ctypes.c_int32), ("emitters", ctypes.POINTER(PlumeEmitter)),
                ("emitter_count", ctypes.c_int32), ("gravity", ctypes.c_float), ("heat_buoyancy", ctypes.c_float),
                ("smoke_weight", ctypes.c_float), ("ambient_k", ctypes.c_float), ("confinement", ctypes.c_float),
                ("turbulence_scale_m", ctypes.c_float), ("turbulence_strength", ctypes.c_float),
                ("turbulence_pattern_time", ctypes.c_float), ("apply_drag", ctypes.c_int32), ("wind", c_float3),
                ("drag_keep", ctypes.c_float), ("solver", ctypes.c_int32), ("solver_iterations", ctypes.c_int32),
                ("multigrid_sweeps", ctypes.c_int32), ("apply_dissipation", ctypes.c_int32),
                ("smoke_keep", ctypes.c_float), ("heat_keep", ctypes.c_float),
                ("phase_events", ctypes.POINTER(ctypes.c_void_p))]

STEP_PHASES = ("forces", "velocity advection", "divergence", "pressure solve", "gradient", "scalar advection")


_P, _I, _F = ctypes.c_void_p, ctypes.c_int32, ctypes.c_float
_INFO, _SHAPE, _F3P = ctypes.POINTER(PlumeGridInfo), ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_float)
_PP = ctypes.POINTER(ctypes.c_void_p)
_F5P = ctypes.POINTER(ctypes.c_float)

SIGNATURES = {
    "plume_abi_version": [],
    "plume_advect_semi_lagrangian": [_INFO, _SHAPE, _P, _P, _P, _P, _P, _F, _F3P, _F, _I, _P],
    "plume_advect_maccormack": [_INFO, _SHAPE, _P, _P, _P, _P, _P, _P, _F, _F3P, _F, _I, _P],
    "plume_emit": [_INFO, _P, _P, _P, _P, _P, ctypes.POINTER(PlumeEmitter), _I, _I, _F, _F, _P],
    "plume_buoyancy": [_INFO, _P, _P, _P, _F, _F, _F, _F, _F, _P],
    "plume_drag": [_INFO, _P, _P, _P, _F3P, _F, _P],
    "plume_confinement": [_INFO, _P, _P, _P, _PP, _PP, _F, _F, _I, _P],
    "plume_turbulence": [_INFO, _P, _P, _P, _I, _F, _F, _F, _F, _P],
    "plume_project_begin": [_INFO, _P, _P, _P, _P, _P],
    "plume_divergence": [_INFO, _P, _P, _P, _P, _P],
    "plume_subtract_gradient": [_INFO, _P, _P, _P, _P, _P],
    "plume_red_black_sweeps": [_INFO, _P, _P, _P, _I, _F, _P],
    "plume_multigrid": [ctypes.POINTER(PlumeLevel), _I, _I, _I, _P],
    "plume_residual": [_INFO, _P, _P, _P, _P],
    "plume_norm_scratch_doubles": [_INFO],
    "plume_residual_f64": [_INFO, _P, _P, _P, _P, _P, _P, _P],
    "plume_multigrid_correct": [ctypes.POINTER(PlumeLevel), _I, _I, _P, _P, _P],
    "plume_tune_solver": [ctypes.c_longlong, ctypes.c_longlong, _I],
    "plume_solver_tuning": [ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                            ctypes.POINTER(ctypes.c_int32)],
    "plume_use_graphs": [_I],
    "plume_split_scratch_floats": [_INFO],
    "plume_tune_split": [ctypes.c_longlong],
    "plume_split_min_cells": [],
    "plume_multigrid_split": [ctypes.POINTER(PlumeLevel), _I, _I, _I, _P, _P],
    "plume_smoke_scratch_doubles": [_INFO],
    "plume_advect_scratch_floats": [_INFO],
    "plume_smoke_budget": [_INFO, _P, _P, _P, _P, _P, _P, _P],
    "plume_triple_sum": [_SHAPE, _P, _P, _P, _P, _P, _P],
    "plume_use_fused_advection": [_I],
    "plume_maccormack_scratch_floats": [_INFO],
    "plume_maccormack_velocity": [_INFO, _P, _P, _P, _P, _P, _P, _F, _P],
    "plume_maccormack_scalars": [_INFO, _P, _P, _P, _P, _P, _P, _P, _F, _F, _F, _I, _P, _P, _P, _P],
    "plume_smoke_budget_static": [_INFO, _P, _P, _P, _P, _P],
    "plume_dissipate": [_INFO, _P, _P, _F, _F, _F, _P],
    "plume_grid_speed": [_INFO, _P, _P, _P, _I, _P, _P],
    "plume_step": [ctypes.POINTER(PlumeStepState), ctypes.POINTER(PlumeStepParams), _P],
    "plume_brick_floats": [_SHAPE],
    "plume_light_volume": [_SHAPE, _P, _I, _F3P, _F, _F, _P, _P, _P],
    "plume_march_light_volume": [_SHAPE, _P, _I, _F3P, _F, _F, _P, _P, _P],
    "plume_normal_field": [_SHAPE, _P, _I, _P, _P, _P, _F3P, _I, _P],
    "plume_brick_max": [_SHAPE, _P, _I, _P, _P],
    "plume_raymarch": [_INFO, _P, _P, _I, _P, _SHAPE, _P, _SHAPE, ctypes.POINTER(PlumeViewParams),
                       ctypes.POINTER(PlumeLookParams), _P, _I, _I, _P, _P],
    "plume_sheet_content_box": [_P, _I, _I, _I, _P, _P, _P],
    "plume_sheet_resample": [_P, _I, _I, _I, _I, _F5P, _P, _P, _P, _I, _P, _P, _P, _I, _I, _I, _I, _I, _P, _P, _P],
    "plume_sheet_blur": [_P, _P, _P, _I, _I, _I, _I, _I, _P, _I, _P],
    "plume_sheet_renormalize": [_P, _I, _I, _P],
    "plume_sheet_ease": [_P, _P, _P, _I, _I, ctypes.c_double, _P],
    "plume_sheet_channel_max": [_P, _I, _I, _I, ctypes.c_double, _P, _P, _P, _P],
    "plume_sheet_quantize": [_P, _I, _I, ctypes.c_double, ctypes.c_double, _I, _I, _P, _P, _P],
    "plume_sheet_pack": [_P, _I, _I, _I, _P, _P],
    "plume_sheet_measure": [_P, _I, _I, _I, _P, _P],
    "plume_view_look": [_P, _I, _I, _P, _P, _I, _P, _I, ctypes.POINTER(PlumeLookInputs), _P, _P],
    "plume_view_center_depth": [_P, _INFO, _F3P, _F3P, _F, _F, _P, _P],
    "plume_view_center_velocity": [_INFO, _P, _P, _P, _P, _P],
    "plume_view_curl": [_INFO, _P, _P, _P],
    "plume_view_speed": [_P, ctypes.c_longlong, _P, _P],
    "plume_view_slice": [ctypes.POINTER(PlumeViewParams), _INFO, _I, _F, _P, _F, _F, _P, _I, _P, _I, _I, _P],
    "plume_view_boundary_layers": [_P, _SHAPE, _P, _P],
    "plume_view_narrow": [_P, _P, ctypes.c_longlong, _P],
    "plume_view_widen": [_P, _P, ctypes.c_longlong, _P],
    "plume_add_source": [_P, _SHAPE, _P, _SHAPE, _SHAPE, _F, _P],
    "plume_source_grad": [_P, _SHAPE, _P, _SHAPE, _SHAPE, _F, _P],
    "plume_smoke_adjoint": [_INFO, _P, _P, _P, _P, _P, _P, _P, _F, _F, _P, _P, _P, _P, _P, _P, _P],
    "plume_thickness_adjoint": [_INFO, ctypes.POINTER(PlumeViewParams), _F, _P, _P, _I, _I, _P, _P, _P, _P],
    "plume_budget_adjoint": [_INFO, _P, _P, _F, _P, _P, _P, _P, _P, _P, _P],
    "plume_maccormack_adjoint": [_INFO, _SHAPE, _F3P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _F, _F, _I, _P],
    "plume_buoyancy_adjoint": [_INFO, _P, _P, _P, _P, _P, _F, _F, _F, _F, _F, _P, _P],
    "plume_drag_adjoint": [_INFO, _P, _P, _P, _P, _P, _P, _F3P, _F, _F, _P, _P],
    "plume_emit_adjoint": [_INFO, _P, _P, _P, _P, ctypes.POINTER(PlumeEmitter), _I, _I, _F, _F, _P],
    "plume_confinement_adjoint": [_INFO, _P, _P, _P, _P, _P, _P, _F, _F, _P, _P, _P],
    "plume_confinement_adjoint_scratch_floats": [_INFO],
}

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded library; raises when it is not built (there is no CPU path)."""
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise RuntimeError(f"{LIBRARY.name} is not built: run `python -m plume_b200.build` (nvcc, sm_100a)")
        loaded = ctypes.CDLL(str(LIBRARY))
        loaded.plume_last_error.restype = ctypes.c_char_p
        loaded.plume_last_error.argtypes = []
        loaded.plume_launch_count.restype = ctypes.c_ulonglong
        loaded.plume_launch_count.argtypes = []
        for name, argtypes in SIGNATURES.items():
            fn = getattr(loaded, name)
            fn.argtypes = argtypes
            wide = name in ("plume_advect_scratch_floats", "plume_brick_floats", "plume_norm_scratch_doubles",
                            "plume_maccormack_scratch_floats", "plume_split_scratch_floats",
                            "plume_split_min_cells", "plume_confinement_adjoint_scratch_floats")
            fn.restype = ctypes.c_longlong if wide else ctypes.c_int
        _lib = loaded
    return _lib


def check(status: int) -> None:
    if status != 0:
        raise RuntimeError(f"libplume_b200: {lib().plume_last_error().decode()} (status {status})")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))


def stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def field_ptr(tensor: torch.Tensor) -> ctypes.c_void_p:
    """The device address of a field array stored as float32, bfloat16 or float16."""
    storage_of(tensor)
    return ptr(tensor, tensor.dtype)


def ptr(tensor: torch.Tensor, dtype=torch.float32) -> ctypes.c_void_p:
    """The device address of a contiguous CUDA tensor of `dtype` (float32 fields by default)."""
    if not tensor.is_cuda:
        raise RuntimeError("plume_b200 kernels need CUDA tensors; there is no CPU path")
    if tensor.dtype != dtype:
        raise TypeError(f"expected a {dtype} tensor, got {tensor.dtype}")
    if not tensor.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return ctypes.c_void_p(tensor.data_ptr())


def shape3(tensor: torch.Tensor):
    return c_int3(*tensor.shape[:3])


def f3(values) -> ctypes.Array:
    return c_float3(*[float(v) for v in values])


EXPORTED = ("plume_last_error", "plume_launch_count", *SIGNATURES)


def launch_count() -> int:
    return int(lib().plume_launch_count())


def ptrs(*tensors) -> ctypes.Array:
    """A C array of device pointers (for the `float* xyz[3]` arguments)."""
    return (ctypes.c_void_p * len(tensors))(*[ptr(t).value for t in tensors])
