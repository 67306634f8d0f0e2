"""ctypes binding of ``libglazier_gpu.so`` (the C ABI in include/glazier_gpu.h).

The library is built ahead of time by ``glazier_b200.build``; loading it
never compiles anything. If it is missing the import fails loudly: there is
no CPU fallback for the device engine.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libglazier_gpu.so"

GLZ_OK, GLZ_ODD_LATTICE, GLZ_DRIVER, GLZ_UNSUPPORTED, GLZ_INVALID = 0, 1, 2, 3, 4

_P = C.c_void_p
_D = C.POINTER(C.c_double)


class GlzModel(C.Structure):
    """``glz_model`` (include/glazier_gpu.h)."""

    _fields_ = [
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("depth", C.c_int32),
        ("neighbour_order", C.c_int32),
        ("n_types", C.c_int32),
        ("n_species", C.c_int32),
        ("temperature", C.c_double),
        ("seed", C.c_uint64),
        ("contact", _D),
        ("target_volume", _D),
        ("lambda_volume", _D),
        ("target_surface", _D),
        ("lambda_surface", _D),
        ("division_volume", _D),
        ("death_rate", _D),
        ("target_length", _D),
        ("lambda_length", _D),
        ("connected", C.POINTER(C.c_uint8)),
        ("max_activity", _D),
        ("lambda_activity", _D),
        ("external", _D),
        ("lambda_nematic", _D),
        ("diffusion", _D),
        ("decay", _D),
        ("initial", _D),
        ("secretion", _D),
        ("uptake", _D),
        ("chemotaxis", _D),
        ("nematic", _D),
    ]


def model_struct(model, keep: list) -> GlzModel:
    """Flatten a ``blueprint.Model`` into a ``glz_model``; the arrays it points
    at are appended to ``keep``, which must outlive every call that reads it."""

    def arr(values, dtype=np.float64):
        a = np.ascontiguousarray(np.asarray(values, dtype=dtype))
        keep.append(a)
        return a

    def dptr(values):
        return arr(values).ctypes.data_as(_D)

    ns = len(model.species)
    m = GlzModel()
    m.width, m.height, m.depth = model.width, model.height, model.depth
    m.neighbour_order = model.neighbour_order
    m.n_types, m.n_species = model.n_types, ns
    m.temperature = model.temperature
    m.seed = model.seed & 0xFFFFFFFFFFFFFFFF
    m.contact = dptr(model.contact)
    for name in ("target_volume", "lambda_volume", "target_surface", "lambda_surface", "division_volume",
                 "death_rate", "target_length", "lambda_length", "max_activity", "lambda_activity",
                 "lambda_nematic"):
        setattr(m, name, dptr(model.per_type(name)))
    m.connected = arr([int(t.connected) for t in model.types], np.uint8).ctypes.data_as(C.POINTER(C.c_uint8))
    m.external = dptr([v for t in model.types for v in t.external])
    m.diffusion = dptr([s.diffusion for s in model.species] or [0.0])
    m.decay = dptr([s.decay for s in model.species] or [0.0])
    m.initial = dptr([s.initial for s in model.species] or [0.0])
    m.secretion = dptr(model.table(model.secretion).reshape(-1) if ns else [0.0])
    m.uptake = dptr(model.table(model.uptake).reshape(-1) if ns else [0.0])
    m.chemotaxis = dptr(model.table(model.chemotaxis).reshape(-1) if ns else [0.0])
    m.nematic = dptr(np.asarray(model.nematic).reshape(-1)) if model.nematic is not None else None
    return m


_lib = None


def lib():
    """The loaded library, with every entry point's signature declared."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is not built; run `python -m glazier_b200.build` (the device engine has no CPU fallback)"
        )
    L = C.CDLL(str(LIB_PATH))
    L.glz_last_error.restype = C.c_char_p
    L.glz_last_error.argtypes = []
    L.glz_gpu_create.restype = C.c_int
    L.glz_gpu_create.argtypes = [C.POINTER(GlzModel), _P, _P, C.c_size_t, _P, _P, C.POINTER(_P)]
    L.glz_gpu_step.restype = C.c_int
    L.glz_gpu_step.argtypes = [_P, C.c_uint64]
    L.glz_gpu_labels.restype = C.c_int
    L.glz_gpu_labels.argtypes = [_P, _P, C.c_size_t]
    L.glz_gpu_field.restype = C.c_int
    L.glz_gpu_field.argtypes = [_P, C.c_int, _P, C.c_size_t]
    for name in ("glz_gpu_volumes", "glz_gpu_surfaces", "glz_gpu_cell_types"):
        getattr(L, name).restype = C.c_int
        getattr(L, name).argtypes = [_P, _P, C.POINTER(C.c_size_t)]
    L.glz_gpu_set_infection.restype = C.c_int
    L.glz_gpu_set_infection.argtypes = [_P, C.c_int, C.c_int, C.c_int, C.c_double]
    L.glz_gpu_set_nematic_field.restype = C.c_int
    L.glz_gpu_set_nematic_field.argtypes = [_P, _P, C.c_size_t]
    L.glz_gpu_mcs.restype = C.c_uint64
    L.glz_gpu_mcs.argtypes = [_P]
    L.glz_gpu_n_labels.restype = C.c_size_t
    L.glz_gpu_n_labels.argtypes = [_P]
    L.glz_gpu_sweep_kernel.restype = C.c_char_p
    L.glz_gpu_sweep_kernel.argtypes = [_P]
    L.glz_gpu_stream.restype = _P
    L.glz_gpu_stream.argtypes = [_P]
    L.glz_gpu_device_labels.restype = C.c_int
    L.glz_gpu_device_labels.argtypes = [_P, C.POINTER(_P)]
    L.glz_gpu_device_field.restype = C.c_int
    L.glz_gpu_device_field.argtypes = [_P, C.c_int, C.POINTER(_P)]
    L.glz_set_device.restype = C.c_int
    L.glz_set_device.argtypes = [C.c_int]
    L.glz_gpu_set_labels.restype = C.c_int
    L.glz_gpu_set_labels.argtypes = [_P, _P, C.c_size_t]
    L.glz_gpu_set_labels_device.restype = C.c_int
    L.glz_gpu_set_labels_device.argtypes = [_P, _P, C.c_size_t]
    L.glz_gpu_set_nematic_field_device.restype = C.c_int
    L.glz_gpu_set_nematic_field_device.argtypes = [_P, _P, C.c_size_t]
    L.glz_gpu_step_profiled.restype = C.c_int
    L.glz_gpu_step_profiled.argtypes = [_P, C.c_uint64, C.POINTER(C.c_double)]
    L.glz_field_step_noalloc.restype = C.c_int
    L.glz_field_step_noalloc.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _P, _P,
                                         C.c_size_t, _P, _P, _P]
    L.glz_gpu_destroy.restype = None
    L.glz_gpu_destroy.argtypes = [_P]
    _declare_extras(L)
    _lib = L
    return L


def _declare_extras(L) -> None:
    """Signatures of the batched ensemble's entry points."""
    L.glz_ens_create.restype = C.c_int
    L.glz_ens_create.argtypes = [C.c_int, C.POINTER(GlzModel), C.POINTER(_P), C.POINTER(_P), C.POINTER(C.c_size_t),
                                 C.POINTER(_P)]
    L.glz_ens_n_labels.restype = C.c_size_t
    L.glz_ens_n_labels.argtypes = [_P, C.c_int]
    L.glz_ens_set_infection.restype = C.c_int
    L.glz_ens_set_infection.argtypes = [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double]
    L.glz_ens_step.restype = C.c_int
    L.glz_ens_step.argtypes = [_P, C.c_uint64]
    L.glz_ens_step_timed.restype = C.c_int
    L.glz_ens_step_timed.argtypes = [_P, C.c_uint64, C.POINTER(C.c_double)]
    L.glz_ens_autotune.restype = C.c_int
    L.glz_ens_autotune.argtypes = [_P, C.c_uint64, C.POINTER(C.c_int)]
    L.glz_ens_set_schedule.restype = C.c_int
    L.glz_ens_set_schedule.argtypes = [_P, C.c_int, C.c_int]
    L.glz_ens_labels.restype = C.c_int
    L.glz_ens_labels.argtypes = [_P, C.c_int, _P, C.c_size_t]
    L.glz_ens_volumes.restype = C.c_int
    L.glz_ens_volumes.argtypes = [_P, C.c_int, _P, C.POINTER(C.c_size_t)]
    L.glz_ens_surfaces.restype = C.c_int
    L.glz_ens_surfaces.argtypes = [_P, C.c_int, _P, C.POINTER(C.c_size_t)]
    L.glz_ens_mcs.restype = C.c_uint64
    L.glz_ens_mcs.argtypes = [_P]
    L.glz_ens_stream.restype = _P
    L.glz_ens_stream.argtypes = [_P]
    L.glz_ens_destroy.restype = None
    L.glz_ens_destroy.argtypes = [_P]
    L.glz_adj_create.restype = C.c_int
    L.glz_adj_create.argtypes = [C.c_int] * 7 + [C.POINTER(_P)]
    L.glz_adj_set_trajectory.restype = C.c_int
    L.glz_adj_set_trajectory.argtypes = [_P, _P]
    L.glz_adj_forward.restype = C.c_int
    L.glz_adj_forward.argtypes = [_P, _P, _P, _P]
    L.glz_adj_backward.restype = C.c_int
    L.glz_adj_backward.argtypes = [_P, _P, _P, _P]
    L.glz_adj_stream.restype = C.c_void_p
    L.glz_adj_stream.argtypes = [_P]
    L.glz_adj_destroy.restype = None
    L.glz_adj_destroy.argtypes = [_P]


def last_error() -> str:
    return lib().glz_last_error().decode(errors="replace")


def ptr(a: np.ndarray):
    return a.ctypes.data_as(_P)
