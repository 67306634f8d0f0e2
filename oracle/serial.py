"""ORACLE — test infrastructure, not the product.

ctypes wrapper over ``serial.c``, the reference's serial f64 engine
(glazier-core/src/cpu.rs) restated in C. Used by the tests as the
distributional reference for the device engine and by the benchmark as the
timed CPU baseline.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import build as _build

_lib = None


class OrcModel(C.Structure):
    _fields_ = [
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("depth", C.c_int32),
        ("neighbour_order", C.c_int32),
        ("n_types", C.c_int32),
        ("n_species", C.c_int32),
        ("temperature", C.c_double),
        ("seed", C.c_uint64),
        ("contact", C.POINTER(C.c_double)),
        ("target_volume", C.POINTER(C.c_double)),
        ("lambda_volume", C.POINTER(C.c_double)),
        ("target_surface", C.POINTER(C.c_double)),
        ("lambda_surface", C.POINTER(C.c_double)),
        ("division_volume", C.POINTER(C.c_double)),
        ("death_rate", C.POINTER(C.c_double)),
        ("target_length", C.POINTER(C.c_double)),
        ("lambda_length", C.POINTER(C.c_double)),
        ("connected", C.POINTER(C.c_uint8)),
        ("max_activity", C.POINTER(C.c_double)),
        ("lambda_activity", C.POINTER(C.c_double)),
        ("external", C.POINTER(C.c_double)),
        ("lambda_nematic", C.POINTER(C.c_double)),
        ("diffusion", C.POINTER(C.c_double)),
        ("decay", C.POINTER(C.c_double)),
        ("initial", C.POINTER(C.c_double)),
        ("secretion", C.POINTER(C.c_double)),
        ("uptake", C.POINTER(C.c_double)),
        ("chemotaxis", C.POINTER(C.c_double)),
        ("nematic", C.POINTER(C.c_double)),
    ]


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = C.CDLL(str(path))
        P = C.c_void_p
        L.orc_create.restype = P
        L.orc_create.argtypes = [C.POINTER(OrcModel), P, C.c_long, C.c_long, C.c_long, C.c_long]
        L.orc_destroy.argtypes = [P]
        L.orc_last_error.restype = C.c_char_p
        L.orc_set_cell_types.argtypes = [P, P, C.c_size_t]
        L.orc_step.argtypes = [P, C.c_uint64]
        L.orc_attempts.argtypes = [P, C.c_uint64]
        L.orc_attempt.argtypes = [P]
        L.orc_attempt.restype = C.c_int
        L.orc_delta_energy.argtypes = [P, C.c_long, C.c_uint32]
        L.orc_delta_energy.restype = C.c_double
        L.orc_energy.argtypes = [P]
        L.orc_energy.restype = C.c_double
        L.orc_sites.argtypes = [P]
        L.orc_sites.restype = C.c_long
        L.orc_n_labels.argtypes = [P]
        L.orc_n_labels.restype = C.c_size_t
        for name in ("orc_mcs", "orc_accepted", "orc_attempted"):
            getattr(L, name).argtypes = [P]
            getattr(L, name).restype = C.c_uint64
        for name in ("orc_labels", "orc_volumes", "orc_surfaces", "orc_cell_types", "orc_lengths",
                     "orc_recounted_surfaces", "orc_set_labels"):
            getattr(L, name).argtypes = [P, P]
        L.orc_field.argtypes = [P, C.c_int, P]
        L.orc_set_field.argtypes = [P, C.c_int, P]
        L.orc_divide_and_die.argtypes = [P, P, P]
        L.orc_substeps_for.argtypes = [C.c_double, C.c_int]
        L.orc_substeps_for.restype = C.c_int
        L.orc_xoshiro_stream.argtypes = [C.c_uint64, C.c_size_t, P]
        L.orc_xoshiro_below.argtypes = [C.c_uint64, C.c_uint64, C.c_size_t, P]
        L.orc_moments_of.argtypes = [P, C.c_size_t, P, P, P]
        L.orc_unwrap_about.argtypes = [P, P, P, P]
        L.orc_offsets.argtypes = [C.c_int, C.c_int, P]
        L.orc_offsets.restype = C.c_int
        L.orc_locally_connected.argtypes = [P, C.c_long, C.c_long, C.c_long, C.c_long, C.c_uint32]
        L.orc_locally_connected.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def model_struct(model, keep: list) -> OrcModel:
    """Flatten a ``glazier_b200.blueprint.Model`` into the C model record
    (the same layout as ``glz_model``); arrays are kept alive in ``keep``."""
    nt, ns = model.n_types, len(model.species)

    def arr(values, dtype=np.float64):
        a = np.ascontiguousarray(np.asarray(values, dtype=dtype))
        keep.append(a)
        return a

    m = OrcModel()
    m.width, m.height, m.depth = model.width, model.height, model.depth
    m.neighbour_order = model.neighbour_order
    m.n_types, m.n_species = nt, ns
    m.temperature = model.temperature
    m.seed = model.seed & 0xFFFFFFFFFFFFFFFF
    m.contact = _dptr(arr(model.contact))
    for name in ("target_volume", "lambda_volume", "target_surface", "lambda_surface", "division_volume",
                 "death_rate", "target_length", "lambda_length", "max_activity", "lambda_activity",
                 "lambda_nematic"):
        setattr(m, name, _dptr(arr(model.per_type(name))))
    m.connected = arr([int(t.connected) for t in model.types], np.uint8).ctypes.data_as(C.POINTER(C.c_uint8))
    m.external = _dptr(arr([v for t in model.types for v in t.external]))
    m.diffusion = _dptr(arr([s.diffusion for s in model.species] or [0.0]))
    m.decay = _dptr(arr([s.decay for s in model.species] or [0.0]))
    m.initial = _dptr(arr([s.initial for s in model.species] or [0.0]))
    m.secretion = _dptr(arr(model.table(model.secretion).reshape(-1) if ns else [0.0]))
    m.uptake = _dptr(arr(model.table(model.uptake).reshape(-1) if ns else [0.0]))
    m.chemotaxis = _dptr(arr(model.table(model.chemotaxis).reshape(-1) if ns else [0.0]))
    m.nematic = _dptr(arr(np.asarray(model.nematic).reshape(-1))) if model.nematic is not None else None
    return m


class SerialOracle:
    """One serial run (cpu.rs ``Simulation``), seeded from a model and a start.

    ``model`` is a ``glazier_b200.blueprint.Model``; ``labels`` (uint32 per
    site) and ``cell_type`` (uint8 per label) give the start, or ``tile`` =
    (side, nx, ny, nz) lays squares down the way ``Simulation::tiled_grid``
    does.
    """

    def __init__(self, model, labels=None, cell_type=None, tile=None):
        L = lib()
        self._keep = []
        m = model_struct(model, self._keep)
        self._model_struct = m
        if labels is not None:
            lab = np.ascontiguousarray(labels, dtype=np.uint32)
            self._keep.append(lab)
            h = L.orc_create(C.byref(m), _ptr(lab), 0, 0, 0, 0)
        else:
            side, nx, ny, nz = tile
            h = L.orc_create(C.byref(m), None, side, nx, ny, nz)
        if not h:
            raise ValueError(L.orc_last_error().decode())
        self.h = h
        self.model = model
        self.sites = model.sites
        if cell_type is not None:
            ct = np.ascontiguousarray(np.asarray(cell_type, dtype=np.uint8)[1:])
            L.orc_set_cell_types(self.h, _ptr(ct), len(ct))

    @classmethod
    def from_start(cls, start):
        return cls(start.model, labels=start.labels, cell_type=start.cell_type)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_destroy(self.h)
            self.h = None

    def step(self, steps: int = 1) -> None:
        lib().orc_step(self.h, steps)

    def attempts(self, n: int) -> None:
        lib().orc_attempts(self.h, n)

    def attempt(self) -> bool:
        return bool(lib().orc_attempt(self.h))

    def delta_energy(self, target: int, new: int) -> float:
        return lib().orc_delta_energy(self.h, target, new)

    def energy(self) -> float:
        return lib().orc_energy(self.h)

    @property
    def n_labels(self) -> int:
        return lib().orc_n_labels(self.h)

    @property
    def mcs(self) -> int:
        return lib().orc_mcs(self.h)

    @property
    def accepted(self) -> int:
        return lib().orc_accepted(self.h)

    def labels(self) -> np.ndarray:
        out = np.empty(self.sites, dtype=np.uint32)
        lib().orc_labels(self.h, _ptr(out))
        return out

    def volumes(self) -> np.ndarray:
        out = np.empty(self.n_labels, dtype=np.uint32)
        lib().orc_volumes(self.h, _ptr(out))
        return out

    def surfaces(self) -> np.ndarray:
        out = np.empty(self.n_labels, dtype=np.int64)
        lib().orc_surfaces(self.h, _ptr(out))
        return out

    def recounted_surfaces(self) -> np.ndarray:
        out = np.empty(self.n_labels, dtype=np.int64)
        lib().orc_recounted_surfaces(self.h, _ptr(out))
        return out

    def cell_types(self) -> np.ndarray:
        out = np.empty(self.n_labels, dtype=np.uint8)
        lib().orc_cell_types(self.h, _ptr(out))
        return out

    def lengths(self) -> np.ndarray:
        out = np.empty(self.n_labels, dtype=np.float64)
        lib().orc_lengths(self.h, _ptr(out))
        return out

    def field(self, k: int) -> np.ndarray:
        out = np.empty(self.sites, dtype=np.float64)
        lib().orc_field(self.h, k, _ptr(out))
        return out

    def set_field(self, k: int, values) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        lib().orc_set_field(self.h, k, _ptr(v))

    def set_labels(self, labels) -> None:
        v = np.ascontiguousarray(labels, dtype=np.uint32)
        lib().orc_set_labels(self.h, _ptr(v))

    def divide_and_die(self):
        a, b = C.c_int(0), C.c_int(0)
        lib().orc_divide_and_die(self.h, C.byref(a), C.byref(b))
        return a.value, b.value


def xoshiro_stream(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint64)
    lib().orc_xoshiro_stream(seed, n, _ptr(out))
    return out


def xoshiro_below(seed: int, bound: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint64)
    lib().orc_xoshiro_below(seed, bound, n, _ptr(out))
    return out


def moments_of(sites) -> tuple:
    s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
    length = C.c_double(0)
    aniso = np.zeros(2)
    axis = np.zeros(3)
    lib().orc_moments_of(_ptr(s), len(s), C.byref(length), _ptr(aniso), _ptr(axis))
    return length.value, (aniso[0], aniso[1]), tuple(axis)


def unwrap_about(anchor, site, extent) -> tuple:
    a = np.asarray(anchor, dtype=np.float64)
    s = np.asarray(site, dtype=np.float64)
    e = np.asarray(extent, dtype=np.float64)
    out = np.zeros(3)
    lib().orc_unwrap_about(_ptr(a), _ptr(s), _ptr(e), _ptr(out))
    return tuple(out)


def offsets(order: int, depth: int) -> list:
    out = np.zeros(26 * 3, dtype=np.int32)
    n = lib().orc_offsets(order, depth, _ptr(out))
    return [tuple(int(v) for v in out[3 * k: 3 * k + 3]) for k in range(n)]


def locally_connected(labels, w, h, d, target, label) -> bool:
    lab = np.ascontiguousarray(labels, dtype=np.uint32)
    return bool(lib().orc_locally_connected(_ptr(lab), w, h, d, target, label))


def substeps_for(diffusion: float, dimensions: int) -> int:
    return lib().orc_substeps_for(diffusion, dimensions)
