"""ORACLE — test infrastructure, not the product.

ctypes wrapper over ``replay.c``: a serial host replay of the device
engine's schedule (colour order, counter hash, per-pass snapshots, f32/f64
operation order). The device must reproduce it bit for bit: labels,
volumes, surfaces, per-colour volumes, exact moment sums and fields.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from .serial import OrcModel, _ptr, lib as _serial_lib, model_struct

_rlib = None


def lib():
    global _rlib
    if _rlib is None:
        L = _serial_lib()  # one library holds both restatements
        P = C.c_void_p
        L.rp_create.restype = P
        L.rp_create.argtypes = [C.POINTER(OrcModel), P, P, C.c_size_t, P]
        L.rp_destroy.argtypes = [P]
        L.rp_last_error.restype = C.c_char_p
        L.rp_step.argtypes = [P, C.c_uint64]
        L.rp_n_labels.argtypes = [P]
        L.rp_n_labels.restype = C.c_size_t
        L.rp_mcs.argtypes = [P]
        L.rp_mcs.restype = C.c_uint64
        L.rp_accepted.argtypes = [P]
        L.rp_accepted.restype = C.c_uint64
        for name in ("rp_labels", "rp_cell_types", "rp_volumes", "rp_surfaces", "rp_volumes_by_colour",
                     "rp_moments", "rp_lengths"):
            getattr(L, name).argtypes = [P, P]
        L.rp_field.argtypes = [P, C.c_int, P]
        L.rp_set_nematic_field.argtypes = [P, P]
        L.rp_set_nematic_field.restype = C.c_int
        L.rp_set_infection.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_double]
        L.rp_set_infection.restype = C.c_int
        L.rp_expf.argtypes = [C.c_float]
        L.rp_expf.restype = C.c_float
        L.rp_draw.argtypes = [C.c_uint64, C.c_uint32, C.c_int32, C.c_int, C.c_int]
        L.rp_draw.restype = C.c_uint64
        L.rp_to_f32.argtypes = [C.c_uint64]
        L.rp_to_f32.restype = C.c_float
        _rlib = L
    return _rlib


class ReplayOracle:
    """A host replay of one device run from the same start."""

    def __init__(self, model, labels, cell_type, fields=None):
        L = lib()
        self._keep: list = []
        m = model_struct(model, self._keep)
        lab = np.ascontiguousarray(labels, dtype=np.uint32).reshape(-1)
        ct = np.ascontiguousarray(cell_type, dtype=np.uint8).reshape(-1)
        fl = None if fields is None else np.ascontiguousarray(fields, dtype=np.float64).reshape(-1)
        self._keep += [lab, ct] + ([fl] if fl is not None else [])
        h = L.rp_create(C.byref(m), _ptr(lab), _ptr(ct), ct.size, _ptr(fl) if fl is not None else None)
        if not h:
            raise ValueError(L.rp_last_error().decode())
        self.h = h
        self.model = model
        self.sites = model.sites
        self.ncol = 8 if model.depth > 1 else 4
        self.nm = 9 if model.depth > 1 else 5

    @classmethod
    def from_start(cls, start, fields=None):
        return cls(start.model, start.labels, start.cell_type, fields)

    def __del__(self):
        if getattr(self, "h", None) and _rlib is not None:
            _rlib.rp_destroy(self.h)
            self.h = None

    def step(self, steps: int = 1) -> None:
        lib().rp_step(self.h, steps)

    def set_nematic_field(self, pairs) -> None:
        """Replace the nematic field, (Q_xx, Q_xy) per site."""
        flat = np.ascontiguousarray(pairs, dtype=np.float64).reshape(-1)
        if flat.size != 2 * self.sites:
            raise ValueError("the nematic field is not two values per site")
        self._keep.append(flat)
        if lib().rp_set_nematic_field(self.h, _ptr(flat)):
            raise ValueError("the model has no nematic coupling to update")

    def set_infection(self, species: int, from_type: int, to_type: int, threshold: float) -> None:
        """The infection rule of glz_gpu_set_infection, same arguments."""
        if lib().rp_set_infection(self.h, species, from_type, to_type, float(threshold)):
            raise ValueError("bad infection rule")

    @property
    def n_labels(self) -> int:
        return lib().rp_n_labels(self.h)

    @property
    def mcs(self) -> int:
        return lib().rp_mcs(self.h)

    @property
    def accepted(self) -> int:
        return lib().rp_accepted(self.h)

    def _get(self, name, n, dtype):
        out = np.empty(n, dtype=dtype)
        getattr(lib(), name)(self.h, _ptr(out))
        return out

    def labels(self):
        return self._get("rp_labels", self.sites, np.uint32)

    def cell_types(self):
        return self._get("rp_cell_types", self.n_labels, np.uint8)

    def volumes(self):
        return self._get("rp_volumes", self.n_labels, np.uint32)

    def surfaces(self):
        return self._get("rp_surfaces", self.n_labels, np.int64)

    def volumes_by_colour(self):
        return self._get("rp_volumes_by_colour", self.n_labels * self.ncol, np.int32).reshape(-1, self.ncol)

    def moments(self):
        return self._get("rp_moments", self.n_labels * self.nm, np.int64).reshape(-1, self.nm)

    def lengths(self):
        return self._get("rp_lengths", self.n_labels, np.float64)

    def field(self, k: int):
        out = np.empty(self.sites, dtype=np.float32)
        lib().rp_field(self.h, k, _ptr(out))
        return out


def expf(x: float) -> float:
    return lib().rp_expf(x)


def draw(seed: int, site: int, step: int, colour: int, index: int) -> int:
    return lib().rp_draw(seed, site, step, colour, index)
