"""``GpuSimulation``: a run kept on the B200, over the C ABI.

The Python face of include/glazier_gpu.h, shaped like the reference's
``glazier_cuda::GpuSimulation`` (glazier-cuda/src/lib.rs:748-1271): build
from a start (``from_start``, the ``from_cpu`` of lib.rs:814), ``step``,
and copy ``labels``, ``field``, ``volumes`` and ``surfaces`` back.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import GLZ_DRIVER, GLZ_INVALID, GLZ_ODD_LATTICE, GLZ_UNSUPPORTED, ptr


class GpuError(ValueError):
    """A refused or failed device call (``GpuError``, lib.rs:723-746); a
    ``ValueError`` as glazier-py raises it (glazier-py/src/lib.rs:13-15)."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


_NAMES = {GLZ_ODD_LATTICE: "odd lattice", GLZ_DRIVER: "driver", GLZ_UNSUPPORTED: "unsupported", GLZ_INVALID: "invalid"}


def check(rc: int) -> None:
    if rc != 0:
        raise GpuError(rc, _lib.last_error())


class _DeviceArray:
    """A bare ``__cuda_array_interface__`` over device memory the engine owns,
    for ``torch.as_tensor`` to wrap without a copy (on the memory's own
    device). Every call that writes it has synchronized its stream before
    returning, so readers need no stream to wait on."""

    def __init__(self, address: int, shape: tuple, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(address), False),
                                         "version": 3, "strides": None, "stream": None}


def _view(address: int, shape: tuple, typestr: str, owner):
    import torch

    t = torch.as_tensor(_DeviceArray(address, shape, typestr))
    t._glazier_owner = owner  # the engine outlives the view while the view is referenced
    return t


def _device_input(tensor, dtypes: tuple, count: int, what: str):
    """A contiguous device tensor of `count` elements of one of `dtypes`, with
    the engine's stream ordered after the work that produced it."""
    import torch

    if not isinstance(tensor, torch.Tensor) or not tensor.is_cuda:
        raise GpuError(GLZ_INVALID, f"the {what} is not a CUDA tensor")
    if tensor.dtype not in dtypes:
        raise GpuError(GLZ_INVALID, f"the {what} is {tensor.dtype}, not one of {dtypes}")
    if tensor.numel() != count:
        raise GpuError(GLZ_INVALID, f"the {what} has {tensor.numel()} values, not {count}")
    return tensor.contiguous()


class GpuSimulation:
    """One run on the device.

    ``model`` is a ``glazier_b200.blueprint.Model``; ``labels`` holds one
    uint32 per site (x fastest, 0 the medium) and ``cell_type`` one uint8 per
    label; ``fields`` is None (every species starts at its ``initial``) or an
    (n_species, sites) array.
    """

    def __init__(self, model, labels, cell_type, fields=None, device: int | None = None):
        L = _lib.lib()
        if device is not None:
            check(L.glz_set_device(int(device)))
        self._keep: list = []
        m = _lib.model_struct(model, self._keep)
        lab = np.ascontiguousarray(labels, dtype=np.uint32).reshape(-1)
        ct = np.ascontiguousarray(cell_type, dtype=np.uint8).reshape(-1)
        fl = None
        if fields is not None:
            fl = np.ascontiguousarray(fields, dtype=np.float64).reshape(-1)
            if fl.size != len(model.species) * lab.size:
                raise GpuError(GLZ_INVALID, f"fields hold {fl.size} values for {len(model.species)} species")
        if lab.size != model.sites:
            raise GpuError(GLZ_INVALID, f"the label field has {lab.size} sites for a lattice of {model.sites}")
        h = C.c_void_p()
        check(L.glz_gpu_create(C.byref(m), ptr(lab), ptr(ct), ct.size, ptr(fl) if fl is not None else None, None,
                               C.byref(h)))
        self._h = h
        self.model = model
        self.sites = model.sites
        self.shape = (model.depth, model.height, model.width)

    @classmethod
    def from_start(cls, start, fields=None, device: int | None = None) -> "GpuSimulation":
        return cls(start.model, start.labels, start.cell_type, fields, device)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().glz_gpu_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def step(self, steps: int = 1) -> None:
        """``GpuSimulation::step`` (lib.rs:1055): run and wait."""
        check(_lib.lib().glz_gpu_step(self._h, int(steps)))

    def step_profiled(self, steps: int = 1) -> tuple:
        """Run like ``step`` and return the device milliseconds of the colour
        sweeps, the field step, and division and death."""
        ms = (C.c_double * 3)()
        check(_lib.lib().glz_gpu_step_profiled(self._h, int(steps), ms))
        return ms[0], ms[1], ms[2]

    def set_labels(self, labels) -> None:
        """Restart from a lattice: upload it and recount every tally."""
        lab = np.ascontiguousarray(labels, dtype=np.uint32).reshape(-1)
        check(_lib.lib().glz_gpu_set_labels(self._h, ptr(lab), lab.size))

    def set_labels_from(self, address: int, sites: int) -> None:
        """``set_labels`` from a raw host address (e.g. pinned memory)."""
        check(_lib.lib().glz_gpu_set_labels(self._h, C.c_void_p(address), int(sites)))

    def labels_to(self, address: int, sites: int) -> None:
        """Copy the lattice to a raw host address (e.g. pinned memory)."""
        check(_lib.lib().glz_gpu_labels(self._h, C.c_void_p(address), int(sites)))

    @property
    def mcs(self) -> int:
        return int(_lib.lib().glz_gpu_mcs(self._h))

    @property
    def n_labels(self) -> int:
        return int(_lib.lib().glz_gpu_n_labels(self._h))

    @property
    def sweep_kernel(self) -> str:
        """The sweep kernel the next step takes ("band", "lean", "direct",
        "compact", "resident", "cluster" or "general")."""
        return _lib.lib().glz_gpu_sweep_kernel(self._h).decode()

    def labels(self) -> np.ndarray:
        out = np.empty(self.sites, dtype=np.uint32)
        check(_lib.lib().glz_gpu_labels(self._h, ptr(out), out.size))
        return out

    def labels_into(self, out: np.ndarray) -> np.ndarray:
        """Copy the lattice into a caller's buffer (pinned host memory works)."""
        check(_lib.lib().glz_gpu_labels(self._h, ptr(out), out.size))
        return out

    def field(self, index: int) -> np.ndarray:
        out = np.empty(self.sites, dtype=np.float64)
        check(_lib.lib().glz_gpu_field(self._h, int(index), ptr(out), out.size))
        return out

    def _per_label(self, name: str, dtype) -> np.ndarray:
        n = C.c_size_t(self.n_labels)
        out = np.empty(n.value, dtype=dtype)
        check(getattr(_lib.lib(), name)(self._h, ptr(out), C.byref(n)))
        return out[: n.value]

    def volumes(self) -> np.ndarray:
        return self._per_label("glz_gpu_volumes", np.uint32)

    def surfaces(self) -> np.ndarray:
        return self._per_label("glz_gpu_surfaces", np.int64)

    def cell_types(self) -> np.ndarray:
        return self._per_label("glz_gpu_cell_types", np.uint8)

    def set_infection(self, species: int, from_type: int, to_type: int, threshold: float) -> None:
        """The infection rule (an extension; glazier has none): after each
        step's field update, a cell of type `from_type` whose summed uptake
        of field `species` has reached `threshold` turns to `to_type`."""
        check(_lib.lib().glz_gpu_set_infection(self._h, int(species), int(from_type), int(to_type), float(threshold)))

    def set_nematic_field(self, pairs) -> None:
        flat = np.ascontiguousarray(pairs, dtype=np.float64).reshape(-1)
        check(_lib.lib().glz_gpu_set_nematic_field(self._h, ptr(flat), flat.size))

    @property
    def stream(self) -> int:
        """The engine's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        return int(_lib.lib().glz_gpu_stream(self._h) or 0)

    def _after_torch(self, tensor) -> None:
        """Make the engine's stream wait for torch's current stream on the
        tensor's device, so the engine reads what torch wrote."""
        import torch

        torch.cuda.ExternalStream(self.stream, device=tensor.device).wait_stream(
            torch.cuda.current_stream(tensor.device))

    def labels_tensor(self):
        """The lattice as a torch tensor on the device, without a copy: int32
        per site (every label is below 2^31), shaped ``shape`` (depth,
        height, width). It aliases the engine's own buffer: it shows what the
        last ``step`` or restart left, stays valid until ``close``, and is for
        reading; a changed lattice goes back through ``set_labels_tensor``.
        The zero-copy form of ``GpuSession.labels``
        (glazier-py/src/lib.rs:215-219)."""
        return _view(self.device_labels(), self.shape, "<i4", self)

    def field_tensor(self, index: int):
        """Species ``index`` as a float32 torch tensor aliasing the device
        field (the engine computes fields in f32; ``field`` widens the same
        values to f64), shaped ``shape``; valid until the next ``step``, which
        moves the field to its other buffer."""
        return _view(self.device_field(index), self.shape, "<f4", self)

    def set_labels_tensor(self, labels) -> None:
        """``set_labels`` from a CUDA tensor of int32 or uint32 labels, one per
        site (x fastest), on the engine's device: copied on the device, then
        every tally recounted."""
        import torch

        t = _device_input(labels, (torch.int32, torch.uint32), self.sites, "lattice")
        self._after_torch(t)
        check(_lib.lib().glz_gpu_set_labels_device(self._h, C.c_void_p(t.data_ptr()), t.numel()))

    def set_nematic_field_tensor(self, field) -> None:
        """``set_nematic_field`` from a CUDA float32 tensor of (Q_xx, Q_xy)
        per site, ``2 * sites`` values, on the engine's device."""
        import torch

        t = _device_input(field, (torch.float32,), 2 * self.sites, "nematic field")
        self._after_torch(t)
        check(_lib.lib().glz_gpu_set_nematic_field_device(self._h, C.c_void_p(t.data_ptr()), t.numel()))

    def device_labels(self) -> int:
        p = C.c_void_p()
        check(_lib.lib().glz_gpu_device_labels(self._h, C.byref(p)))
        return int(p.value or 0)

    def device_field(self, index: int) -> int:
        p = C.c_void_p()
        check(_lib.lib().glz_gpu_device_field(self._h, int(index), C.byref(p)))
        return int(p.value or 0)
