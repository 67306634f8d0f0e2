"""A batch of independent Cellular Potts replicas run as one on the B200.

The Python face of the ``glz_ens_*`` entry points: every replica whose model
prices contact, volume and surface only goes through one persistent launch
per colour, one Monte Carlo step replayed from a CUDA graph; a replica with
fields, division, death or the other terms runs as its own engine beside the
batch, at the same time. Each replica's results are bit-identical to a
``GpuSimulation`` run of the same start, so the schedule the autotuner picks
changes only the time.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .engine import GpuError, check


class Ensemble:
    """Replicas given as ``glazier_b200.blueprint.Start`` objects (their
    models may differ in size, parameters and terms; the batched ones share a
    neighbourhood)."""

    def __init__(self, starts, device: int | None = None):
        L = _lib.lib()
        if device is not None:
            check(L.glz_set_device(int(device)))
        self._keep: list = []
        n = len(starts)
        models = (_lib.GlzModel * n)()
        labels = (C.c_void_p * n)()
        types = (C.c_void_p * n)()
        counts = (C.c_size_t * n)()
        for i, st in enumerate(starts):
            models[i] = _lib.model_struct(st.model, self._keep)
            lab = np.ascontiguousarray(st.labels, dtype=np.uint32).reshape(-1)
            ct = np.ascontiguousarray(st.cell_type, dtype=np.uint8).reshape(-1)
            self._keep += [lab, ct]
            labels[i] = lab.ctypes.data
            types[i] = ct.ctypes.data
            counts[i] = ct.size
        h = C.c_void_p()
        check(L.glz_ens_create(n, models, labels, types, counts, C.byref(h)))
        self._h = h
        self.n = n
        self.sites = [st.model.sites for st in starts]

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().glz_ens_destroy(self._h)
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

    def n_labels(self, i: int) -> int:
        """Labels replica ``i`` has issued, the medium included."""
        return int(_lib.lib().glz_ens_n_labels(self._h, int(i)))

    def set_infection(self, i: int, species: int, from_type: int, to_type: int, threshold: float) -> None:
        """The infection rule for replica ``i`` (``GpuSimulation.set_infection``)."""
        check(_lib.lib().glz_ens_set_infection(self._h, int(i), int(species), int(from_type), int(to_type),
                                               float(threshold)))

    def step(self, steps: int = 1) -> None:
        check(_lib.lib().glz_ens_step(self._h, int(steps)))

    def step_timed(self, steps: int = 1) -> float:
        """Run and return the device milliseconds."""
        ms = C.c_double(0.0)
        check(_lib.lib().glz_ens_step_timed(self._h, int(steps), C.byref(ms)))
        return ms.value

    def autotune(self, trial_steps: int = 3) -> int:
        choice = C.c_int(-1)
        check(_lib.lib().glz_ens_autotune(self._h, int(trial_steps), C.byref(choice)))
        return choice.value

    def set_schedule(self, schedule: int, max_ctas: int = 0) -> None:
        check(_lib.lib().glz_ens_set_schedule(self._h, int(schedule), int(max_ctas)))

    @property
    def mcs(self) -> int:
        return int(_lib.lib().glz_ens_mcs(self._h))

    def _replica(self, i: int) -> int:
        if not 0 <= int(i) < self.n:
            raise GpuError(_lib.GLZ_INVALID, f"no such replica: {i} of {self.n}")
        return int(i)

    def labels(self, i: int) -> np.ndarray:
        i = self._replica(i)
        out = np.empty(self.sites[i], dtype=np.uint32)
        check(_lib.lib().glz_ens_labels(self._h, int(i), _lib.ptr(out), out.size))
        return out

    def volumes(self, i: int) -> np.ndarray:
        n = C.c_size_t(self.n_labels(i))
        out = np.empty(n.value, dtype=np.uint32)
        check(_lib.lib().glz_ens_volumes(self._h, int(i), _lib.ptr(out), C.byref(n)))
        return out

    def surfaces(self, i: int) -> np.ndarray:
        n = C.c_size_t(self.n_labels(i))
        out = np.empty(n.value, dtype=np.int64)
        check(_lib.lib().glz_ens_surfaces(self._h, int(i), _lib.ptr(out), C.byref(n)))
        return out
