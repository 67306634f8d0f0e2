"""The field step, differentiable with respect to its parameters.

``FieldAdjoint`` wraps the ``glz_adj_*`` entry points: given a recorded
trajectory of site owners (the cell type owning each site after each Monte
Carlo step, 255 for the medium), its forward runs the engine's own f32 field
step for every step of the trajectory, and its backward runs the hand-written
adjoint, recomputing every `checkpoint_every`-step segment from a saved
state. ``field_trajectory`` exposes it to PyTorch as a
``torch.autograd.Function``: gradients flow to the parameters
(D, decay per species; secretion, uptake per type and species) and to the
initial fields. The discrete sweep that produced the trajectory is never
differentiated.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .engine import check

MEDIUM = 255


def owner_types(labels: np.ndarray, cell_type: np.ndarray) -> np.ndarray:
    """The owner-type map of a lattice: each site's cell type, 255 where the
    medium (label 0) sits."""
    out = np.asarray(cell_type, dtype=np.uint8)[np.asarray(labels, dtype=np.int64)]
    out[np.asarray(labels) == 0] = MEDIUM
    return out


def record_trajectory(sim, steps: int) -> np.ndarray:
    """Run a GpuSimulation for `steps` Monte Carlo steps and record, after
    each, the owner type of every site: the exchange mask of that step's field
    update for a model without division or death."""
    out = np.empty((steps, sim.sites), dtype=np.uint8)
    for t in range(steps):
        sim.step(1)
        out[t] = owner_types(sim.labels(), sim.cell_types())
    return out


class FieldAdjoint:
    """The forward and adjoint of `steps` field steps on one lattice."""

    def __init__(self, width: int, height: int, depth: int, n_species: int, n_types: int, trajectory,
                 checkpoint_every: int = 10, device: int | None = None):
        L = _lib.lib()
        if device is not None:
            check(L.glz_set_device(int(device)))
        traj = np.ascontiguousarray(trajectory, dtype=np.uint8)
        steps = traj.shape[0]
        h = C.c_void_p()
        check(L.glz_adj_create(width, height, depth, n_species, n_types, steps, checkpoint_every, C.byref(h)))
        self._h = h
        check(L.glz_adj_set_trajectory(h, _lib.ptr(traj)))
        self.shape = (n_species, width * height * depth)
        self.n_params = 2 * n_species + 2 * n_types * n_species
        self.steps = steps

    @property
    def stream(self) -> int:
        """The address of the CUDA stream the handle's work runs on."""
        return int(_lib.lib().glz_adj_stream(self._h) or 0)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().glz_adj_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, params, fields0):
        """params: n_params f64 values; fields0: a contiguous f32 CUDA tensor of
        shape (n_species, sites). Returns the fields after every step."""
        import torch

        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64))
        f0 = fields0.detach().to(torch.float32).contiguous()
        if f0.shape != self.shape or not f0.is_cuda:
            raise ValueError(f"fields0 must be a CUDA tensor of shape {self.shape}")
        if p.size != self.n_params:
            raise ValueError(f"{p.size} parameters for {self.n_params}")
        out = torch.empty_like(f0)
        # the handle runs on its own stream: let torch's pending work land first
        torch.cuda.current_stream(f0.device).synchronize()
        check(_lib.lib().glz_adj_forward(self._h, _lib.ptr(p), C.c_void_p(f0.data_ptr()), C.c_void_p(out.data_ptr())))
        return out

    def backward(self, grad_final):
        """The gradients of a loss whose gradient at the final fields is
        `grad_final`, with respect to the parameters of the last forward (f64
        numpy) and to the initial fields (f32 tensor)."""
        import torch

        g = grad_final.detach().to(torch.float32).contiguous()
        if g.shape != self.shape or not g.is_cuda:
            raise ValueError(f"grad_final must be a CUDA tensor of shape {self.shape}")
        gp = np.zeros(self.n_params, dtype=np.float64)
        gf = torch.empty_like(g)
        torch.cuda.current_stream(g.device).synchronize()
        check(_lib.lib().glz_adj_backward(self._h, C.c_void_p(g.data_ptr()), _lib.ptr(gp), C.c_void_p(gf.data_ptr())))
        return gp, gf


def _function():
    import torch

    class FieldTrajectory(torch.autograd.Function):
        @staticmethod
        def forward(ctx, params, fields0, adjoint):
            ctx.adjoint = adjoint
            ctx.params_device = params.device
            out = adjoint.forward(params.detach().cpu().numpy(), fields0)
            return out

        @staticmethod
        def backward(ctx, grad_out):
            gp, gf = ctx.adjoint.backward(grad_out)
            return torch.from_numpy(gp).to(ctx.params_device), gf, None

    return FieldTrajectory


_FN = None


def field_trajectory(params, fields0, adjoint: FieldAdjoint):
    """The fields after the adjoint's trajectory, as a differentiable function
    of `params` (f64 tensor) and `fields0` (f32 CUDA tensor)."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(params, fields0, adjoint)
