"""The field step that allocates nothing, against the engine's own.

glz_field_step_noalloc is for callers that cannot call cudaMalloc: a host
application that fixes its device-memory budget at start-up and forbids
allocation afterwards, or a coupled solver that hands this library only
buffers it owns. It keeps its scratch in one fixed device array instead.

The test drives it through the C ABI on device buffers: after each engine
step it takes the engine's lattice and the field from before the step, runs
the no-allocation step, and requires the engine's field after the step bit
for bit (the tolerance the field parity tests hold), on two calls in a row.
The file sorts last so a run that stops at the first failure has already run
every other test.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import sheet_model, tiled, with_species

pytestmark = pytest.mark.gpu


def test_the_field_step_without_allocation_matches_the_engines(device):
    import torch

    from glazier_b200 import _lib

    # Cells in one corner, medium elsewhere; species "a" takes three
    # sub-steps (D = 0.6 past the plane's 0.25 limit), "b" one.
    model = sheet_model(width=64, height=48, seed=13)
    with_species(model, [("a", 0.6, 0.02, 0.0), ("b", 0.1, 0.01, 1.0)], [[0.0, 0.0], [0.3, 0.0]],
                 [[0.0, 0.0], [0.05, 0.1]], [[0.0, 0.0], [0.0, 0.0]])
    start = tiled(model, 8, 6, 4)
    rng = np.random.default_rng(5)
    fields = rng.uniform(0.0, 2.0, size=(2, model.sites))

    sim = device.GpuSimulation.from_start(start, fields)
    L = _lib.lib()
    dev = torch.device("cuda", 0)
    cell_type = torch.from_numpy(start.cell_type.copy()).to(dev)
    field_in = torch.from_numpy(fields.astype(np.float32).reshape(-1)).to(dev)
    diffusion = np.array([s.diffusion for s in model.species])
    decay = np.array([s.decay for s in model.species])
    secretion = model.table(model.secretion).reshape(-1).copy()
    uptake = model.table(model.uptake).reshape(-1).copy()

    for call in range(2):
        sim.step(1)
        out = torch.empty_like(field_in)
        rc = L.glz_field_step_noalloc(
            model.width, model.height, model.depth, 2, model.n_types, _lib.ptr(diffusion), _lib.ptr(decay),
            _lib.ptr(secretion), _lib.ptr(uptake), C.c_void_p(sim.device_labels()), C.c_void_p(cell_type.data_ptr()),
            start.cell_type.size, C.c_void_p(field_in.data_ptr()), C.c_void_p(out.data_ptr()), None)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        want = np.stack([sim.field(k) for k in range(2)]).astype(np.float32)
        got = out.cpu().numpy().reshape(2, -1)
        assert np.array_equal(got, want), f"call {call}: {int((got != want).sum())} values differ"
        field_in = out
    sim.close()


def test_a_step_past_the_scratch_limit_is_refused(device):
    from glazier_b200 import _lib

    L = _lib.lib()
    one = np.array([2.0])  # 8 sub-steps in a plane, so two scratch buffers
    zero = np.array([0.0])
    big = 2048 * 2048  # two buffers of 4 Mi values: past the 4 Mi the entry point holds
    rc = L.glz_field_step_noalloc(2048, 2048, 1, 1, 1, _lib.ptr(one), _lib.ptr(zero), _lib.ptr(zero),
                                  _lib.ptr(zero), C.c_void_p(16), C.c_void_p(16), 1, C.c_void_p(16),
                                  C.c_void_p(16), None)
    assert rc == _lib.GLZ_INVALID and big * 2 > (1 << 22)
    assert "scratch" in _lib.last_error()
