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
    # refused before any device work, so the buffer addresses are never used
    rc = L.glz_field_step_noalloc(2048, 2048, 1, 1, 1, _lib.ptr(one), _lib.ptr(zero), _lib.ptr(zero),
                                  _lib.ptr(zero), C.c_void_p(16), C.c_void_p(16), 1, C.c_void_p(1 << 40),
                                  C.c_void_p(1 << 41), None)
    assert rc == _lib.GLZ_INVALID and big * 2 > (1 << 22)
    assert "scratch" in _lib.last_error()


def _noalloc(model, labels, cell_type, n_labels, field_in, out):
    """One call through the C ABI on device tensors; returns its status."""
    from glazier_b200 import _lib

    diffusion = np.array([s.diffusion for s in model.species])
    decay = np.array([s.decay for s in model.species])
    secretion = model.table(model.secretion).reshape(-1).copy()
    uptake = model.table(model.uptake).reshape(-1).copy()
    return _lib.lib().glz_field_step_noalloc(
        model.width, model.height, model.depth, len(model.species), model.n_types, _lib.ptr(diffusion),
        _lib.ptr(decay), _lib.ptr(secretion), _lib.ptr(uptake), C.c_void_p(labels.data_ptr()),
        C.c_void_p(cell_type.data_ptr()), n_labels, C.c_void_p(field_in.data_ptr()), C.c_void_p(out.data_ptr()),
        None)


def test_the_volume_field_step_without_allocation_matches_the_engines(device):
    """A 16^3 volume, six faces a site: species "a" takes three sub-steps
    (D = 0.4 past the volume's 1/6 limit), "b" one; two calls in a row."""
    import torch

    from glazier_b200 import _lib

    model = sheet_model(width=16, height=16, depth=16, seed=17, target_volume=512.0, order=3)
    with_species(model, [("a", 0.4, 0.03, 0.0), ("b", 0.05, 0.01, 0.5)], [[0.0, 0.0], [0.2, 0.1]],
                 [[0.0, 0.0], [0.04, 0.2]], [[0.0, 0.0], [0.0, 0.0]])
    start = tiled(model, 8, 1, 1, 1)  # one cube of side 8 in a medium
    fields = np.random.default_rng(11).uniform(0.0, 1.5, size=(2, model.sites))
    sim = device.GpuSimulation.from_start(start, fields)
    dev = torch.device("cuda", 0)
    cell_type = torch.from_numpy(start.cell_type.copy()).to(dev)
    field_in = torch.from_numpy(fields.astype(np.float32).reshape(-1)).to(dev)
    for call in range(2):
        sim.step(1)
        labels = torch.from_numpy(sim.labels().view(np.int32)).to(dev)
        out = torch.empty_like(field_in)
        rc = _noalloc(model, labels, cell_type, start.cell_type.size, field_in, out)
        assert rc == 0, _lib.last_error()
        want = np.stack([sim.field(k) for k in range(2)]).astype(np.float32)
        got = out.cpu().numpy().reshape(2, -1)
        assert np.array_equal(got, want), f"call {call}: {int((got != want).sum())} values differ"
        field_in = out
    sim.close()


def _plane_case():
    import torch

    model = sheet_model(width=32, height=32, seed=3)
    with_species(model, [("a", 0.1, 0.02, 0.0)], [[0.0], [0.3]], [[0.0], [0.05]], [[0.0], [0.0]])
    start = tiled(model, 8, 2, 2)
    dev = torch.device("cuda", 0)
    field = torch.from_numpy(np.random.default_rng(2).uniform(0.0, 1.0, model.sites).astype(np.float32)).to(dev)
    labels = torch.from_numpy(start.labels.view(np.int32).copy()).to(dev)
    cell_type = torch.from_numpy(start.cell_type.copy()).to(dev)
    return model, start, labels, cell_type, field


def test_overlapping_buffers_are_refused(device):
    import torch

    from glazier_b200 import _lib

    model, start, labels, cell_type, field = _plane_case()
    before = field.clone()
    rc = _noalloc(model, labels, cell_type, start.cell_type.size, field, field)
    assert rc == _lib.GLZ_INVALID and "overlap" in _lib.last_error()
    assert torch.equal(field, before)


def test_a_bad_label_or_type_is_reported_and_its_sites_take_no_exchange(device):
    """A label at or past n_labels, or a cell type at or past n_types, is
    reported (GLZ_INVALID); its sites get diffusion and decay only, which is
    what the medium gets, so the output equals a call with them made medium."""
    import torch

    from glazier_b200 import _lib

    model, start, labels, cell_type, field = _plane_case()
    n = start.cell_type.size
    cell_sites = torch.nonzero(labels == 1).flatten()
    medium = labels.clone()
    medium[cell_sites] = 0
    want = torch.empty_like(field)
    assert _noalloc(model, medium, cell_type, n, field, want) == 0, _lib.last_error()

    bad_label = labels.clone()
    bad_label[cell_sites] = n  # one past the type table
    out = torch.empty_like(field)
    assert _noalloc(model, bad_label, cell_type, n, field, out) == _lib.GLZ_INVALID
    assert "label" in _lib.last_error()
    assert torch.equal(out, want)

    bad_type = cell_type.clone()
    bad_type[1] = model.n_types  # one past the rate tables
    out = torch.empty_like(field)
    assert _noalloc(model, labels, bad_type, n, field, out) == _lib.GLZ_INVALID
    assert "cell type" in _lib.last_error()
    assert torch.equal(out, want)

    # the status word starts clean on the next call
    out = torch.empty_like(field)
    assert _noalloc(model, labels, cell_type, n, field, out) == 0, _lib.last_error()
