"""The zero-copy session: the lattice and the fields as device tensors, and
restarts and nematic fields handed over from device tensors.

The reference's coupling loop (README.md:332-337, glazier-py/src/lib.rs:184-241)
copies the lattice to the host and the nematic field back every round; here
the same loop stays on the device. Each test holds the device form to the host
form it replaces: same values, same run.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

from conftest import tiled
from glazier_b200.blueprint import CellType, Model

pytestmark = pytest.mark.gpu


def _nematic_model(size=64, seed=7):
    # gpu_nematic.rs:16-36, with a field that varies from site to site
    m = Model(width=size, height=size, contact=[0.0, 16.0, 16.0, 8.0],
              types=[CellType(), CellType(target_volume=64.0, lambda_volume=2.0, lambda_nematic=6.0)],
              temperature=10.0, neighbour_order=2, seed=seed)
    angle = 0.6
    m.nematic = np.tile([math.cos(2 * angle), math.sin(2 * angle)], (size * size, 1))
    return m


def _field_from_labels(labels):
    """A nematic field computed from a lattice, every value exact in f32 (so
    the host form, which takes f64, carries the same numbers): the solver
    side of a coupling round."""
    if isinstance(labels, np.ndarray):
        lab = labels.astype(np.int64)
        return ((lab % 7) - 3).astype(np.float32) / 4, ((lab % 5) - 2).astype(np.float32) / 4
    return ((labels % 7) - 3).float() / 4, ((labels % 5) - 2).float() / 4


def test_the_lattice_view_is_the_engine_buffer_without_a_copy(device):
    import torch

    from glazier_b200.workloads import monolayer

    start = monolayer(128)
    sim = device.GpuSimulation.from_start(start)
    sim.step(10)
    view = sim.labels_tensor()
    assert view.is_cuda and view.dtype == torch.int32
    assert tuple(view.shape) == (1, 128, 128)
    assert view.data_ptr() == sim.device_labels()
    assert np.array_equal(view.cpu().numpy().reshape(-1).view(np.uint32), sim.labels())
    sim.step(10)  # the same view shows the new lattice
    assert np.array_equal(view.cpu().numpy().reshape(-1).view(np.uint32), sim.labels())
    sim.close()


def test_a_field_view_holds_the_values_the_host_copy_widens(device):
    from glazier_b200.workloads import INFECTION_RULE, infection_start

    start = infection_start(size=128, grid=8, immune=8)
    sim = device.GpuSimulation.from_start(start)
    sim.set_infection(*INFECTION_RULE)
    sim.step(5)
    for index in range(len(start.model.species)):
        view = sim.field_tensor(index)
        assert tuple(view.shape) == (1, 128, 128)
        assert np.array_equal(view.cpu().numpy().reshape(-1).astype(np.float64), sim.field(index))
    sim.close()


def test_a_restart_from_a_device_tensor_runs_as_one_from_the_host(device):
    import torch

    from glazier_b200.workloads import monolayer

    start = monolayer(128)
    shifted = np.roll(start.labels.reshape(128, 128), (3, 5), axis=(0, 1)).reshape(-1).astype(np.uint32)
    host = device.GpuSimulation.from_start(start)
    dev = device.GpuSimulation.from_start(start)
    host.step(3)
    dev.step(3)
    host.set_labels(shifted)
    dev.set_labels_tensor(torch.from_numpy(shifted.view(np.int32)).cuda())
    for sim in (host, dev):
        sim.step(20)
    assert np.array_equal(host.labels(), dev.labels())
    assert np.array_equal(host.volumes(), dev.volumes())
    assert np.array_equal(host.surfaces(), dev.surfaces())
    host.close()
    dev.close()


def test_a_coupling_loop_on_the_device_runs_as_the_host_loop(device):
    # README.md:332-337: rounds of steps, the lattice out, a new field in
    import torch

    model = _nematic_model()
    host = device.GpuSimulation.from_start(tiled(model, 8))
    dev = device.GpuSimulation.from_start(tiled(model, 8))
    for _ in range(4):
        host.step(25)
        dev.step(25)
        q_xx, q_xy = _field_from_labels(host.labels())
        host.set_nematic_field(np.stack([q_xx, q_xy], axis=1).astype(np.float64))
        lab = dev.labels_tensor().reshape(-1)
        t_xx, t_xy = _field_from_labels(lab)
        dev.set_nematic_field_tensor(torch.stack([t_xx, t_xy], dim=1))
    assert np.array_equal(host.labels(), dev.labels())
    assert np.array_equal(host.volumes(), dev.volumes())
    assert np.array_equal(host.surfaces(), dev.surfaces())
    host.close()
    dev.close()


def test_the_session_hands_out_the_lattice_and_takes_a_field_on_the_device(device):
    import json
    from pathlib import Path

    import torch

    from glazier_b200 import native

    golden = json.loads((Path(__file__).parent / "golden" / "serial_reference.json").read_text())
    text = golden["parse"]["monolayer.json"]["text"]
    session = native.GpuSession(text)
    session.step(5)
    view = session.labels_tensor()
    assert view.reshape(-1).cpu().tolist() == session.labels()
    # a monolayer without a nematic coupling refuses a field, as the host form does
    field = torch.zeros(2 * view.numel(), dtype=torch.float32, device=view.device)
    with pytest.raises(ValueError, match="no nematic coupling"):
        session.set_nematic_field_tensor(field)


def test_device_inputs_that_are_not_on_the_device_or_not_the_lattice_are_refused(device):
    import torch

    from glazier_b200 import _lib
    from glazier_b200.workloads import monolayer

    sim = device.GpuSimulation.from_start(monolayer(128))
    with pytest.raises(device.GpuError, match="not a CUDA tensor"):
        sim.set_labels_tensor(torch.zeros(128 * 128, dtype=torch.int32))
    with pytest.raises(device.GpuError, match="values, not"):
        sim.set_labels_tensor(torch.zeros(128 * 127, dtype=torch.int32, device="cuda"))
    with pytest.raises(device.GpuError, match="float32"):
        sim.set_labels_tensor(torch.zeros(128 * 128, dtype=torch.float32, device="cuda"))
    # through the C ABI, a host address is refused before any copy
    host = np.zeros(128 * 128, dtype=np.uint32)
    rc = _lib.lib().glz_gpu_set_labels_device(sim.handle, host.ctypes.data_as(C.c_void_p), host.size)
    assert rc == _lib.GLZ_INVALID
    assert "not device memory" in _lib.last_error()
    sim.close()
