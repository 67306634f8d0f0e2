"""Bit-exact parity: the device engine against the host replay of its schedule.

Every case runs the same start on the B200 (through the C ABI) and on the
replay (oracle/replay.c) and requires identical labels, per-label volumes,
surfaces and cell types, and bit-identical f32 fields. Each case runs with
the sweep's tensor-copy window load on and off, with the persistent grid at
its default and capped at three CTAs (each CTA then walks several tiles
through every window buffer), and on both sweep kernels (the lean one takes
the models that price contact, volume and surface only; the general one
every model), so every load path and both kernels are held to one result.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import sheet_model, tiled, with_species
from glazier_b200.blueprint import Start
from oracle.replay import ReplayOracle

pytestmark = pytest.mark.gpu


def _plain():
    return tiled(sheet_model(seed=1)), 20


def _surface():
    return tiled(sheet_model(seed=3, target_surface=34.0, lambda_surface=0.1)), 20


def _von_neumann():
    return tiled(sheet_model(seed=5, order=1, contact=(0, 12, 12, 6))), 20


def _large():
    # 384 x 192: the tiles at x0 = 128, y0 = 32..128 lie clear of the periodic
    # edge, so their windows arrive by tensor copy
    m = sheet_model(width=384, height=192, seed=2, contact=(0, 10, 10, 10), lambda_volume=1.0,
                    target_surface=92.0, lambda_surface=0.2)
    return tiled(m), 10


def _ragged():
    # 264 x 180: tiles overhang the right and bottom edges, and edge windows
    # take a tensor copy with out-of-lattice cells filled, then patched
    m = sheet_model(width=264, height=180, seed=9, contact=(0, 10, 10, 10), lambda_volume=1.0,
                    target_surface=92.0, lambda_surface=0.2)
    return tiled(m), 8


def _ragged_volume():
    # 152 x 24 x 20: overhanging tiles on x and z, edge windows copied and patched
    m = sheet_model(width=152, height=24, depth=20, seed=10, target_volume=512.0, order=3,
                    contact=(0, 10, 10, 10), lambda_volume=1.0)
    return tiled(m), 3


def _unaligned():
    # 34 columns: rows are not whole 16-byte units, so the window takes plain loads
    return tiled(sheet_model(width=34, height=22, seed=4), 6), 25


def _medium():
    m = sheet_model(width=96, height=64, seed=6)
    return tiled(m, 8, 6, 4), 20


def _volume(order):
    def make():
        m = sheet_model(width=32, height=32, depth=32, seed=31, target_volume=512.0, order=order,
                        target_surface=3176.0 if order == 3 else 0.0, lambda_surface=0.2 if order == 3 else 0.0)
        return tiled(m), 6
    return make


def _volume_wide():
    # 192 x 32 x 32: four tiles lie clear of the edge and take tensor copies
    m = sheet_model(width=192, height=32, depth=32, seed=8, target_volume=512.0, order=3, contact=(0, 10, 10, 10),
                    lambda_volume=1.0)
    return tiled(m), 4


def _fields():
    m = with_species(sheet_model(seed=11), [("IFNg", 0.4, 0.01, 0.0), ("b", 0.7, 0.02, 1.0)],
                     [[0.0, 0.0], [0.2, 0.0]], [[0.0, 0.0], [0.01, 0.1]], [[0.0, 0.0], [3.0, -2.0]])
    return tiled(m), 20


def _length():
    return tiled(sheet_model(seed=41, target_length=24.0, lambda_length=1.0)), 20


def _length_volume():
    m = sheet_model(width=32, height=32, depth=32, seed=12, target_volume=512.0, order=3,
                    target_length=14.0, lambda_length=0.5)
    return tiled(m), 3


def _connected():
    m = sheet_model(seed=23, contact=(0, 4, 4, 4), lambda_volume=1.0, temperature=40.0, connected=True)
    return tiled(m), 20


def _drift():
    # a drift along +x for the cells, diagonal pulls included (Moore picks)
    m = sheet_model(seed=13, external=(0.75, -0.25, 0.0))
    return tiled(m, 8, 6, 6), 25


def _motility():
    # Act: a strong memory (max 20, lambda 60), writes deferred to the pass's end
    m = sheet_model(seed=17, max_activity=20.0, lambda_activity=60.0, target_volume=64.0)
    return tiled(m, 8, 5, 5), 25


def _nematic():
    # a random director field the cells' long axes couple to (and a length
    # term beside it, so both read the same moment words)
    m = sheet_model(seed=19, lambda_nematic=3.0, target_length=10.0, lambda_length=0.5)
    m.nematic = np.random.default_rng(19).uniform(-0.5, 0.5, size=(m.sites, 2))
    return tiled(m), 20


def _nematic_volume():
    m = sheet_model(width=32, height=32, depth=32, seed=20, target_volume=512.0, order=3, lambda_nematic=40.0)
    m.nematic = np.random.default_rng(20).uniform(-1.0, 1.0, size=(m.sites, 2))
    return tiled(m), 4


def _population():
    m = sheet_model(seed=8, division_volume=72.0, death_rate=0.005, target_volume=100.0)
    return tiled(m, 6, 6, 6), 40


def _two_types_plane():
    # 128 x 128, two cell types in a checker of cells and a medium border:
    # per-type contact, volume and surface tables; a small plane that a
    # cluster of four CTAs holds, rows and labels spread over them
    from glazier_b200.blueprint import CellType, Model

    m = Model(width=128, height=128, contact=[0.0, 16.0, 16.0, 16.0, 8.0, 12.0, 16.0, 12.0, 10.0],
              types=[CellType(), CellType(target_volume=64.0, lambda_volume=2.0),
                     CellType(target_volume=48.0, lambda_volume=1.0, target_surface=30.0, lambda_surface=0.1)],
              temperature=10.0, neighbour_order=2, seed=29)
    start = tiled(m, 8, 14, 14)
    cell_type = np.asarray(start.cell_type).copy()
    cell_type[1:] = 1 + (np.arange(1, cell_type.size) % 2)
    return Start(m, start.labels, cell_type.astype(np.uint8)), 20


def _chemotaxis_ramp():
    m = with_species(sheet_model(seed=21), [("attractant", 0.0, 0.0, 0.0)], [[0.0], [0.0]], [[0.0], [0.0]],
                     [[0.0], [4.0]])
    labels = np.zeros(64 * 64, dtype=np.uint32)
    ys, xs = np.divmod(np.arange(64 * 64), 64)
    labels[(xs >= 24) & (xs < 32) & (ys >= 24) & (ys < 32)] = 1
    start = Start(m, labels, np.array([0, 1], dtype=np.uint8))
    fields = xs.astype(np.float64)[None, :]
    return (start, fields), 30


CASES = {
    "plain": _plain,
    "surface": _surface,
    "von-neumann": _von_neumann,
    "large": _large,
    "ragged": _ragged,
    "ragged-volume": _ragged_volume,
    "unaligned": _unaligned,
    "medium": _medium,
    "volume-26": _volume(3),
    "volume-18": _volume(2),
    "volume-6": _volume(1),
    "volume-wide": _volume_wide,
    "fields": _fields,
    "length": _length,
    "length-volume": _length_volume,
    "connected": _connected,
    "population": _population,
    "drift": _drift,
    "motility": _motility,
    "nematic": _nematic,
    "nematic-volume": _nematic_volume,
    "chemotaxis-ramp": _chemotaxis_ramp,
    "two-types-plane": _two_types_plane,
}


@pytest.mark.parametrize("kernel", ["band", "cluster", "resident", "direct", "compact", "gathered", "lean", "general"])
@pytest.mark.parametrize("ctas", ["0", "3"])
@pytest.mark.parametrize("tma", ["1", "0"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_the_device_reproduces_the_replay_bit_for_bit(device, name, tma, ctas, kernel, monkeypatch):
    """`ctas` 3 caps the sweep's persistent grid at three CTAs, so every CTA
    walks several tiles and every window buffer takes tensor copies; `kernel`
    forces the lean models onto the band sweep (a plane's rows streamed by
    bands, every pass of a call in one launch), the cluster (a plane held in one thread-block
    cluster's shared memory), the resident (every MCS of a call in one
    launch, for models with nothing between passes), the direct (one thread a
    target, or with `compact` each warp's unlike copies queued and priced in
    full rounds, or with `gathered` a block's), the lean or the general kernel (models with other terms
    always take the general one)."""
    if kernel in ("band", "cluster", "resident", "direct", "compact", "gathered") and (tma == "0" or ctas == "3"):
        pytest.skip("the band, resident and direct kernels take no tensor copies and no grid cap")
    made, steps = CASES[name]()
    start, fields = made if isinstance(made, tuple) else (made, None)
    monkeypatch.setenv("GLAZIER_SWEEP_TMA", tma)
    monkeypatch.setenv("GLAZIER_SWEEP_CTAS", ctas)
    monkeypatch.setenv("GLAZIER_SWEEP_LEAN", "0" if kernel == "general" else "1")
    monkeypatch.setenv("GLAZIER_SWEEP_DIRECT",
                       "1" if kernel in ("cluster", "resident", "direct", "compact", "gathered") else "0")
    monkeypatch.setenv("GLAZIER_SWEEP_COMPACT", {"compact": "1", "gathered": "2"}.get(kernel, "0"))
    monkeypatch.setenv("GLAZIER_SWEEP_RESIDENT", "1" if kernel in ("cluster", "resident") else "0")
    monkeypatch.setenv("GLAZIER_SWEEP_CLUSTER", "1" if kernel == "cluster" else "0")
    monkeypatch.setenv("GLAZIER_SWEEP_BAND", "1" if kernel == "band" else "0")
    gpu = device.GpuSimulation.from_start(start, fields)
    replay = ReplayOracle.from_start(start, fields)
    for chunk in (1, steps - 1):
        gpu.step(chunk)
        replay.step(chunk)
        assert gpu.n_labels == replay.n_labels
        labels = gpu.labels()
        want = replay.labels()
        assert np.array_equal(labels, want), f"{int((labels != want).sum())} sites differ after {gpu.mcs} MCS"
        assert np.array_equal(gpu.volumes(), replay.volumes())
        assert np.array_equal(gpu.surfaces(), replay.surfaces())
        assert np.array_equal(gpu.cell_types(), replay.cell_types())
        for k in range(len(start.model.species)):
            assert np.array_equal(gpu.field(k).astype(np.float32), replay.field(k))
    gpu.close()


@pytest.mark.parametrize("ctas", ["0", "3"])
def test_the_infection_model_reproduces_the_replay_bit_for_bit(device, ctas, monkeypatch):
    """The two-field infection model with its healthy-to-infected rule (an
    extension with no reference counterpart, so its oracle is the replay with
    the same rule): labels, volumes, surfaces, cell types and both fields
    identical over 60 MCS, with infections taking place."""
    from glazier_b200.workloads import INFECTION_RULE, infection_start

    monkeypatch.setenv("GLAZIER_SWEEP_CTAS", ctas)
    start = infection_start()
    gpu = device.GpuSimulation.from_start(start)
    replay = ReplayOracle.from_start(start)
    gpu.set_infection(*INFECTION_RULE)
    replay.set_infection(*INFECTION_RULE)
    for chunk in (1, 29, 30):
        gpu.step(chunk)
        replay.step(chunk)
        assert gpu.n_labels == replay.n_labels
        labels = gpu.labels()
        want = replay.labels()
        assert np.array_equal(labels, want), f"{int((labels != want).sum())} sites differ after {gpu.mcs} MCS"
        assert np.array_equal(gpu.volumes(), replay.volumes())
        assert np.array_equal(gpu.surfaces(), replay.surfaces())
        assert np.array_equal(gpu.cell_types(), replay.cell_types())
        for k in range(2):
            assert np.array_equal(gpu.field(k).astype(np.float32), replay.field(k))
    types, vols = gpu.cell_types(), gpu.volumes()
    assert int(((types == 2) & (vols > 0)).sum()) > 3
    gpu.close()


def test_a_bad_infection_rule_is_refused(device):
    from glazier_b200.engine import GpuError
    from glazier_b200.workloads import infection_start

    gpu = device.GpuSimulation.from_start(infection_start())
    for rule in ((2, 1, 2, 5.0), (0, 0, 2, 5.0), (0, 1, 1, 5.0), (0, 1, 2, -1.0), (0, 1, 2, 1e12)):
        with pytest.raises(GpuError):
            gpu.set_infection(*rule)
    gpu.close()


def test_a_replaced_nematic_field_reproduces_the_replay_bit_for_bit(device):
    """glz_gpu_set_nematic_field mid-run: the per-cell sums follow the new
    field on both sides."""
    start, steps = _nematic()
    gpu = device.GpuSimulation.from_start(start)
    replay = ReplayOracle.from_start(start)
    gpu.step(5)
    replay.step(5)
    field = np.random.default_rng(7).uniform(-1.0, 1.0, size=(start.model.sites, 2))
    gpu.set_nematic_field(field)
    replay.set_nematic_field(field)
    gpu.step(10)
    replay.step(10)
    assert np.array_equal(gpu.labels(), replay.labels())
    assert np.array_equal(gpu.volumes(), replay.volumes())
    gpu.close()

