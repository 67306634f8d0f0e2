"""Every term in a volume on the device: the reference's own check, and
bit-exact parity with the host replay of the schedule.

- `the_device_runs_every_term_in_a_volume` (glazier-tests/tests/
  volume_terms.rs:217-277) with its bands: a 32^3 volume of 8^3 cells with
  the connectivity veto, Act motility, a drift along z, death, the surface
  term, one secreted field and chemotaxis up it, 60 MCS; cells survive, the
  counters equal the lattice they wrote, the field fills.
- The same model, and the infection slab (blueprints/infection-volume.json:
  a 64 x 64 x 32 slab, 18 neighbours, a field of D 0.5 that takes three
  sub-steps, the veto over the 26 ring, death, motile immune cells climbing
  the virus), against the replay: labels, volumes, surfaces, cell types and
  the f32 field identical after the first MCS and after 12, on the direct
  kernel (plain, warp-queued and block-queued) and on the tiled general kernel with the window's
  tensor copy on and off and the persistent grid at its default and capped at
  three CTAs.
- Division in a volume: cells that grow past their division volume are cut
  through their centroid across the power-iteration axis, against the replay.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from glazier_b200.blueprint import Blueprint, CellType, Model, Species, Start
from oracle.replay import ReplayOracle

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "serial_reference.json"


def _every_term(seed=67) -> Start:
    """volume_terms.rs:13-31 `base`, with the terms of :222-245."""
    cell = CellType(target_volume=512.0, lambda_volume=2.0, connected=True, max_activity=20.0,
                    lambda_activity=60.0, external=(0.0, 0.0, 1.0), death_rate=0.002, target_surface=300.0,
                    lambda_surface=0.05)
    m = Model(width=32, height=32, depth=32, contact=[0.0, 16.0, 16.0, 8.0], types=[CellType(), cell],
              temperature=10.0, neighbour_order=2, seed=seed,
              species=[Species("signal", 0.3, 0.01, 0.0)], secretion=[[0.0], [0.2]], uptake=[[0.0], [0.0]],
              chemotaxis=[[0.0], [10.0]])
    m.validate()
    return Start.tiled(m, 8)


def _infection_volume() -> Start:
    text = json.loads(GOLDEN.read_text())["parse"]["infection-volume.json"]["text"]
    return Blueprint.from_json(text).start()


def _division_volume() -> Start:
    """64 cells of side 6 in medium in a 36^3 volume that grow toward 300
    sites and divide at 224; a death rate on the second type."""
    m = Model(width=36, height=36, depth=36, contact=[0.0, 16.0, 16.0, 16.0, 8.0, 12.0, 16.0, 12.0, 10.0],
              types=[CellType(), CellType(target_volume=300.0, lambda_volume=2.0, division_volume=224.0),
                     CellType(target_volume=216.0, lambda_volume=2.0, death_rate=0.01)],
              temperature=12.0, neighbour_order=3, seed=71)
    start = Start.tiled_grid(m, 6, 4, 4, 4)
    cell_type = np.asarray(start.cell_type).copy()
    cell_type[1:] = 1 + (np.arange(1, cell_type.size) % 5 == 0)
    return Start(m, start.labels, cell_type.astype(np.uint8))


def test_the_device_runs_every_term_in_a_volume(device):
    start = _every_term()
    started = int(start.labels.max())
    gpu = device.GpuSimulation.from_start(start)
    gpu.step(60)
    volumes = gpu.volumes()
    live = int((volumes[1:] > 0).sum())
    assert 0 < live <= started, f"{live} of {started} cells left"
    labels = gpu.labels()
    counted = np.bincount(labels.astype(np.int64), minlength=volumes.size)
    assert np.array_equal(volumes[1:], counted[1:volumes.size])
    assert float(gpu.field(0).sum()) > 0.0, "the field never filled"
    gpu.close()


CASES = {"every-term": _every_term, "infection-volume": _infection_volume, "division-volume": _division_volume}


# (kernel, tensor copies, persistent grid cap): the direct kernel (one thread
# per target, the default for these sizes), its warp- and block-queued forms,
# and the tiled general kernel with its window copied by TMA or by plain
# loads, its grid at the default or capped at three CTAs
MODES = {"direct": ("direct", "1", "0"), "compact": ("compact", "1", "0"), "gathered": ("gathered", "1", "0"),
         "tiled": ("general", "1", "0"), "tiled-plain": ("general", "0", "0"), "tiled-capped": ("general", "1", "3")}


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("name", sorted(CASES))
def test_a_volume_with_every_term_reproduces_the_replay_bit_for_bit(device, name, mode, monkeypatch):
    kernel, tma, ctas = MODES[mode]
    monkeypatch.setenv("GLAZIER_SWEEP_TMA", tma)
    monkeypatch.setenv("GLAZIER_SWEEP_CTAS", ctas)
    monkeypatch.setenv("GLAZIER_SWEEP_DIRECT", "0" if kernel == "general" else "1")
    monkeypatch.setenv("GLAZIER_SWEEP_COMPACT", {"compact": "1", "gathered": "2"}.get(kernel, "0"))
    start = CASES[name]()
    gpu = device.GpuSimulation.from_start(start)
    assert gpu.sweep_kernel == kernel
    replay = ReplayOracle.from_start(start)
    for chunk in (1, 11):
        gpu.step(chunk)
        replay.step(chunk)
        assert gpu.n_labels == replay.n_labels
        labels, want = gpu.labels(), replay.labels()
        assert np.array_equal(labels, want), f"{int((labels != want).sum())} sites differ after {gpu.mcs} MCS"
        assert np.array_equal(gpu.volumes(), replay.volumes())
        assert np.array_equal(gpu.surfaces(), replay.surfaces())
        assert np.array_equal(gpu.cell_types(), replay.cell_types())
        for k in range(len(start.model.species)):
            assert np.array_equal(gpu.field(k).astype(np.float32), replay.field(k))
    assert replay.accepted > 0
    if name == "division-volume":
        assert gpu.n_labels > int(start.labels.max()) + 1, "no cell divided"
    gpu.close()
