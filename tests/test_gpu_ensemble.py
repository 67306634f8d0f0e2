"""The batched ensemble against the plain engine, replica by replica.

Every replica of an ensemble must land on exactly the lattice, volumes and
surfaces a GpuSimulation of the same start lands on, whatever schedule the
ensemble runs (replica order, persistent grid, tensor-copy windows on or off)
and after the autotuner has timed its candidates on a snapshot.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import sheet_model, tiled
from glazier_b200.blueprint import Start
from glazier_b200.workloads import ensemble_starts, monolayer
from oracle.replay import ReplayOracle

pytestmark = pytest.mark.gpu


def _starts():
    # uneven sides and rectangles, each with its own parameters and seed
    out = []
    for i, (w, h) in enumerate([(64, 64), (160, 96), (128, 128), (96, 200), (288, 64), (72, 80)]):
        st = monolayer(8, contact=6.0 + i, lambda_volume=0.5 + 0.25 * i, temperature=6.0 + 2 * i, seed=100 + i,
                       lambda_surface=0.1 * (i % 2), target_surface=92.0)
        st.model.width, st.model.height = w, h
        out.append(Start.tiled(st.model, 8))
    return out


def _plain(device, start, steps):
    sim = device.GpuSimulation.from_start(start)
    sim.step(steps)
    return sim.labels(), sim.volumes(), sim.surfaces()


@pytest.mark.parametrize("tma", ["1", "0"])
def test_each_replica_matches_its_own_plain_run(device, tma, monkeypatch):
    from glazier_b200.ensemble import Ensemble

    monkeypatch.setenv("GLAZIER_SWEEP_TMA", tma)
    starts = _starts()
    ens = Ensemble(starts)
    ens.step(4)
    ens.step(8)
    assert ens.mcs == 12
    for i, st in enumerate(starts):
        labels, volumes, surfaces = _plain(device, st, 12)
        assert np.array_equal(ens.labels(i), labels), f"replica {i}"
        assert np.array_equal(ens.volumes(i), volumes), f"replica {i}"
        assert np.array_equal(ens.surfaces(i), surfaces), f"replica {i}"
    ens.close()


def test_a_replica_matches_the_host_replay(device):
    from glazier_b200.ensemble import Ensemble

    starts = _starts()
    ens = Ensemble(starts)
    ens.step(6)
    replay = ReplayOracle.from_start(starts[1])
    replay.step(6)
    assert np.array_equal(ens.labels(1), replay.labels())
    assert np.array_equal(ens.volumes(1), replay.volumes())


# schedule bit 0: replica order; bits 1-2: tile shape (0 windowed, 1-3 direct
# blocks of 32 x 8, 16 x 16, 64 x 4 targets); bit 3: a step's passes in one
# cooperative launch
@pytest.mark.parametrize("schedule,ctas", [(0, 0), (1, 0), (0, 3), (1, 7), (2, 0), (3, 0), (4, 0), (7, 0), (10, 0),
                                           (13, 0), (15, 0)])
def test_the_schedule_changes_only_the_time(device, schedule, ctas):
    from glazier_b200.ensemble import Ensemble

    starts = _starts()
    ref = Ensemble(starts)
    ref.step(5)
    ens = Ensemble(starts)
    ens.set_schedule(schedule, ctas)
    ens.step(5)
    for i in range(len(starts)):
        assert np.array_equal(ens.labels(i), ref.labels(i)), f"replica {i}"


def test_autotuning_leaves_the_run_where_it_was(device):
    from glazier_b200.ensemble import Ensemble

    starts = ensemble_starts(12, low=64, high=256)
    ref = Ensemble(starts)
    ref.step(3)
    ens = Ensemble(starts)
    ens.step(1)
    choice = ens.autotune(2)
    assert choice >= 0
    assert ens.mcs == 1
    ens.step(2)
    for i in range(len(starts)):
        assert np.array_equal(ens.labels(i), ref.labels(i)), f"replica {i}"
        assert np.array_equal(ens.volumes(i), ref.volumes(i)), f"replica {i}"


def _plain_with_rule(device, start, steps, rule):
    sim = device.GpuSimulation.from_start(start)
    if rule is not None:
        sim.set_infection(*rule)
    sim.step(steps)
    out = sim.labels(), sim.volumes(), sim.surfaces(), sim.n_labels
    sim.close()
    return out


def test_replicas_with_more_terms_run_beside_the_batch_and_match_their_plain_runs(device):
    # three batched monolayers, an infection model (fields, division, death,
    # length, chemotaxis, connectivity) and a dividing sheet that run as their
    # own engines at the same time
    from glazier_b200.ensemble import Ensemble
    from glazier_b200.workloads import INFECTION_RULE, infection_start

    # 36-site cells with room around them, growing toward 100 sites and
    # dividing at 48 (the parity suite's population sheet)
    dividing = tiled(sheet_model(seed=77, division_volume=48.0, death_rate=0.01, target_volume=100.0), 6, 6, 6)
    starts = _starts()[:3] + [infection_start(seed=5, size=128, grid=6, immune=4), dividing]
    rules = [None, None, None, INFECTION_RULE, None]
    ens = Ensemble(starts)
    ens.set_infection(3, *INFECTION_RULE)
    ens.autotune(2)
    ens.step(4)
    ens.step(26)
    assert ens.mcs == 30
    for i, (st, rule) in enumerate(zip(starts, rules)):
        labels, volumes, surfaces, n_labels = _plain_with_rule(device, st, 30, rule)
        assert ens.n_labels(i) == n_labels, f"replica {i}"
        assert np.array_equal(ens.labels(i), labels), f"replica {i}"
        assert np.array_equal(ens.volumes(i), volumes), f"replica {i}"
        assert np.array_equal(ens.surfaces(i), surfaces), f"replica {i}"
    assert ens.n_labels(4) > starts[4].cell_type.size  # the sheet divided
    ens.close()


def test_an_ensemble_of_engine_replicas_alone_runs(device):
    from glazier_b200.ensemble import Ensemble
    from glazier_b200.workloads import INFECTION_RULE, infection_start

    starts = [infection_start(seed=s, size=96, grid=4, immune=3) for s in (1, 2)]
    ens = Ensemble(starts)
    for i in range(2):
        ens.set_infection(i, *INFECTION_RULE)
    assert ens.autotune(2) == 0
    ens.step(10)
    assert ens.mcs == 10
    for i, st in enumerate(starts):
        labels, volumes, _, _ = _plain_with_rule(device, st, 10, INFECTION_RULE)
        assert np.array_equal(ens.labels(i), labels)
        assert np.array_equal(ens.volumes(i), volumes)
    ens.close()


def test_the_ensemble_refuses_what_it_does_not_run(device):
    from glazier_b200.engine import GpuError
    from glazier_b200.ensemble import Ensemble
    from glazier_b200.workloads import INFECTION_RULE

    ens = Ensemble(_starts()[:2])
    with pytest.raises(GpuError, match="batched and has no fields"):
        ens.set_infection(0, *INFECTION_RULE)
    with pytest.raises(GpuError, match="no such replica"):
        ens.labels(2)
    ens.close()
    odd = monolayer(64)
    odd.model.width = 66
    odd = Start.tiled(odd.model, 8)
    odd.model.width = 65
    with pytest.raises(GpuError):
        Ensemble([odd])
