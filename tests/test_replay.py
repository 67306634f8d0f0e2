"""The host replay of the device schedule, on the CPU.

The replay is the device algorithm written serially; these tests hold it to
the reference's statistics before any device runs it, and check the pieces
the device shares with it: the counter hash, the Metropolis exp and the
bookkeeping.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import pieces, recount_volumes, sheet_model, spread, tiled, with_species
from oracle import replay as R
from oracle.serial import SerialOracle

M64 = 2**64 - 1


def _mix(z):
    z = (z + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def test_the_hash_is_the_reference_formula():
    # glazier-cuda/src/lib.rs:33-46
    for seed, site, step, colour, index in [(1, 0, 0, 0, 0), (7, 123456, 99, 3, 1), (2**63 + 5, 2**31, 1, 7, 1)]:
        want = _mix(seed ^ ((0xD1B54A32D192ED03 * site) & M64) ^ ((0xA0761D6478BD642F * step) & M64)
                    ^ ((0xE7037ED1A0B428DB * (4 * colour + index)) & M64))
        assert R.draw(seed, site, step, colour, index) == want


def test_the_metropolis_exp_is_within_two_ulps_of_libm():
    xs = np.concatenate([-np.geomspace(1e-8, 87.0, 20000).astype(np.float32), np.float32([0.0, -1.0, -0.5])])
    worst = 0
    for x in xs:
        got = np.float32(R.expf(float(x)))
        want = np.float32(math.exp(float(x)))
        ulps = abs(int(got.view(np.int32)) - int(want.view(np.int32)))
        worst = max(worst, ulps)
    assert worst <= 2, worst
    assert R.expf(-100.0) == 0.0 and R.expf(0.0) == 1.0


def _replay(model, start=None, steps=0, fields=None):
    start = start or tiled(model)
    r = R.ReplayOracle.from_start(start, fields)
    if steps:
        r.step(steps)
    return r


def test_the_replay_keeps_its_counters_with_the_lattice():
    m = sheet_model(seed=3, target_surface=34.0, lambda_surface=0.1)
    r = _replay(m, steps=60)
    labels = r.labels()
    assert np.array_equal(r.volumes(), recount_volumes(labels, r.n_labels))
    check = SerialOracle(m, labels=labels, cell_type=r.cell_types())
    assert np.array_equal(r.surfaces(), check.recounted_surfaces())
    by_colour = r.volumes_by_colour()
    assert np.array_equal(by_colour.sum(axis=1)[1:], r.volumes()[1:].astype(np.int64))


def test_the_replay_agrees_with_the_serial_engine_in_distribution():
    # gpu_matches_cpu.rs:48-92 on the replay: same cells, same mean, spread within a quarter
    m = sheet_model(seed=1)
    cpu = SerialOracle.from_start(tiled(m))
    cpu.step(200)
    r = _replay(m, steps=200)
    vc, vr = cpu.volumes()[1:], r.volumes()[1:]
    assert vc.size == vr.size
    assert abs(vc.mean() - vr.mean()) < 1e-9
    sc, sr = spread(vc, 64.0), spread(vr, 64.0)
    assert abs(sc - sr) / max(sc, sr) < 0.25, (sc, sr)


def test_the_replay_keeps_every_cell():
    # gpu_matches_cpu.rs:120-138
    r = _replay(sheet_model(seed=7), steps=300)
    v = r.volumes()
    assert v.size - 1 == 64 and (v[1:] >= 1).all()


def test_the_replay_stretches_cells_like_the_serial_engine():
    # gpu_matches_cpu.rs:155-203
    stated = sheet_model(seed=41, target_length=24.0, lambda_length=1.0)
    cpu = SerialOracle.from_start(tiled(stated))
    cpu.step(200)
    r = _replay(stated, steps=200)
    loose = SerialOracle.from_start(tiled(sheet_model(seed=41)))
    loose.step(200)
    free = loose.lengths()[1:].mean()
    serial = cpu.lengths()[1:].mean()
    device = r.lengths()[1:].mean()
    assert serial > free and device > free
    assert abs(serial - device) / max(serial, device) < 0.15, (serial, device)


def test_the_replay_keeps_connected_cells_whole():
    # glazier-tests/tests/connectivity.rs:115-155
    loose = _replay(sheet_model(seed=23, contact=(0, 4, 4, 4), lambda_volume=1.0, temperature=40.0), steps=200)
    whole = _replay(sheet_model(seed=23, contact=(0, 4, 4, 4), lambda_volume=1.0, temperature=40.0,
                                connected=True), steps=200)
    assert pieces(loose.labels(), 64, 64) > 64
    assert pieces(whole.labels(), 64, 64) == 64


def test_the_replay_kills_at_the_stated_rate():
    # gpu_population.rs:119-153
    m = sheet_model(seed=9, death_rate=0.01)
    start = tiled(m, 8, 10, 10)  # clamped to the 8 by 8 that fit, as in the reference test
    started = start.n_cells
    r = R.ReplayOracle.from_start(start)
    r.step(80)
    live = int((r.volumes()[1:] > 0).sum())
    survival = 0.99**80
    expected, sd = started * survival, math.sqrt(started * survival * (1 - survival))
    assert abs(live - expected) < 3 * sd


def test_the_replay_divides_and_conserves_sites():
    # gpu_population.rs:101-117
    m = sheet_model(seed=7, division_volume=40.0, target_volume=100.0)
    r = R.ReplayOracle.from_start(tiled(m, 8, 4, 4))
    r.step(1)
    v = r.volumes()
    assert int((v[1:] > 0).sum()) > 16
    assert int(v[1:].sum()) == int((r.labels() != 0).sum())
    assert np.array_equal(v, recount_volumes(r.labels(), r.n_labels))


def test_the_replay_field_matches_the_f64_field_step():
    # fields to 1e-5 relative of the f64 serial step on the same labels
    m = with_species(sheet_model(seed=11), [("IFNg", 0.4, 0.01, 0.0)], [[0.0], [0.2]], [[0.0], [0.01]],
                     [[0.0], [0.0]])
    m.temperature = 1e-6  # freeze the lattice so both see the same owners
    m.types[1].lambda_volume = 0.0
    start = tiled(m)
    r = R.ReplayOracle.from_start(start)
    cpu = SerialOracle.from_start(start)
    r.step(30)
    cpu.step(30)
    assert np.array_equal(r.labels(), cpu.labels())
    f32, f64 = r.field(0).astype(np.float64), cpu.field(0)
    assert np.max(np.abs(f32 - f64) / np.maximum(np.abs(f64), 1e-30)) < 1e-5


def test_the_infection_rule_spreads_and_only_from_healthy_cells():
    """The infection rule (an extension, no reference counterpart): over 40
    MCS of the two-field infection model the centre cell's virus infects its
    neighbours; without the rule the healthy cells stay healthy; a threshold
    no cell can reach switches none; a bad rule is refused."""
    from glazier_b200.workloads import INFECTION_RULE, infection_start

    def run(rule, steps=40):
        st = infection_start()
        r = R.ReplayOracle.from_start(st)
        if rule is not None:
            r.set_infection(*rule)
        r.step(steps)
        return st, r.cell_types(), r.volumes()

    st, types, vols = run(INFECTION_RULE)
    alive = vols > 0
    infected = int(((types == 2) & alive).sum())
    assert infected > 3
    # immune cells (type 3) never switch
    assert np.array_equal(types[257:289], st.cell_type[257:289])
    _, plain, _ = run(None)
    assert int((plain[1:257] == 2).sum()) == 1
    _, high, _ = run((0, 1, 2, 1e9))
    assert np.array_equal(high[:257], plain[:257])
    r = R.ReplayOracle.from_start(infection_start())
    with pytest.raises(ValueError):
        r.set_infection(0, 1, 1, 5.0)
    with pytest.raises(ValueError):
        r.set_infection(2, 1, 2, 5.0)
    with pytest.raises(ValueError):
        r.set_infection(0, 1, 2, 1e12)  # past the fixed-point range


def test_the_motility_log_is_within_two_ulps_of_libm():
    """The motility term's own log (the atanh series) against the C library's,
    over the activity values a run can hold and a spread of positive floats."""
    import ctypes as C

    L = R.lib()
    L.rp_logf.argtypes = [C.c_float]
    L.rp_logf.restype = C.c_float
    xs = np.concatenate([np.arange(1, 101, dtype=np.float32),
                         np.float32(2.0) ** np.random.default_rng(5).uniform(-30, 30, 4000).astype(np.float32),
                         np.float32([0.5, 0.75, 1.41421, 1.41422, 1e-40, 3.4e38])])
    for x in xs:
        got = np.float32(L.rp_logf(float(x)))
        want = np.float32(math.log(float(x)))
        ulp = np.spacing(np.abs(want)) if want != 0 else np.float32(1e-45)
        assert abs(float(got) - float(want)) <= 2 * float(ulp) + 1e-7 * (abs(float(want)) < 1e-3), (x, got, want)


@pytest.mark.parametrize("name", ["nematic", "nematic-volume", "motility", "drift"])
def test_each_extra_term_changes_the_run(name):
    """On the replay, each term's parity case lands elsewhere without the
    term, so a device that skipped the term could not match it."""
    import copy

    from test_gpu_parity import CASES

    made, steps = CASES[name]()
    start = made
    plain = copy.deepcopy(start)
    for t in plain.model.types:
        t.lambda_nematic = 0.0
        t.lambda_activity = 0.0
        t.external = (0.0, 0.0, 0.0)
    a, b = R.ReplayOracle.from_start(start), R.ReplayOracle.from_start(plain)
    a.step(steps)
    b.step(steps)
    assert not np.array_equal(a.labels(), b.labels())
