"""The reference's own device tests, run on the B200 engine.

Each test restates one of glazier-tests' GPU tests (file:line given) with the
same model, the same steps and the same band, the serial oracle standing in
for the reference's serial engine.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import pieces, recount_volumes, sheet_model, spread, tiled, with_species
from glazier_b200.blueprint import Start
from oracle.serial import SerialOracle

pytestmark = pytest.mark.gpu


def _serial(model, steps, start=None):
    o = SerialOracle.from_start(start or tiled(model))
    o.step(steps)
    return o


def test_the_gpu_reproduces_the_serial_run_in_distribution(device):
    # gpu_matches_cpu.rs:48-92
    m = sheet_model(seed=1)
    cpu = _serial(m, 200)
    gpu = device.GpuSimulation.from_start(tiled(m))
    gpu.step(200)
    vc, vg = cpu.volumes()[1:], gpu.volumes()
    assert vc.size == vg.size - 1, "cell counts differ"
    assert abs(vc.mean() - vg[1:].mean()) < 1e-9
    sc, sg = spread(vc, 64.0), spread(vg[1:], 64.0)
    assert abs(sc - sg) / max(sc, sg) < 0.25, (sc, sg)
    assert np.array_equal(recount_volumes(gpu.labels(), gpu.n_labels), vg), "the device volume counter drifted"


def test_the_device_surface_counter_matches_the_lattice_it_wrote(device):
    # gpu_matches_cpu.rs:103-118
    m = sheet_model(seed=3, target_surface=34.0, lambda_surface=0.1)
    gpu = device.GpuSimulation.from_start(tiled(m))
    gpu.step(150)
    check = SerialOracle(m, labels=gpu.labels(), cell_type=gpu.cell_types())
    assert np.array_equal(gpu.surfaces(), check.recounted_surfaces())


def test_a_device_run_conserves_its_cells(device):
    # gpu_matches_cpu.rs:120-138
    gpu = device.GpuSimulation.from_start(tiled(sheet_model(seed=7)))
    gpu.step(300)
    v = gpu.volumes()
    assert v.size - 1 == 64 and (v[1:] >= 1).all()


def test_the_device_refuses_a_lattice_it_cannot_colour(device):
    # gpu_matches_cpu.rs:140-149
    m = sheet_model(width=33, height=32)
    start = Start.tiled(m, 8)
    with pytest.raises(device.GpuError, match="even sides"):
        device.GpuSimulation.from_start(start)


def test_the_device_stretches_cells_the_way_the_serial_engine_does(device):
    # gpu_matches_cpu.rs:155-203
    stated = sheet_model(seed=41, target_length=24.0, lambda_length=1.0)
    cpu = _serial(stated, 200)
    gpu = device.GpuSimulation.from_start(tiled(stated))
    gpu.step(200)
    on_device = SerialOracle(stated, labels=gpu.labels(), cell_type=gpu.cell_types())
    free = _serial(sheet_model(seed=41), 200).lengths()[1:].mean()
    serial = cpu.lengths()[1:].mean()
    dev = on_device.lengths()[1:].mean()
    assert serial > free and dev > free
    assert abs(serial - dev) / max(serial, dev) < 0.15, (serial, dev)


def _secreting(seed):
    return with_species(sheet_model(seed=seed), [("IFNg", 0.4, 0.01, 0.0)], [[0.0], [0.2]], [[0.0], [0.01]],
                        [[0.0], [0.0]])


def test_the_device_solves_a_field_the_way_the_serial_engine_does(device):
    # gpu_matches_cpu.rs:230-257
    cpu = _serial(_secreting(11), 60)
    gpu = device.GpuSimulation.from_start(tiled(_secreting(11)))
    gpu.step(60)
    dev, ser = gpu.field(0).sum(), cpu.field(0).sum()
    assert dev > 0
    assert abs(dev - ser) / max(dev, ser) < 0.02


def test_a_device_field_stays_where_it_started_without_sources(device):
    # gpu_matches_cpu.rs:259-285
    m = _secreting(12)
    m.secretion = [[0.0], [0.0]]
    m.uptake = [[0.0], [0.0]]
    m.species[0].decay = 0.0
    m.species[0].initial = 2.0
    gpu = device.GpuSimulation.from_start(tiled(m))
    gpu.step(40)
    total = gpu.field(0).sum()
    assert abs(total - 2.0 * 4096) / (2.0 * 4096) < 1e-4


def test_the_device_climbs_a_gradient(device):
    # gpu_matches_cpu.rs:287-336
    m = with_species(sheet_model(seed=21), [("attractant", 0.0, 0.0, 0.0)], [[0.0], [0.0]], [[0.0], [0.0]],
                     [[0.0], [4.0]])
    ys, xs = np.divmod(np.arange(64 * 64), 64)
    labels = ((xs >= 24) & (xs < 32) & (ys >= 24) & (ys < 32)).astype(np.uint32)
    start = Start(m, labels, np.array([0, 1], dtype=np.uint8))
    centre = lambda lab: xs[lab == 1].mean()  # noqa: E731
    gpu = device.GpuSimulation.from_start(start, xs.astype(np.float64)[None, :])
    gpu.step(300)
    assert centre(gpu.labels()) - centre(labels) > 3.0


def test_the_device_runs_a_volume(device):
    # gpu_matches_cpu.rs:338-392
    m = sheet_model(width=32, height=32, depth=32, seed=31, target_volume=512.0)
    cpu = _serial(m, 40)
    gpu = device.GpuSimulation.from_start(tiled(m))
    gpu.step(40)
    dv = gpu.volumes()
    assert dv.size == cpu.n_labels
    assert int(dv[1:].sum()) == int(cpu.volumes()[1:].sum())
    assert np.array_equal(dv[1:], recount_volumes(gpu.labels(), dv.size)[1:])
    sc, sg = spread(cpu.volumes()[1:], 512.0), spread(dv[1:], 512.0)
    assert abs(sc - sg) / max(sc, sg) < 0.3, (sc, sg)


def _pop_model(division_volume, death_rate, target_volume, seed):
    return sheet_model(seed=seed, division_volume=division_volume, death_rate=death_rate, target_volume=target_volume)


def _live(v):
    return int((np.asarray(v)[1:] > 0).sum())


def test_the_device_kills_cells_at_the_stated_rate(device):
    # gpu_population.rs:45-59
    start = tiled(_pop_model(0.0, 0.02, 64.0, 5), 8, 6, 6)
    gpu = device.GpuSimulation.from_start(start)
    gpu.step(50)
    expected = start.n_cells * 0.98**50
    assert abs(_live(gpu.volumes()) - expected) < 0.35 * start.n_cells


def test_a_dead_cell_leaves_medium_on_the_device(device):
    # gpu_population.rs:61-78
    gpu = device.GpuSimulation.from_start(tiled(_pop_model(0.0, 1.0, 64.0, 6), 8, 2, 2))
    gpu.step(1)
    assert _live(gpu.volumes()) == 0
    assert (gpu.labels() == 0).all()


def test_the_device_divides_and_conserves_the_sites(device):
    # gpu_population.rs:80-99
    start = tiled(_pop_model(40.0, 0.0, 100.0, 7), 8, 4, 4)
    gpu = device.GpuSimulation.from_start(start)
    gpu.step(1)
    v = gpu.volumes()
    assert _live(v) > start.n_cells
    assert int(v[1:].sum()) == int((gpu.labels() != 0).sum())


def test_the_device_counters_match_the_lattice_they_wrote(device):
    # gpu_population.rs:101-117
    gpu = device.GpuSimulation.from_start(tiled(_pop_model(72.0, 0.005, 100.0, 8), 6, 6, 6))
    gpu.step(120)
    v = gpu.volumes()
    assert np.array_equal(v[1:], recount_volumes(gpu.labels(), v.size)[1:])


def test_both_engines_lose_cells_at_the_rate_the_description_states(device):
    # gpu_population.rs:119-153
    steps, rate = 80, 0.01
    start = tiled(_pop_model(0.0, rate, 64.0, 9), 8, 10, 10)
    cpu = SerialOracle.from_start(start)
    cpu.step(steps)
    gpu = device.GpuSimulation.from_start(start)
    gpu.step(steps)
    survival = (1 - rate) ** steps
    expected = start.n_cells * survival
    sd = math.sqrt(start.n_cells * survival * (1 - survival))
    for name, left in (("serial", _live(cpu.volumes())), ("device", _live(gpu.volumes()))):
        assert abs(left - expected) < 3 * sd, (name, left, expected, sd)


def _conn_model(connected, temperature):
    return sheet_model(seed=23, contact=(0, 4, 4, 4), lambda_volume=1.0, temperature=temperature,
                       connected=connected)


def test_the_device_keeps_cells_whole_where_nothing_else_does(device):
    # glazier-tests/tests/connectivity.rs:120-155
    loose = device.GpuSimulation.from_start(tiled(_conn_model(False, 40.0)))
    whole = device.GpuSimulation.from_start(tiled(_conn_model(True, 40.0)))
    loose.step(200)
    whole.step(200)
    assert pieces(loose.labels(), 64, 64) > 64
    assert pieces(whole.labels(), 64, 64) == 64


def test_the_device_and_the_serial_engine_agree_on_a_constrained_sheet(device):
    # glazier-tests/tests/connectivity.rs:157-189
    m = _conn_model(True, 20.0)
    cpu = _serial(m, 150)
    gpu = device.GpuSimulation.from_start(tiled(m))
    gpu.step(150)
    dv = gpu.volumes()
    assert int(dv[1:].sum()) == int(cpu.volumes()[1:].sum())
    sc, sg = spread(cpu.volumes()[1:], 64.0), spread(dv[1:], 64.0)
    assert abs(sc - sg) / max(sc, sg) < 0.3, (sc, sg)


def _lone_cell(model):
    """motility.rs:35-45: one 8 x 8 cell at x, y in [44, 52) on an empty 96 x 96
    lattice."""
    labels = np.zeros((model.height, model.width), dtype=np.uint32)
    labels[44:52, 44:52] = 1
    return Start(model, labels.reshape(-1), np.array([1, 1], dtype=np.uint8))


def _motility_model(max_activity, lambda_activity, external, connected):
    # motility.rs:10-32
    from glazier_b200.blueprint import CellType, Model

    return Model(width=96, height=96, contact=[0.0, 16.0, 16.0, 8.0],
                 types=[CellType(), CellType(target_volume=64.0, lambda_volume=2.0, connected=connected,
                                             max_activity=max_activity, lambda_activity=lambda_activity,
                                             external=tuple(external))],
                 temperature=10.0, neighbour_order=2, seed=29)


def _centroid(labels, width):
    ys, xs = np.divmod(np.flatnonzero(np.asarray(labels) == 1), width)
    return xs.mean(), ys.mean()


@pytest.mark.parametrize("sign", [1.0, -1.0])
def test_the_device_drifts_a_cell_the_way_it_points(device, sign):
    # motility.rs:199-215 (device) and 107-132 (the reversed drift)
    st = _lone_cell(_motility_model(0.0, 0.0, (3.0 * sign, 0.0, 0.0), True))
    x0, y0 = _centroid(st.labels, 96)
    gpu = device.GpuSimulation.from_start(st)
    gpu.step(300)
    x1, y1 = _centroid(gpu.labels(), 96)
    gpu.close()
    assert sign * (x1 - x0) > 5.0, f"the cell moved {x1 - x0} along x"
    assert abs(y1 - y0) < 4.0, f"the cell wandered {y1 - y0} across the drift"


def test_the_device_makes_a_cell_travel_on_its_memory(device):
    # motility.rs:181-197: over 400 MCS a cell with a memory (max 20, lambda 60)
    # travels more than three times as far as a plain one
    def travelled(max_activity, lambda_activity):
        st = _lone_cell(_motility_model(max_activity, lambda_activity, (0.0, 0.0, 0.0), False))
        x0, y0 = _centroid(st.labels, 96)
        gpu = device.GpuSimulation.from_start(st)
        gpu.step(400)
        x1, y1 = _centroid(gpu.labels(), 96)
        gpu.close()
        return math.hypot(x1 - x0, y1 - y0)

    still, motile = travelled(0.0, 0.0), travelled(20.0, 60.0)
    assert motile > 3.0 * still, f"a motile cell went {motile} on the device against {still} for a plain one"


def _nematic_model(lambda_nematic, angle):
    # gpu_nematic.rs:16-36
    from glazier_b200.blueprint import CellType, Model

    m = Model(width=64, height=64, contact=[0.0, 16.0, 16.0, 8.0],
              types=[CellType(), CellType(target_volume=64.0, lambda_volume=2.0, lambda_nematic=lambda_nematic)],
              temperature=10.0, neighbour_order=2, seed=7)
    m.nematic = np.tile([math.cos(2 * angle), math.sin(2 * angle)], (64 * 64, 1))
    return m


def _order(labels, width, height):
    """gpu_nematic.rs:38-58: the nematic order |<exp(2 i theta)>| of the cells'
    long axes and their mean director, over cells of eight sites or more."""
    labels = np.asarray(labels).reshape(height, width)
    c = s = n = 0.0
    for l in np.unique(labels[labels > 0]):
        ys, xs = np.nonzero(labels == l)
        if xs.size < 8:
            continue
        # the cell's frame: minimum image about its first site
        x0, y0 = xs[0], ys[0]
        ux = (xs - x0 + width // 2) % width - width // 2
        uy = (ys - y0 + height // 2) % height - height // 2
        cxx, cyy = ux.var(), uy.var()
        cxy = (ux * uy).mean() - ux.mean() * uy.mean()
        trace = cxx + cyy
        if trace <= 1e-12:
            continue
        a0, a1 = (cxx - cyy) / trace, 2 * cxy / trace
        norm = math.hypot(a0, a1)
        if norm < 1e-9:
            continue
        c += a0 / norm
        s += a1 / norm
        n += 1
    return math.hypot(c, s) / n, 0.5 * math.atan2(s, c)


def test_the_device_aligns_cells_along_the_field_as_the_serial_engine_does(device):
    # gpu_nematic.rs:74-105
    angle, steps = 0.6, 400
    coupled = _nematic_model(6.0, angle)
    gpu = device.GpuSimulation.from_start(tiled(coupled, 8))
    gpu.step(steps)
    s_gpu, director = _order(gpu.labels(), 64, 64)
    gpu.close()
    s_cpu, _ = _order(_serial(coupled, steps, tiled(coupled, 8)).labels(), 64, 64)
    off = min(abs(director - angle), math.pi - abs(director - angle))
    assert s_gpu > 0.7, f"device order {s_gpu}"
    assert off < 0.15, f"device director {director} against the field's {angle}"
    assert abs(s_gpu - s_cpu) < 0.15, f"device {s_gpu} against serial {s_cpu}"
    blind = _nematic_model(0.0, angle)
    gpu = device.GpuSimulation.from_start(tiled(blind, 8))
    gpu.step(steps)
    s_blind, _ = _order(gpu.labels(), 64, 64)
    gpu.close()
    assert s_blind < 0.4, f"uncoupled device order {s_blind}"


def test_a_replaced_field_turns_the_cells_on_the_device(device):
    # gpu_nematic.rs:107-131
    from glazier_b200.engine import GpuError

    first = 0.2
    second = first + math.pi / 2
    coupled = _nematic_model(6.0, first)
    gpu = device.GpuSimulation.from_start(tiled(coupled, 8))
    gpu.step(400)
    _, before = _order(gpu.labels(), 64, 64)
    turned = np.tile([math.cos(2 * second), math.sin(2 * second)], (64 * 64, 1))
    gpu.set_nematic_field(turned)
    gpu.step(800)
    s_after, after = _order(gpu.labels(), 64, 64)

    def off(d, a):
        return min(abs(d - a), math.pi - abs(d - a))

    assert off(before, first) < 0.15, f"before {before}"
    assert s_after > 0.7, f"order after the turn {s_after}"
    assert off(after, second) < 0.15, f"after {after} against {second}"
    with pytest.raises(GpuError):
        gpu.set_nematic_field(turned[1:])
    gpu.close()
