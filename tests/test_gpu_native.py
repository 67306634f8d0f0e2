"""The ``_native`` entry points on the device engine.

Restates glazier's tests/test_native_engine.py (the run shape and the
volume sum) and drives ``GpuSession`` the way glazier-py exposes it.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from glazier_b200 import native

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "serial_reference.json").read_text())
MONOLAYER = GOLDEN["parse"]["monolayer.json"]["text"]


def test_a_short_run_returns_a_lattice_of_the_stated_shape(device):
    # tests/test_native_engine.py:27-37
    labels, width, height, depth = native.run(MONOLAYER, 5)
    field = np.asarray(labels, dtype=np.uint32).reshape(depth, height, width)
    parsed = native.parse(MONOLAYER)
    assert field.shape == (parsed["depth"], parsed["height"], parsed["width"])
    side, nx, ny, nz = parsed["initial"]
    assert np.unique(field[field > 0]).size == nx * ny * nz


def test_volumes_come_back_per_cell(device):
    # tests/test_native_engine.py:40-48
    volumes = native.run_volumes(MONOLAYER, 5)
    parsed = native.parse(MONOLAYER)
    side, nx, ny, nz = parsed["initial"]
    assert len(volumes) == nx * ny * nz + 1
    assert sum(volumes[1:]) == parsed["width"] * parsed["height"] * parsed["depth"]


def test_a_session_keeps_the_run_on_the_device(device):
    # glazier-py/src/lib.rs:184-241
    session = native.GpuSession(MONOLAYER)
    assert session.mcs == 0
    session.step(3)
    session.step(2)
    assert session.mcs == 5
    labels = session.labels()
    assert len(labels) == 128 * 128
    with pytest.raises(ValueError, match="expected"):
        session.set_nematic_field([0.0, 0.0])
    with pytest.raises(ValueError, match="no nematic coupling"):
        session.set_nematic_field([0.0] * (2 * 128 * 128))


def test_every_reference_blueprint_the_engine_runs_starts_and_steps(device):
    ran = 0
    for name, entry in GOLDEN["parse"].items():
        raw = json.loads(entry["text"])
        if raw.get("nematic_field") or raw["initial"].get("labels"):
            continue
        # motility and drift blueprints (immune-motile.json) run like the rest
        session = native.GpuSession(entry["text"])
        session.step(2)
        ran += 1
    assert ran >= 10


def test_a_session_applies_the_descriptions_infection_rule(device):
    """A description with the `infection` extension key: the session's engine
    switches healthy cells to infected as their virus uptake passes the
    threshold; the same description without the key switches none."""
    text = {
        "name": "infection rule", "width": 64, "height": 64,
        "types": [{"name": "Healthy", "target_volume": 64, "lambda_volume": 2, "uptake": {"virus": 0.05}},
                  {"name": "Infected", "target_volume": 64, "lambda_volume": 2, "secretion": {"virus": 2.0}}],
        "fields": [{"name": "virus", "diffusion": 0.2, "decay": 0.01}],
        "contact": [0, 16, 16, 16, 10, 10, 16, 10, 10], "temperature": 10, "neighbour_order": 2, "seed": 3,
        "steps": 30, "dump_every": 0, "initial": {"side": 8, "nx": 8, "ny": 8, "fractions": {"Infected": 0.05}},
        "units": {"micron_per_site": 1, "minute_per_step": 1},
        "infection": {"field": "virus", "from": "Healthy", "to": "Infected", "threshold": 3},
    }
    counts = []
    for with_rule in (True, False):
        spec = dict(text)
        if not with_rule:
            del spec["infection"]
        session = native.GpuSession(json.dumps(spec))
        before = int((session.simulation.cell_types()[1:] == 2).sum())
        session.step(30)
        counts.append((before, int((session.simulation.cell_types()[1:] == 2).sum())))
        session.simulation.close()
    (before, after), (plain_before, plain_after) = counts
    assert before == plain_before > 0
    assert after > before
    assert plain_after == plain_before
