"""Generate the golden fixtures that pin the serial oracle to the reference.

Runs glazier's own compiled module (``python/glazier/_native.abi3.so`` in
the reference checkout, run as a program and never read) on the reference's
blueprints and on a few synthetic descriptions that switch on the terms the
blueprints leave to a second cell type (length, chemotaxis, division,
death, 3D surface). Writes ``serial_reference.json``: per case the
description text, the step count, a SHA-256 of the final lattice and the
per-label volumes, plus the ``parse`` reading of every blueprint.

The shipped module is an older build than the reference source: it starts
every cell as the first type (it ignores ``initial.fractions``) and ignores
``connected``, ``max_activity``, ``external`` and ``lambda_nematic``. The
cases below stay inside what it runs, and the tests seed the oracle the same
way.

Usage (in a checkout that has the reference, never on the GPU box):
    python tests/golden/make_golden.py /path/to/glazier
"""

from __future__ import annotations

import hashlib
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

SKIP = {"monolayer-nematic.json"}  # the shipped build ignores lambda_nematic

SYNTHETIC = {
    "length-64": {
        "name": "a sheet stretched by the length term",
        "width": 64, "height": 64,
        "types": [{"name": "Cell", "target_volume": 64.0, "lambda_volume": 2.0,
                   "target_length": 24.0, "lambda_length": 1.0}],
        "contact": [0.0, 16.0, 16.0, 8.0],
        "temperature": 10.0, "neighbour_order": 2, "seed": 41, "steps": 12, "dump_every": 0,
        "initial": {"side": 8, "nx": 8, "ny": 8},
        "units": {"micron_per_site": 1.0, "minute_per_step": 1.0},
    },
    "chemotaxis-division-64": {
        "name": "cells that secrete, climb, divide and die",
        "width": 64, "height": 64,
        "types": [{"name": "Cell", "target_volume": 100.0, "lambda_volume": 2.0,
                   "division_volume": 80.0, "death_rate": 0.01,
                   "secretion": {"attractant": 0.1}, "uptake": {"attractant": 0.02},
                   "chemotaxis": {"attractant": 5.0}}],
        "fields": [{"name": "attractant", "diffusion": 0.2, "decay": 0.01, "initial": 0.5}],
        "contact": [0.0, 16.0, 16.0, 8.0],
        "temperature": 10.0, "neighbour_order": 2, "seed": 7, "steps": 12, "dump_every": 0,
        "initial": {"side": 8, "nx": 6, "ny": 6},
        "units": {"micron_per_site": 1.0, "minute_per_step": 1.0},
    },
    "surface-3d-32": {
        "name": "a block of cubes with a surface term",
        "width": 32, "height": 32, "depth": 32,
        "types": [{"name": "Cell", "target_volume": 512.0, "lambda_volume": 1.0,
                   "target_surface": 3176.0, "lambda_surface": 0.2}],
        "contact": [0.0, 10.0, 10.0, 10.0],
        "temperature": 10.0, "neighbour_order": 3, "seed": 3, "steps": 3, "dump_every": 0,
        "initial": {"side": 8, "nx": 4, "ny": 4, "nz": 4},
        "units": {"micron_per_site": 1.0, "minute_per_step": 1.0},
    },
    "von-neumann-fields-64": {
        "name": "four neighbours and two fields with sub-steps",
        "width": 64, "height": 64,
        "types": [{"name": "Cell", "target_volume": 64.0, "lambda_volume": 1.0,
                   "secretion": {"a": 0.3}, "uptake": {"b": 0.1}}],
        "fields": [{"name": "a", "diffusion": 0.6, "decay": 0.02, "initial": 0.0},
                   {"name": "b", "diffusion": 0.1, "decay": 0.0, "initial": 1.0}],
        "contact": [0.0, 12.0, 12.0, 6.0],
        "temperature": 8.0, "neighbour_order": 1, "seed": 11, "steps": 12, "dump_every": 0,
        "initial": {"side": 8, "nx": 7, "ny": 7},
        "units": {"micron_per_site": 1.0, "minute_per_step": 1.0},
    },
}


def digest(labels) -> str:
    return hashlib.sha256(np.asarray(labels, dtype="<u4").tobytes()).hexdigest()


def main(reference: Path) -> None:
    sys.path.insert(0, str(reference / "python"))
    from glazier import _native  # the reference's own compiled module

    cases = []
    for path in sorted((reference / "blueprints").glob("*.json")):
        if path.name in SKIP:
            continue
        text = path.read_text()
        raw = json.loads(text)
        sites = raw["width"] * raw["height"] * raw.get("depth", 1)
        steps = 10 if sites <= 70_000 else 2
        cwd = os.getcwd()
        os.chdir(path.parent)
        try:
            labels, w, h, d = _native.run(text, steps)
            volumes = _native.run_volumes(text, steps)
        finally:
            os.chdir(cwd)
        cases.append({"case": path.name, "text": text, "steps": steps, "labels_sha256": digest(labels),
                      "volumes": list(map(int, volumes))})
    for name, raw in SYNTHETIC.items():
        text = json.dumps(raw)
        labels, w, h, d = _native.run(text, raw["steps"])
        volumes = _native.run_volumes(text, raw["steps"])
        cases.append({"case": name, "text": text, "steps": raw["steps"], "labels_sha256": digest(labels),
                      "volumes": list(map(int, volumes))})
    parses = {}
    for path in sorted((reference / "blueprints").glob("*.json")):
        parses[path.name] = {"text": path.read_text(), "parse": _native.parse(path.read_text())}
    out = {
        "generator": "tests/golden/make_golden.py",
        "engine": "glazier 0.3.0 python/glazier/_native.abi3.so (serial engine), every cell started as type 1",
        "cases": cases,
        "parse": parses,
    }
    (HERE / "serial_reference.json").write_text(json.dumps(out, indent=1))
    print(f"wrote {len(cases)} cases and {len(parses)} parse readings")


if __name__ == "__main__":
    main(Path(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GLAZIER_REFERENCE", ".")))
