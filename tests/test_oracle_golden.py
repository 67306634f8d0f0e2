"""The serial oracle against the reference's own engine, bit for bit.

The fixtures in golden/serial_reference.json were made by running glazier's
compiled module on the reference blueprints and on synthetic descriptions
(golden/make_golden.py). The oracle must land on the same lattice (SHA-256)
and the same per-label volumes after the same steps, which pins its
arithmetic, its random stream and its bookkeeping to the reference's.
"""

from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from glazier_b200.blueprint import Blueprint, parse_dict
from oracle.serial import SerialOracle

GOLDEN = json.loads((Path(__file__).parent / "golden" / "serial_reference.json").read_text())
CASES = {c["case"]: c for c in GOLDEN["cases"]}


def _start(text: str):
    bp = Blueprint.from_json(text)
    raw = json.loads(text)
    if raw.get("nematic_field") or (raw["initial"].get("labels")):
        pytest.skip("needs a file beside the description")
    start = bp.start(".")
    # The shipped module starts every cell as the first type.
    start.cell_type[:] = 1
    return start


@pytest.mark.parametrize("name", sorted(CASES))
def test_the_oracle_lands_where_the_reference_does(name):
    case = CASES[name]
    oracle = SerialOracle.from_start(_start(case["text"]))
    oracle.step(case["steps"])
    digest = hashlib.sha256(oracle.labels().astype("<u4").tobytes()).hexdigest()
    assert digest == case["labels_sha256"], f"{name}: the lattice differs from the reference's"
    assert oracle.volumes().tolist() == case["volumes"]


@pytest.mark.parametrize("name", sorted(GOLDEN["parse"]))
def test_the_blueprint_reader_reads_what_the_reference_reads(name):
    entry = GOLDEN["parse"][name]
    mine = parse_dict(Blueprint.from_json(entry["text"]))
    for key, value in entry["parse"].items():
        assert key in mine, key
        if isinstance(value, list) and value and isinstance(value[0], float):
            assert np.allclose(mine[key], value, rtol=0, atol=1e-12), key
        else:
            assert mine[key] == value, key
