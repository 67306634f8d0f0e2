"""The C ABI library and the host-side boundary, without a GPU.

The library must load and export every entry point include/glazier_gpu.h
declares, and the refusals the reference makes before touching a device
(odd sides, unsupported terms, bad arguments) must come back as statuses.
"""

from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import sheet_model, tiled
from glazier_b200 import _lib, build
from glazier_b200.blueprint import Blueprint, BlueprintError

HEADERS = sorted((Path(__file__).resolve().parents[1] / "include").glob("*.h"))


def declared_symbols():
    names = []
    for header in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        names += re.findall(r"^[A-Za-z_][\w \t\*]*?\b(glz_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def L():
    build.build()
    return _lib.lib()


def test_the_library_exports_every_declared_entry_point(L):
    names = declared_symbols()
    assert "glz_gpu_create" in names and len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def _create(model, start=None):
    keep = []
    m = _lib.model_struct(model, keep)
    start = start or tiled(model)
    h = C.c_void_p()
    rc = _lib.lib().glz_gpu_create(C.byref(m), _lib.ptr(start.labels), _lib.ptr(start.cell_type),
                                   start.cell_type.size, None, None, C.byref(h))
    return rc, h


def test_an_odd_side_is_refused_with_the_reference_message(L):
    # gpu_matches_cpu.rs:140-149
    m = sheet_model(width=34, height=32)
    m.width = 33
    start = tiled(sheet_model(width=33, height=32))
    rc, h = _create(m, start)
    assert rc == _lib.GLZ_ODD_LATTICE and not h.value
    assert "even sides" in _lib.last_error()


def test_an_activity_without_the_motility_term_is_refused(L):
    """Every term of the reference's model runs on the device; an activity
    field for a model that never reads it is refused rather than dropped."""
    import ctypes as C

    m = sheet_model(width=32, height=32)
    start = tiled(m)
    keep: list = []
    gm = _lib.model_struct(m, keep)
    lab = np.ascontiguousarray(start.labels, dtype=np.uint32)
    ct = np.ascontiguousarray(start.cell_type, dtype=np.uint8)
    act = np.ones(m.sites)
    h = C.c_void_p()
    rc = L.glz_gpu_create(C.byref(gm), _lib.ptr(lab), _lib.ptr(ct), ct.size, None, _lib.ptr(act), C.byref(h))
    assert rc == _lib.GLZ_UNSUPPORTED and not h.value
    assert "motility" in _lib.last_error()


def test_a_label_past_the_type_table_is_refused(L):
    m = sheet_model(width=32, height=32)
    start = tiled(m)
    start.cell_type = start.cell_type[:-3].copy()
    rc, _ = _create(m, start)
    assert rc == _lib.GLZ_INVALID


def test_the_reader_refuses_what_the_reference_refuses():
    base = {
        "name": "x", "width": 16, "height": 16, "types": [{"name": "A", "target_volume": 16, "lambda_volume": 1}],
        "contact": [0, 1, 1, 1], "temperature": 10, "neighbour_order": 2, "seed": 1, "steps": 1, "dump_every": 0,
        "initial": {"side": 4, "nx": 2, "ny": 2}, "units": {"micron_per_site": 1, "minute_per_step": 1},
    }
    import copy
    import json

    bad = copy.deepcopy(base)
    bad["initial"]["fractions"] = {"B": 0.5}
    with pytest.raises(BlueprintError, match="does not state"):
        Blueprint.from_json(json.dumps(bad))
    bad = copy.deepcopy(base)
    bad["types"][0]["secretion"] = {"nothing": 1.0}
    with pytest.raises(BlueprintError, match="not a field"):
        Blueprint.from_json(json.dumps(bad))
    bad = copy.deepcopy(base)
    bad["types"][0]["presents"] = {"cadherin": 1.0}
    with pytest.raises(BlueprintError, match="declares none"):
        Blueprint.from_json(json.dumps(bad))
    bad = copy.deepcopy(base)
    bad["contact"] = [0, 1, 2, 1]
    with pytest.raises(BlueprintError, match="asymmetric"):
        Blueprint.from_json(json.dumps(bad))


def test_the_reader_takes_an_infection_rule_and_refuses_a_bad_one():
    """The `infection` key is an extension glazier's reader lacks: a good rule
    comes back in engine indices (field, from type, to type, threshold), a
    rule naming something undeclared is refused."""
    import copy
    import json

    base = {
        "name": "x", "width": 16, "height": 16,
        "types": [{"name": "Healthy", "target_volume": 16, "lambda_volume": 1, "uptake": {"virus": 0.02}},
                  {"name": "Infected", "target_volume": 16, "lambda_volume": 1, "secretion": {"virus": 1.0}}],
        "fields": [{"name": "virus", "diffusion": 0.05}],
        "contact": [0, 16, 16, 16, 10, 10, 16, 10, 10], "temperature": 10, "neighbour_order": 2, "seed": 1,
        "steps": 1, "dump_every": 0, "initial": {"side": 4, "nx": 2, "ny": 2},
        "units": {"micron_per_site": 1, "minute_per_step": 1},
        "infection": {"field": "virus", "from": "Healthy", "to": "Infected", "threshold": 5},
    }
    assert Blueprint.from_json(json.dumps(base)).infection_rule() == (0, 1, 2, 5.0)
    plain = copy.deepcopy(base)
    del plain["infection"]
    assert Blueprint.from_json(json.dumps(plain)).infection_rule() is None
    for key, value, message in (("field", "toxin", "does not declare"), ("to", "Immune", "does not state"),
                                ("to", "Healthy", "to itself"), ("threshold", -1, ">= 0")):
        bad = copy.deepcopy(base)
        bad["infection"][key] = value
        with pytest.raises(BlueprintError, match=message):
            Blueprint.from_json(json.dumps(bad))


def test_initial_types_hand_out_rounded_shares_in_order():
    # blueprint.rs:247-261: 2% of 256 is 5.12, so five cells, the first five
    import json

    raw = {
        "name": "x", "width": 128, "height": 128,
        "types": [{"name": "A", "target_volume": 64, "lambda_volume": 1},
                  {"name": "B", "target_volume": 64, "lambda_volume": 1}],
        "contact": [0, 1, 1, 1, 1, 1, 1, 1, 1], "temperature": 10, "neighbour_order": 2, "seed": 1, "steps": 1,
        "dump_every": 0, "initial": {"side": 8, "nx": 16, "ny": 16, "fractions": {"B": 0.02}},
        "units": {"micron_per_site": 1, "minute_per_step": 1},
    }
    types = Blueprint.from_json(json.dumps(raw)).initial_types(256)
    assert types[:5].tolist() == [2] * 5 and (types[5:] == 1).all()
