"""The `--engine gpu` runner (glazier_b200/cli.py) against the reference's
runner, glazier/src/main.rs: its usage errors and exit codes, the `--check`
report's keys (main.rs:58-98), and on the device the files a run writes
(labels_NNNNN.npy every dump_every steps, the final lattice, summary.json
with the keys of main.rs:176-200, trace.csv) and that they hold the run the
engine itself makes from the same description."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from glazier_b200 import cli, native

GOLDEN = Path(__file__).resolve().parent / "golden" / "serial_reference.json"

# main.rs:58-98, in the reference's order
CHECK_KEYS = ["name", "width", "height", "n_types", "contact", "target_volume", "lambda_volume", "target_surface",
              "lambda_surface", "target_length", "lambda_length", "connected", "max_activity", "lambda_activity",
              "external", "lambda_nematic", "nematic_field", "initial_labels", "chemotaxis", "division_volume",
              "death_rate", "species", "diffusion", "decay", "secretion", "uptake", "temperature",
              "neighbour_order", "seed", "steps", "initial", "micron_per_site", "minute_per_step"]
# main.rs:176-200
SUMMARY_KEYS = ["name", "engine", "steps", "seconds", "setup_seconds", "overall_seconds", "n_cells", "n_labels",
                "fields", "mean_volume", "width", "height", "micron_per_site", "minute_per_step"]


def _text(name):
    return json.loads(GOLDEN.read_text())["parse"][name]["text"]


def _write(tmp_path, name, **overrides):
    raw = json.loads(_text(name))
    raw.update(overrides)
    path = tmp_path / name
    path.write_text(json.dumps(raw))
    return path


def test_usage_errors_exit_with_status_2(tmp_path, capsys):
    path = _write(tmp_path, "monolayer.json")
    assert cli.main([]) == 2
    assert cli.main(["--model", str(path), "--bogus"]) == 2
    assert cli.main(["--model", str(path)]) == 2  # neither --out nor --check
    assert cli.main(["--model"]) == 2
    assert cli.main(["--model", str(path), "--out", str(tmp_path / "o"), "--engine", "cpu"]) == 2
    assert "usage" in capsys.readouterr().err


def test_a_bad_description_exits_with_status_1(tmp_path, capsys):
    bad = tmp_path / "bad.json"
    bad.write_text("{not json")
    assert cli.main(["--model", str(bad), "--check"]) == 1
    assert cli.main(["--model", str(tmp_path / "missing.json"), "--check"]) == 1
    assert "cannot read" in capsys.readouterr().err


@pytest.mark.parametrize("name", ["monolayer.json", "infection.json", "monolayer-connected.json", "volume.json"])
def test_check_reports_what_the_reader_took(tmp_path, capsys, name):
    path = _write(tmp_path, name)
    assert cli.main(["--model", str(path), "--check"]) == 0
    got = json.loads(capsys.readouterr().out)
    assert list(got) == CHECK_KEYS
    parsed = native.parse(_text(name))
    for key in CHECK_KEYS:
        if key in parsed:
            assert got[key] == parsed[key], key


def test_labels_are_written_as_the_reference_shapes_them(tmp_path):
    lab = np.arange(2 * 3 * 4, dtype=np.uint32)
    cli.write_labels(tmp_path / "p.npy", lab[:12], 4, 3, 1)
    cli.write_labels(tmp_path / "v.npy", lab, 4, 3, 2)
    p, v = np.load(tmp_path / "p.npy"), np.load(tmp_path / "v.npy")
    assert p.shape == (3, 4) and p.dtype == np.dtype("<u4") and p[2, 1] == 9
    assert v.shape == (2, 3, 4) and v[1, 2, 3] == 23


@pytest.mark.gpu
def test_a_run_writes_the_dumps_the_summary_and_the_trace(device, tmp_path, capsys):
    path = _write(tmp_path, "infection.json", steps=30, dump_every=10)
    out = tmp_path / "run"
    assert cli.main(["--model", str(path), "--out", str(out), "--engine", "gpu", "--trace"]) == 0
    assert "30 steps" in capsys.readouterr().out
    names = sorted(p.name for p in out.iterdir())
    assert names == ["labels_00010.npy", "labels_00020.npy", "labels_00030.npy", "summary.json", "trace.csv"]
    summary = json.loads((out / "summary.json").read_text())
    assert list(summary) == SUMMARY_KEYS
    assert summary["engine"] == "gpu" and summary["steps"] == 30

    # the same description through the engine gives the same lattices
    session = native.GpuSession(path.read_text(), base=str(tmp_path))
    for step in (10, 20, 30):
        session.step(10)
        want = np.asarray(session.labels(), dtype=np.uint32).reshape(128, 128)
        assert np.array_equal(np.load(out / f"labels_{step:05d}.npy"), want), step
    volumes = session.simulation.volumes()
    live = volumes[1:][volumes[1:] > 0]
    assert summary["n_cells"] == live.size and summary["n_labels"] == volumes.size - 1
    assert summary["mean_volume"] == pytest.approx(float(live.mean()))
    for k, name in enumerate(("virus", "interferon")):
        assert summary["fields"][name] == pytest.approx(float(session.simulation.field(k).sum()))
    session.simulation.close()

    rows = (out / "trace.csv").read_text().splitlines()
    assert rows[0].startswith("step,cells,mean_volume") and len(rows) == 31
    assert rows[-1].split(",")[1] == str(summary["n_cells"])
