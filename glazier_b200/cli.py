"""Run a Blueprint on the device and write the label fields.

The command line of the reference's runner (glazier/src/main.rs) for its
device path, over this engine:

    python -m glazier_b200.cli --model <blueprint.json> --out <dir> [--engine gpu] [--trace]
    python -m glazier_b200.cli --model <blueprint.json> --check

- `--out`: runs the description's steps, writing `labels_NNNNN.npy` every
  `dump_every` steps (not at the last step, main.rs:320-331) and, at the
  end, `labels_<steps>.npy` and `summary.json` with the keys of main.rs:
  176-200 (`seconds` times the steps alone; engine creation is
  `setup_seconds`). Lattices are C-order uint32 `.npy` files shaped
  (height, width) in a plane and (depth, height, width) in a volume
  (glazier-core/src/npy.rs:11-50).
- `--trace`: also `trace.csv`, one row per step with the live cells, their
  mean volume and each field's total (main.rs:236-262). The device engine
  steps one MCS at a time for it.
- `--check`: prints what this reader took from the description with the
  keys of main.rs:58-98, for comparison with another reader.
- `--engine`: `gpu` (the default here). The reference's serial engine is not
  part of this build: `--engine cpu` is refused with exit status 2.

Exit status: 0 on success, 1 on a description or run error, 2 on a usage
error, as the reference's runner returns them.
"""

from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

USAGE = (
    "usage: python -m glazier_b200.cli --model <blueprint.json> --out <dir> [--engine gpu] [--trace]\n"
    "       python -m glazier_b200.cli --model <blueprint.json> --check\n"
    "\n"
    "Writes labels_NNNNN.npy per dump and summary.json at the end.\n"
    "--check parses the description and prints what this engine read, so a\n"
    "second reader of the same file can be compared against it.\n"
    "--trace writes trace.csv, one row per step: live cells, mean volume,\n"
    "and the total of every field."
)


def _usage() -> int:
    print(USAGE, file=sys.stderr)
    return 2


def write_labels(path: Path, labels: np.ndarray, width: int, height: int, depth: int) -> None:
    """A lattice as a C-order uint32 array, two-dimensional in a plane."""
    shape = (depth, height, width) if depth > 1 else (height, width)
    np.save(path, np.ascontiguousarray(labels, dtype="<u4").reshape(shape), allow_pickle=False)


def check_dict(bp) -> dict:
    """main.rs:58-98: what the reader took from the description."""
    m = bp.model()
    per = lambda name: [getattr(t, name) for t in m.types]  # noqa: E731
    return {
        "name": bp.name,
        "width": m.width,
        "height": m.height,
        "n_types": m.n_types,
        "contact": list(m.contact),
        "target_volume": per("target_volume"),
        "lambda_volume": per("lambda_volume"),
        "target_surface": per("target_surface"),
        "lambda_surface": per("lambda_surface"),
        "target_length": per("target_length"),
        "lambda_length": per("lambda_length"),
        "connected": [bool(t.connected) for t in m.types],
        "max_activity": per("max_activity"),
        "lambda_activity": per("lambda_activity"),
        "external": [list(t.external) for t in m.types],
        "lambda_nematic": per("lambda_nematic"),
        "nematic_field": bp.nematic_field,
        "initial_labels": bp.initial["labels"],
        "chemotaxis": [list(r) for r in m.chemotaxis],
        "division_volume": per("division_volume"),
        "death_rate": per("death_rate"),
        "species": [s.name for s in m.species],
        "diffusion": [s.diffusion for s in m.species],
        "decay": [s.decay for s in m.species],
        "secretion": [list(r) for r in m.secretion],
        "uptake": [list(r) for r in m.uptake],
        "temperature": m.temperature,
        "neighbour_order": m.neighbour_order,
        "seed": m.seed,
        "steps": bp.steps,
        "initial": [int(bp.initial["side"]), int(bp.initial["nx"]), int(bp.initial["ny"]), int(bp.initial["nz"])],
        "micron_per_site": float(bp.raw["units"]["micron_per_site"]),
        "minute_per_step": float(bp.raw["units"]["minute_per_step"]),
    }


def _live_mean(volumes: np.ndarray) -> tuple:
    """Live cells and their mean volume: a label at volume zero died."""
    live = volumes[1:][volumes[1:] > 0]
    return int(live.size), (float(live.astype(np.float64).mean()) if live.size else 0.0)


def run_gpu(bp, start, out: Path, trace: bool) -> dict:
    """main.rs:285-351: create the engine, step in chunks of `dump_every`,
    dump between chunks; returns the timings, the final labels and volumes,
    and each field's total."""
    from .engine import GpuSimulation

    began = time.perf_counter()
    sim = GpuSimulation.from_start(start)
    if bp.infection_rule() is not None:
        sim.set_infection(*bp.infection_rule())
    setup = time.perf_counter() - began
    species = [s.name for s in start.model.species]
    rows = []
    if trace:
        rows.append(",".join(["step", "cells", "mean_volume", *species]))
    chunk = 1 if trace else (bp.dump_every if bp.dump_every > 0 else bp.steps)
    done = 0
    w, h, d = bp.width, bp.height, bp.depth
    with sim:
        while done < bp.steps:
            take = min(chunk, bp.steps - done)
            sim.step(take)
            done += take
            if trace:
                cells, mean = _live_mean(sim.volumes())
                totals = [f"{float(sim.field(k).sum()):.6f}" for k in range(len(species))]
                rows.append(",".join([str(done), str(cells), f"{mean:.3f}", *totals]))
            if bp.dump_every > 0 and done % bp.dump_every == 0 and done != bp.steps:
                write_labels(out / f"labels_{done:05d}.npy", sim.labels(), w, h, d)
        stepping = time.perf_counter() - began
        fields = {name: float(sim.field(k).sum()) for k, name in enumerate(species)}
        labels, volumes = sim.labels(), sim.volumes()
    if trace:
        (out / "trace.csv").write_text("\n".join(rows) + "\n")
    return {"setup": setup, "stepping": stepping, "fields": fields, "labels": labels, "volumes": volumes}


def main(argv=None) -> int:
    from .blueprint import Blueprint, BlueprintError

    args = list(sys.argv[1:] if argv is None else argv)
    model_path = out = None
    engine = "gpu"
    check = trace = False
    i = 0
    while i < len(args):
        a = args[i]
        if a in ("--model", "--out", "--engine"):
            if i + 1 >= len(args):
                return _usage()
            value = args[i + 1]
            i += 2
            if a == "--model":
                model_path = Path(value)
            elif a == "--out":
                out = Path(value)
            else:
                engine = value
            continue
        if a == "--check":
            check = True
        elif a == "--trace":
            trace = True
        else:
            return _usage()
        i += 1
    if model_path is None:
        return _usage()
    try:
        text = model_path.read_text()
    except OSError as e:
        print(f"cannot read {model_path}: {e}", file=sys.stderr)
        return 1
    try:
        bp = Blueprint.from_json(text)
    except BlueprintError as e:
        print(f"{model_path}: {e}", file=sys.stderr)
        return 1
    if check:
        print(json.dumps(check_dict(bp), indent=2))
        return 0
    if out is None:
        return _usage()
    if engine != "gpu":
        print(f"unknown engine {engine}: this build runs the device engine only (--engine gpu)", file=sys.stderr)
        return _usage()
    try:
        out.mkdir(parents=True, exist_ok=True)
    except OSError as e:
        print(f"cannot create {out}: {e}", file=sys.stderr)
        return 1
    try:
        start = bp.start(model_path.parent)
    except BlueprintError as e:
        print(str(e), file=sys.stderr)
        return 1
    overall_began = time.perf_counter()
    try:
        r = run_gpu(bp, start, out, trace)
    except Exception as e:  # the engine's GpuError and driver failures
        print(str(e), file=sys.stderr)
        return 1
    overall = time.perf_counter() - overall_began
    cells, mean = _live_mean(r["volumes"])
    summary = {
        "name": bp.name,
        "engine": engine,
        "steps": bp.steps,
        "seconds": r["stepping"] if r["stepping"] > 0.0 else overall - r["setup"],
        "setup_seconds": r["setup"],
        "overall_seconds": overall,
        "n_cells": cells,
        "n_labels": int(r["volumes"].size) - 1,
        "fields": dict(sorted(r["fields"].items())),
        "mean_volume": mean,
        "width": bp.width,
        "height": bp.height,
        "micron_per_site": float(bp.raw["units"]["micron_per_site"]),
        "minute_per_step": float(bp.raw["units"]["minute_per_step"]),
    }
    try:
        (out / "summary.json").write_text(json.dumps(summary, indent=2))
    except OSError as e:
        print(f"cannot write the summary: {e}", file=sys.stderr)
        return 1
    write_labels(out / f"labels_{bp.steps:05d}.npy", r["labels"], bp.width, bp.height, bp.depth)
    print(f"{engine}: {bp.steps} steps in {summary['seconds']:.3f} s, {cells} cells, mean volume {mean:.1f}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
