#!/usr/bin/env python
"""Benchmark: site-updates/s of the plain 2D Cellular Potts sweep at 4096^2.

Workload (the reference's scaling configuration at its largest plane): a
periodic 4096 x 4096 int32 lattice tiled by 262,144 square cells of side 8,
one cell type, Moore contact J = 10, lambda_V = 1 with V_target = 64,
lambda_S = 0.2 with S_target = 92 (an 8 x 8 square's initial unlike-bond
count), T = 10, counter-hash RNG from seed 1. Synthetic: the lattice is the
tiling itself, as the reference's bench builds it (glazier/examples/bench.rs).

One timed step is one Monte Carlo step (16.8 M site updates). `value` is
device time (CUDA events on the engine's stream), inputs resident in HBM,
L2 flushed by a 256 MB write between timed steps. `e2e` runs whole jobs
through the public API from pinned host memory: upload the lattice
(glz_gpu_set_labels), 100 MCS (glz_gpu_step), download it (glz_gpu_labels);
two handles, each on its own stream and host thread, run their jobs side by
side so that one job's copies overlap the other's sweeps (`one_handle` is the
same jobs on one handle, back to back).

`--impl reference` times the reference's serial engine (its C restatement,
pinned bit for bit to the reference's compiled module) on the host cores,
one independent replica per core.

Multi-GPU: replicas only. Under torchrun each rank runs its own lattice
with no exchange; value is all ranks' site updates over the slowest rank.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PUBLISHED_4096 = 3.76e9  # README.md:121 of the reference: 4096^2, 100 MCS in 0.446 s (RTX 5060 Laptop)
FALLBACK_HBM_GBS = 6650.0
BYTES_PER_SITE_UPDATE = 20  # 4 colour passes x 4 B label read + 4 B label write per site per MCS
METRIC = "site-updates/s (plain 2D sweep, 4096^2)"


def metric_for(size: int) -> str:
    """The metric's name for a plane of `size`^2 (the default is the 4096^2 plane)."""
    return METRIC.replace("4096^2", f"{size}^2")


def workload(size: int):
    from glazier_b200.blueprint import CellType, Model, Start

    model = Model(
        width=size,
        height=size,
        contact=[0.0, 10.0, 10.0, 10.0],
        types=[CellType(), CellType(target_volume=64.0, lambda_volume=1.0, target_surface=92.0, lambda_surface=0.2)],
        temperature=10.0,
        neighbour_order=2,
        seed=1,
    )
    return Start.tiled(model, 8)


def config_dict(size: int, n: int) -> dict:
    return {
        "workload": f"plain 2D monolayer {size}x{size}, {(size // 8) ** 2} cells of side 8, Moore J=10, "
                    "lambda_V=1 V_t=64, lambda_S=0.2 S_t=92, T=10, seed 1",
        "sites": size * size,
        "step": "one Monte Carlo step (sites copy attempts, 4 colour passes)",
        "l2": "flushed between timed steps (256 MB write); the lattice is 64 MB",
        "parallelism": f"replicas x{n}" if n > 1 else "single replica",
        "e2e_step": "one job: upload lattice from pinned host, 100 MCS, download lattice; two handles on their "
                    "own streams and host threads run their jobs side by side",
        "baseline_note": "vs_baseline divides by the reference README's 4096^2 device figure (RTX 5060 Laptop, "
                         "bench.rs model J=[0,16,16,8], lambda_V=2, no surface term)",
    }


class Clocks:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out = ""

    def summary(self) -> dict:
        rows = []
        for line in (self.out or "").splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for _, _, flags in rows for k, f in enumerate(flags) if f.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def measured_peak() -> tuple:
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        peaks = json.loads(path.read_text())
        return float(peaks["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# DRAM bytes (read + write) of one launch of the headline sweep kernel on the
# 4096^2 workload, from an ncu capture of that kernel with cold caches
# (profiles/lean_sweep_2d_4096.md), with the kernel it was measured on; a
# figure measured on another kernel is not reported.
TRAFFIC = {"kernel": "lean", "bytes_per_launch": 79988480.0}


def ensemble_compare(mcs: int, device: int) -> dict:
    """64 uneven monolayer replicas (sides log-uniform 128..1024, own T, J and
    lambda_V): one batched ensemble under a CUDA graph against looping the
    plain engine over the same replicas. Both wait for their own results; the
    replicas' lattices come out identical."""
    import torch

    from glazier_b200.engine import GpuSimulation
    from glazier_b200.ensemble import Ensemble
    from glazier_b200.workloads import ensemble_starts

    starts = ensemble_starts(64)
    sites = sum(st.model.sites for st in starts)
    ens = Ensemble(starts, device=device)
    choice = ens.autotune(3)
    ens.step(3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    device_ms = ens.step_timed(mcs)
    batched_s = time.perf_counter() - t0
    sims = [GpuSimulation.from_start(st, device=device) for st in starts]
    for sim in sims:
        sim.step(3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for sim in sims:
        sim.step(mcs)
    looped_s = time.perf_counter() - t0
    same = all(np.array_equal(ens.labels(i), sims[i].labels()) for i in (0, 17, 63))
    for sim in sims:
        sim.close()
    ens.close()
    return {"replicas": 64, "sites": sites, "mcs": mcs, "batched_s": batched_s, "batched_device_ms": device_ms,
            "looped_plain_s": looped_s, "speedup": looped_s / batched_s,
            "batched_site_updates_per_s": sites * mcs / batched_s, "schedule_choice": choice,
            "lattices_identical": bool(same)}


def mixed_ensemble_compare(mcs: int, device: int) -> dict:
    """The configuration's full mix: 64 replicas alternating the plain
    monolayer and the two-field infection model (sides log-uniform 128..1024,
    own T, J and lambda_V; `mixed_ensemble_starts`). The monolayers run as
    one batch and each infection model as an engine whose captured step sits
    beside the batch's in one graph, replayed once per MCS; against looping
    the plain engine over the same replicas. Wall clock to every
    replica's result, both ways; a batched and an infection replica compared
    for identity."""
    import torch

    from glazier_b200.engine import GpuSimulation
    from glazier_b200.ensemble import Ensemble
    from glazier_b200.workloads import INFECTION_RULE, mixed_ensemble_starts

    starts, infected = mixed_ensemble_starts(64)
    sites = sum(st.model.sites for st in starts)
    ens = Ensemble(starts, device=device)
    for i in infected:
        ens.set_infection(i, *INFECTION_RULE)
    ens.autotune(3)
    ens.step(3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ens.step(mcs)
    mixed_s = time.perf_counter() - t0
    sims = [GpuSimulation.from_start(st, device=device) for st in starts]
    for i in infected:
        sims[i].set_infection(*INFECTION_RULE)
    for sim in sims:
        sim.step(3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for sim in sims:
        sim.step(mcs)
    looped_s = time.perf_counter() - t0
    same = all(np.array_equal(ens.labels(i), sims[i].labels()) for i in (0, infected[0], infected[-1]))
    for sim in sims:
        sim.close()
    ens.close()
    return {"replicas": 64, "infection_replicas": len(infected), "sites": sites, "mcs": mcs, "mixed_s": mixed_s,
            "looped_plain_s": looped_s, "speedup": looped_s / mixed_s, "lattices_identical": bool(same),
            "note": "monolayers batched (autotuned tile shape and colour schedule); each infection model's clocked "
                    "step beside the batch's, one graph replay per MCS for all 64"}


def adjoint_compare(steps: int, every: int, repeats: int, device: int) -> dict:
    """The field adjoint at 512^2 (4096 cells, two fields, four types): record
    `steps` MCS of owners from the engine, then time the adjoint's forward and
    backward (checkpoint every `every` steps, with recompute) on its stream
    with CUDA events, beside the plain engine's own field step over the same
    steps. Algorithmic bytes: 20 per site per field per step."""
    import torch

    from glazier_b200.adjoint import FieldAdjoint, owner_types
    from glazier_b200.engine import GpuSimulation
    from glazier_b200.workloads import adjoint_start, uniform01

    start = adjoint_start()
    m = start.model
    S, sites = len(m.species), m.sites
    sim = GpuSimulation.from_start(start, device=device)
    traj = np.empty((steps, sites), dtype=np.uint8)
    field_ms = 0.0
    for t in range(steps):
        field_ms += sim.step_profiled(1)[1]
        traj[t] = owner_types(sim.labels(), sim.cell_types())
    sim.close()
    params = np.concatenate([[sp.diffusion for sp in m.species], [sp.decay for sp in m.species],
                             np.asarray(m.secretion, dtype=np.float64).reshape(-1),
                             np.asarray(m.uptake, dtype=np.float64).reshape(-1)])
    adj = FieldAdjoint(m.width, m.height, 1, S, m.n_types, traj, checkpoint_every=every, device=device)
    f0 = torch.zeros(adj.shape, dtype=torch.float32, device=f"cuda:{device}")
    noise = np.array([2.0 * uniform01(1, i, 9) - 1.0 for i in range(params.size)])
    target = adj.forward(params * (1.0 + 0.1 * noise), f0)  # perturbed by 10% uniform noise
    # the loss gradient at the final fields (the forward is deterministic)
    grad = 2.0 * (adj.forward(params, f0) - target) / target.numel()
    stream = torch.cuda.ExternalStream(adj.stream, device=f"cuda:{device}")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    fwd, bwd = [], []
    for r in range(repeats + 2):
        ev[0].record(stream)
        adj.forward(params, f0)
        ev[1].record(stream)
        adj.backward(grad)
        ev[2].record(stream)
        ev[2].synchronize()
        if r >= 2:  # two warm-up rounds
            fwd.append(ev[0].elapsed_time(ev[1]))
            bwd.append(ev[1].elapsed_time(ev[2]))
    adj.close()
    f_ms, b_ms = statistics.median(fwd), statistics.median(bwd)
    nbytes = 20 * sites * S * steps
    return {"lattice": f"{m.width}x{m.height}", "cells": start.n_cells, "fields": S, "steps": steps,
            "checkpoint_every": every, "forward_ms": f_ms, "backward_ms": b_ms,
            "plain_field_step_ms": field_ms, "adjoint_over_plain": (f_ms + b_ms) / field_ms,
            "achieved_gbs": nbytes / ((f_ms + b_ms) / 1e3) / 1e9, "bytes_per_site_field_step": 20,
            "note": "fields are 1 MB each: the working set sits in L2, so HBM is not the bound here"}


def _device_ms(sim, run, device: int) -> float:
    """Milliseconds of device time `run` takes on the engine's stream."""
    import torch

    stream = torch.cuda.ExternalStream(sim.stream, device=f"cuda:{device}")
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    run()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b)


def infection_compare(mcs: int, cpu_mcs: int, device: int) -> dict:
    """The two-field infection model at 256^2 (centred 16 x 16 tissue with one
    infected cell, 32 immune cells at random in the medium; fields, division,
    death, length, chemotaxis and the connectivity veto all on) with its
    infection rule: `mcs` MCS on the device from the start, phases timed with
    CUDA events. Beside it the serial engine (the pinned restatement of the
    reference's CPU engine, one core) on the same start without the rule, which
    the reference does not have, over `cpu_mcs` MCS."""
    from glazier_b200.engine import GpuSimulation
    from glazier_b200.workloads import INFECTION_RULE, infection_start
    from oracle.serial import SerialOracle

    start = infection_start()
    sites = start.model.sites
    # the default path: every step replayed from the engine's captured graph,
    # device time by events on its stream around the whole run
    sim = GpuSimulation.from_start(start, device=device)
    sim.set_infection(*INFECTION_RULE)
    total = _device_ms(sim, lambda: sim.step(mcs), device)
    types, vols = sim.cell_types(), sim.volumes()
    infected = int(((types == 2) & (vols > 0)).sum())
    cells = int((vols[1:] > 0).sum())
    sim.close()
    # the phases, from a second run of the same start with every launch queued
    # from the host and each phase bracketed by events
    sim = GpuSimulation.from_start(start, device=device)
    sim.set_infection(*INFECTION_RULE)
    ms = sim.step_profiled(mcs)
    sim.close()
    o = SerialOracle.from_start(start)
    t = time.perf_counter()
    o.step(cpu_mcs)
    cpu_s = time.perf_counter() - t
    return {"lattice": "256x256", "mcs": mcs, "device_ms": total,
            "phase_ms": {"sweep": ms[0], "fields": ms[1], "population": ms[2], "run": "host-queued launches"},
            "site_updates_per_s": sites * mcs / (total / 1e3), "live_cells_end": cells,
            "infected_end": infected,
            "cpu_serial": {"mcs": cpu_mcs, "seconds": cpu_s, "site_updates_per_s": sites * cpu_mcs / cpu_s,
                           "cores": 1, "kind": "port", "note": "same start, infection rule off (the reference has none)"}}


# The reference's published device times (README.md:116-121, 206-210, 248-250;
# RTX 5060 Laptop): plane sizes with bench.rs's model, and three blueprints.
PUBLISHED_SIZES = {128: 0.002, 256: 0.002, 512: 0.007, 1024: 0.024, 2048: 0.097, 4096: 0.446}
PUBLISHED_BLUEPRINTS = {"volume.json": (50, 0.092), "infection-volume.json": (60, 0.081),
                        "infection-512.json": (200, 1.66)}


def published_rows(device: int) -> dict:
    """The reference's published rows on this engine: 100 MCS of bench.rs's
    model (tiled 8 x 8 cells, contact [0,16,16,8], lambda_V 2, V_t 64, T 10,
    Moore, seed 1; glazier/examples/bench.rs) at each plane size, and the
    three blueprints' steps, each timed from a created engine to the end of
    its steps on the host clock (what the reference's figures time) and on
    the device (CUDA events)."""
    import torch

    from glazier_b200 import native
    from glazier_b200.blueprint import CellType, Model, Start
    from glazier_b200.engine import GpuSimulation

    rows = {}
    for size, published in PUBLISHED_SIZES.items():
        m = Model(width=size, height=size, contact=[0.0, 16.0, 16.0, 8.0],
                  types=[CellType(), CellType(target_volume=64.0, lambda_volume=2.0)], temperature=10.0,
                  neighbour_order=2, seed=1)
        # a first engine pays the process's one-time costs (module loading,
        # kernel attributes); the timed one starts from its own start
        warm = GpuSimulation.from_start(Start.tiled(m, 8), device=device)
        warm.step(2)
        warm.close()
        sim = GpuSimulation.from_start(Start.tiled(m, 8), device=device)
        torch.cuda.synchronize()
        t = time.perf_counter()
        dev_ms = _device_ms(sim, lambda: sim.step(100), device)
        wall = time.perf_counter() - t
        sim.close()
        rows[f"{size}^2"] = {"mcs": 100, "wall_s": wall, "device_ms": dev_ms, "published_s": published,
                             "site_updates_per_s": size * size * 100 / wall, "speedup": published / wall}
    texts = json.loads((ROOT / "tests" / "golden" / "serial_reference.json").read_text())["parse"]
    for name, (steps, published) in PUBLISHED_BLUEPRINTS.items():
        session = native.GpuSession(texts[name]["text"])
        torch.cuda.synchronize()
        t = time.perf_counter()
        dev_ms = _device_ms(session.simulation, lambda: session.simulation.step(steps), device)
        wall = time.perf_counter() - t
        session.simulation.close()
        rows[name] = {"mcs": steps, "wall_s": wall, "device_ms": dev_ms, "published_s": published,
                      "speedup": published / wall}
    return rows


def coupling_leg(device: int, rounds: int = 3, steps: int = 250) -> dict:
    """The reference's coupling round (README.md:332-337): a 512^2 monolayer
    of 8 x 8 cells under a nematic field (contact [0,16,16,8], lambda_V 2,
    V_t 64, lambda_nematic 6, T 10, Moore, seed 1), rounds of 250 MCS, after
    each the lattice out and a new field in. Timed on the host clock per
    round: the steps, and the hand-over both ways, through host copies
    (``labels`` + ``set_nematic_field``) and through device tensors
    (``labels_tensor`` + ``set_nematic_field_tensor``). The new field is a
    function of the labels computed where the lattice is (numpy or torch);
    the reference's figures: 0.21 s of steps and 0.08 s of transfer a round."""
    import math

    import numpy as np
    import torch

    from glazier_b200.blueprint import CellType, Model, Start
    from glazier_b200.engine import GpuSimulation

    m = Model(width=512, height=512, contact=[0.0, 16.0, 16.0, 8.0],
              types=[CellType(), CellType(target_volume=64.0, lambda_volume=2.0, lambda_nematic=6.0)],
              temperature=10.0, neighbour_order=2, seed=1)
    m.nematic = np.tile([math.cos(1.2), math.sin(1.2)], (512 * 512, 1))
    out = {"lattice": "512^2", "mcs_per_round": steps, "rounds": rounds, "published_steps_s": 0.21,
           "published_transfer_s": 0.08}
    def hand_over(sim, mode):
        if mode == "host":
            lab = sim.labels().astype(np.int64)
            q = np.stack([((lab % 7) - 3) / 4.0, ((lab % 5) - 2) / 4.0], axis=1)
            sim.set_nematic_field(q)
        else:
            lab = sim.labels_tensor().reshape(-1)
            q = torch.stack([((lab % 7) - 3).float() / 4, ((lab % 5) - 2).float() / 4], dim=1)
            sim.set_nematic_field_tensor(q)
        torch.cuda.synchronize()

    for mode in ("host", "device"):
        sim = GpuSimulation.from_start(Start.tiled(m, 8), device=device)
        sim.step(2)
        hand_over(sim, mode)  # one-time costs (torch's kernels load on first use)
        step_s = hand_s = 0.0
        for _ in range(rounds):
            t = time.perf_counter()
            sim.step(steps)
            step_s += time.perf_counter() - t
            t = time.perf_counter()
            hand_over(sim, mode)
            hand_s += time.perf_counter() - t
        sim.close()
        out[mode] = {"steps_s_per_round": step_s / rounds, "handover_s_per_round": hand_s / rounds}
    return out


def volume_leg(mcs: int, device: int, peak: float) -> dict:
    """The scaling configuration's volume: a periodic 128^3 lattice of 4096
    cubic cells of side 8, 26 neighbours, J 10, lambda_V 1 at V_t 512,
    lambda_S 0.2 at S_t 3176 (a cube's initial unlike-bond count), T 10, seed
    1; `mcs` MCS after 3 of warm-up, L2 flushed before each, device time. Its
    algorithmic bytes are 36 per site-update (8 passes x 4 B read + 4 B
    written)."""
    import torch

    from glazier_b200.engine import GpuSimulation
    from glazier_b200.workloads import initial_surface, monolayer

    start = monolayer(128, depth=128, lambda_surface=0.2, target_surface=initial_surface(8, 3))
    sim = GpuSimulation.from_start(start, device=device)
    sim.step(3)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device=f"cuda:{device}")
    sweep = 0.0
    for _ in range(mcs):
        flush.zero_()
        torch.cuda.synchronize()
        sweep += sim.step_profiled(1)[0]
    sim.close()
    sites = start.model.sites
    rate = sites * mcs / (sweep / 1e3)
    return {"lattice": "128^3", "cells": start.n_cells, "mcs": mcs, "sweep_ms_per_mcs": sweep / mcs,
            "site_updates_per_s": rate, "bytes_per_site_update": 36,
            "roofline_frac": rate * 36 / 1e9 / peak, "l2": "flushed before each MCS (the lattice is 8 MB)"}


def cpu_baseline(size: int, seconds: float) -> dict:
    """The serial engine on one host core, a bounded sample of the same lattice."""
    from oracle.serial import SerialOracle

    start = workload(size)
    o = SerialOracle.from_start(start)
    o.attempts(200_000)  # warm
    t = time.perf_counter()
    probe = 2_000_000
    o.attempts(probe)
    rate = probe / (time.perf_counter() - t)
    n = max(probe, int(rate * seconds))
    t = time.perf_counter()
    o.attempts(n)
    dt = time.perf_counter() - t
    return {"value": n / dt, "unit": "site-updates/s", "cores": 1, "kind": "port",
            "sample": f"{n} serial copy attempts ({n / start.model.sites:.2f} MCS) on the {size}^2 lattice, "
                      "C restatement of glazier-core/src/cpu.rs pinned bit-exact to the reference module"}


def _reference_worker(args):
    size, per_step, steps, warmup = args
    sys.path.insert(0, str(ROOT))
    from oracle.serial import SerialOracle

    o = SerialOracle.from_start(workload(size))
    for _ in range(warmup):
        o.attempts(per_step)
    t = time.perf_counter()
    for _ in range(steps):
        o.attempts(per_step)
    return time.perf_counter() - t


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp

    cores = os.cpu_count() or 1
    from oracle import build as obuild

    obuild.build()
    # calibrate: a step is about half a second of one core's work
    from oracle.serial import SerialOracle

    o = SerialOracle.from_start(workload(args.size))
    t = time.perf_counter()
    o.attempts(1_000_000)
    rate = 1_000_000 / (time.perf_counter() - t)
    del o
    per_step = max(100_000, int(rate * 0.5))
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        times = pool.map(_reference_worker, [(args.size, per_step, args.steps, args.warmup)] * cores)
    wall = max(times)
    total = per_step * args.steps * cores
    value = total / wall
    line = {
        "metric": metric_for(args.size), "value": value, "unit": "site-updates/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(args.size, args.gpus),
        "cpu_baseline": {"value": value, "unit": "site-updates/s", "cores": cores, "kind": "port",
                         "sample": f"{cores} independent serial replicas, {per_step} copy attempts per step each"},
        "e2e": {"value": value, "unit": "site-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


class Ranks:
    """One process per GPU as torchrun starts them (RANK, WORLD_SIZE,
    LOCAL_RANK, MASTER_* from the environment): a barrier and the max over
    ranks, the only collectives the bench takes, since its replicas exchange
    nothing. NCCL on the GPUs; gloo with CPU tensors for tests of the host
    side. A short process-group timeout ends a wait on a rank that is gone."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        import torch

        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.cuda = backend == "nccl"
        self.dist = None
        if self.cuda:
            torch.cuda.set_device(self.local if self.world > 1 else 0)
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist
        self.device = torch.device("cuda", torch.cuda.current_device()) if self.cuda else torch.device("cpu")

    def barrier(self) -> None:
        import torch

        if self.dist is not None:
            self.dist.barrier()
        if self.cuda:
            torch.cuda.synchronize()

    def max_over_ranks(self, x: float) -> float:
        import torch

        if self.dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def whole_job_rate(units_per_rank: float, slowest_s: float, world: int) -> float:
    """Units all ranks processed over the slowest rank's time: the
    whole-job figure of a weakly scaled run."""
    return units_per_rank * world / slowest_s


def run_ours(args) -> None:
    import torch

    ranks = Ranks("nccl")
    world, rank, local = ranks.world, ranks.rank, ranks.local
    dev = ranks.device
    barrier, max_over_ranks = ranks.barrier, ranks.max_over_ranks

    from glazier_b200.engine import GpuSimulation

    start = workload(args.size)
    sites = start.model.sites
    sim = GpuSimulation.from_start(start, device=torch.cuda.current_device())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device=dev)  # 256 MB, past the 126 MB L2

    sim.step(args.warmup)
    phys = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")
    smi_index = int(phys[local]) if len(phys) > local and phys[local].strip().isdigit() else local
    sweep_ms = field_ms = pop_ms = 0.0
    barrier()
    with Clocks(smi_index) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            s, f, p = sim.step_profiled(1)
            sweep_ms += s
            field_ms += f
            pop_ms += p
        barrier()
    total_ms = sweep_ms + field_ms + pop_ms
    slowest = max_over_ranks(total_ms)
    value = whole_job_rate(sites * args.steps, slowest / 1e3, world)
    kernel = sim.sweep_kernel
    # the band sweep runs a step's four colour passes in one launch; the
    # per-pass kernels launch once per pass (the workload has no fields and no
    # population, so nothing else runs)
    launches_per_step = 1 if kernel == "band" else 4

    # end to end through the public API, host buffers pinned: one handle
    # running its jobs back to back, then two handles (each on its own
    # stream, driven by its own host thread) so that one job's copies overlap
    # the other's sweeps
    pinned_in = torch.from_numpy(start.labels.view(np.int32)).pin_memory()
    jobs, job_mcs = args.e2e_jobs, 100
    sims = [sim, GpuSimulation.from_start(start, device=torch.cuda.current_device())]
    pinned_out = [torch.empty(sites, dtype=torch.int32).pin_memory() for _ in sims]
    for s_ in sims:
        s_.set_labels_from(pinned_in.data_ptr(), sites)
        s_.step(1)
    torch.cuda.synchronize()

    def run_jobs(k: int) -> None:
        for _ in range(jobs):
            sims[k].set_labels_from(pinned_in.data_ptr(), sites)
            sims[k].step(job_mcs)
            sims[k].labels_to(pinned_out[k].data_ptr(), sites)

    barrier()
    t0 = time.perf_counter()
    run_jobs(0)
    torch.cuda.synchronize()
    serial_s = max_over_ranks(time.perf_counter() - t0)
    serial_value = whole_job_rate(sites * job_mcs * jobs, serial_s, world)
    barrier()
    t0 = time.perf_counter()
    workers = [threading.Thread(target=run_jobs, args=(k,)) for k in range(len(sims))]
    for w in workers:
        w.start()
    for w in workers:
        w.join()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = whole_job_rate(sites * job_mcs * jobs * len(sims), e2e_s, world)
    for out in pinned_out:
        assert int(out.max()) <= (args.size // 8) ** 2
    sims[1].close()

    peak, peak_kind = measured_peak()
    launch_s = (sweep_ms / 1e3) / (args.steps * launches_per_step)
    bytes_per_launch = sites * BYTES_PER_SITE_UPDATE / launches_per_step  # one MCS spread over its launches
    achieved = bytes_per_launch / launch_s / 1e9
    kernel_name = {"band": "band_sweep_kernel<8,1> (one MCS: four colour passes)",
                   "lean": "lean_sweep_kernel<2,8,1> (one colour pass)"}.get(kernel, kernel)
    traffic = TRAFFIC["bytes_per_launch"] if TRAFFIC["kernel"] == kernel else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": peak_kind, "kernel": kernel_name,
                "algorithmic_bytes_per_launch": bytes_per_launch, "launch_ms": launch_s * 1e3}

    sim.close()
    ranks.close()
    if rank != 0:
        return
    line = {
        "metric": metric_for(args.size), "value": value, "unit": "site-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": value / PUBLISHED_4096, "dtype": "f32", "data": "synthetic",
        "config": config_dict(args.size, world),
        "e2e": {"value": e2e_value, "unit": "site-updates/s", "h2d_bytes_per_step": sites * 4,
                "d2h_bytes_per_step": sites * 4, "jobs": jobs * len(sims), "mcs_per_job": job_mcs,
                "handles": len(sims), "one_handle": {"value": serial_value, "jobs": jobs}},
        "roofline": roofline,
        "gpu_launches": args.steps * launches_per_step,
        "clocks": clocks.summary(),
        "phase_ms": {"sweep": sweep_ms, "fields": field_ms, "population": pop_ms},
    }
    # The side legs, verbose ones first: a reader of the line's end (a log
    # tail) sees the compact figures of the volume, infection, adjoint and
    # ensemble legs and the CPU baseline.
    dev_index = torch.cuda.current_device()
    if world == 1 and not args.no_published:
        line["published_rows"] = published_rows(dev_index)
        line["coupling"] = coupling_leg(dev_index)
        line["volume"] = volume_leg(20, dev_index, peak)
    if world == 1 and not args.no_infection:
        line["infection"] = infection_compare(200, 20, dev_index)
    if world == 1 and not args.no_adjoint:
        line["adjoint"] = adjoint_compare(50, 10, 5, dev_index)
    if world == 1 and not args.no_ensemble:
        line["ensemble"] = ensemble_compare(100, dev_index)
        line["mixed_ensemble"] = mixed_ensemble_compare(100, dev_index)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.size, args.cpu_seconds)
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--e2e-jobs", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-infection", action="store_true")
    ap.add_argument("--no-published", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("at least 3 warm-up steps")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
