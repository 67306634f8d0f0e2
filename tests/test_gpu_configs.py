"""Bit-exact parity at the benchmark configurations' own sizes.

Each case builds the start the benchmark builds, runs it on the B200 with the
engine's default kernel selection (every GLAZIER_SWEEP_* override removed),
and requires the lattice, per-label volumes and surfaces to equal the host
replay of the schedule (oracle/replay.c) after a first MCS and at the end:
  - the plain monolayer: 128^2, 256 cells of side 8, J=10, lambda_V=1,
    V_t=64, T=10, 100 MCS;
  - the scaling sweep's planes with the surface term (lambda_S=0.2, S_t=92):
    1024^2 and 4096^2 for 10 MCS each, the former on the block-queued direct
    kernel, the latter on the windowed lean kernel's full persistent grid
    (444 CTAs walking their tiles through their three-stage TMA window
    rings), and 2048^2 for 4 MCS on the lean kernel with 2.3 tiles a CTA;
  - the scaling sweep's 128^3 volume, 26 neighbours, lambda_S=0.2,
    S_t=3176, for 10 MCS, on the block-queued direct kernel;
  - a lean volume just past the size from which the direct kernel queues its
    copies (204^3 sites, 2^20 targets a pass), so the default thresholds are
    held to the replay too.
The form follows glazier-tests/tests/gpu_matches_cpu.rs:48-92 (a device run
against a host run of the same start), with exact equality in place of the
reference's distribution bands, since this engine's schedule is replayable.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from glazier_b200.workloads import initial_surface, monolayer
from oracle.replay import ReplayOracle

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _default_kernels(monkeypatch):
    for name in list(os.environ):
        if name.startswith("GLAZIER_SWEEP_"):
            monkeypatch.delenv(name)


def _run_both(device, start, steps, kernel):
    gpu = device.GpuSimulation.from_start(start)
    assert gpu.sweep_kernel == kernel
    replay = ReplayOracle.from_start(start)
    for chunk in (1, steps - 1):
        gpu.step(chunk)
        replay.step(chunk)
        labels, want = gpu.labels(), replay.labels()
        assert np.array_equal(labels, want), f"{int((labels != want).sum())} sites differ after {gpu.mcs} MCS"
        assert np.array_equal(gpu.volumes(), replay.volumes())
        assert np.array_equal(gpu.surfaces(), replay.surfaces())
    assert replay.accepted > 0
    gpu.close()


def test_the_plain_monolayer_replays_bit_for_bit_over_100_mcs(device):
    start = monolayer(128)
    assert start.model.sites == 128 * 128 and int(start.labels.max()) == 256
    _run_both(device, start, 100, "cluster")


def test_the_1024_plane_with_the_surface_term_replays_bit_for_bit(device):
    start = monolayer(1024, lambda_surface=0.2, target_surface=initial_surface(8))
    assert start.model.types[1].target_surface == 92.0
    _run_both(device, start, 10, "gathered")


def test_the_2048_plane_replays_bit_for_bit_on_the_lean_kernel(device):
    start = monolayer(2048, lambda_surface=0.2, target_surface=initial_surface(8))
    _run_both(device, start, 4, "lean")


def test_the_4096_plane_with_the_surface_term_replays_bit_for_bit(device):
    start = monolayer(4096, lambda_surface=0.2, target_surface=initial_surface(8))
    _run_both(device, start, 10, "lean")


def test_the_128_volume_with_the_surface_term_replays_bit_for_bit(device):
    start = monolayer(128, depth=128, lambda_surface=0.2, target_surface=initial_surface(8, 3))
    assert start.model.types[1].target_surface == 3176.0
    _run_both(device, start, 10, "gathered")


def test_a_volume_past_the_queueing_threshold_replays_bit_for_bit(device):
    start = monolayer(204, depth=204, side=6, lambda_surface=0.2, target_surface=initial_surface(6, 3))
    assert start.model.sites // 8 >= 1 << 20
    _run_both(device, start, 3, "compact")
