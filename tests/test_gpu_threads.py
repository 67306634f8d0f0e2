"""Handles driven from several host threads at once.

One handle is one stream and is not thread-safe (glazier-py's GpuSession is
`unsendable`, glazier-py/src/lib.rs:184), but distinct handles may run side
by side on their own host threads, as the benchmark's end-to-end leg does.
Each handle's run must then be the run it has alone: the same lattice,
volumes and surfaces bit for bit, whichever kernel its size takes.
"""

from __future__ import annotations

import threading

import numpy as np
import pytest

from glazier_b200.workloads import initial_surface, monolayer

pytestmark = pytest.mark.gpu


def _alone(device, start, steps):
    sim = device.GpuSimulation.from_start(start)
    sim.step(steps)
    out = sim.labels(), sim.volumes(), sim.surfaces(), sim.sweep_kernel
    sim.close()
    return out


@pytest.mark.parametrize("size", [128, 512, 1024, 2048, 4096])
def test_two_handles_on_two_threads_each_run_as_alone(device, size):
    start = monolayer(size, lambda_surface=0.2, target_surface=initial_surface(8))
    steps = 6
    want = _alone(device, start, steps)
    sims = [device.GpuSimulation.from_start(start) for _ in range(2)]
    errors = []

    def drive(sim):
        try:
            for _ in range(3):
                sim.step(2)
        except Exception as exc:  # reported on the main thread
            errors.append(exc)

    workers = [threading.Thread(target=drive, args=(s,)) for s in sims]
    for w in workers:
        w.start()
    for w in workers:
        w.join()
    assert not errors, errors
    for sim in sims:
        assert sim.sweep_kernel == want[3]
        assert np.array_equal(sim.labels(), want[0])
        assert np.array_equal(sim.volumes(), want[1])
        assert np.array_equal(sim.surfaces(), want[2])
        sim.close()
