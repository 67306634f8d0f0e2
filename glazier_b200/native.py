"""The ``glazier._native`` entry points, over the device engine.

Mirrors glazier-py/src/lib.rs: the same names, arguments, return shapes and
errors (``ValueError``), so a caller of ``glazier._native`` switches by
import. ``parse`` reads a description exactly as the reference does; ``run``
and ``run_volumes`` run it on the B200 engine, whose sweep agrees with the
serial engine in distribution (the reference's own device path is
checkerboard and agrees the same way, glazier-cuda/src/lib.rs:1-15).
"""

from __future__ import annotations

from .blueprint import Blueprint, BlueprintError, parse_dict
from .engine import GpuError, GpuSimulation

__all__ = ["parse", "run", "run_volumes", "GpuSession"]


def _blueprint(text: str) -> Blueprint:
    try:
        return Blueprint.from_json(text)
    except BlueprintError as e:
        raise ValueError(str(e)) from None


def parse(text: str) -> dict:
    """What this engine read from a description (glazier-py/src/lib.rs:18-146)."""
    return parse_dict(_blueprint(text))


def _simulate(text: str, steps, base: str = "."):
    bp = _blueprint(text)
    try:
        start = bp.start(base)
    except BlueprintError as e:
        raise ValueError(str(e)) from None
    sim = GpuSimulation.from_start(start)
    if bp.infection_rule() is not None:
        sim.set_infection(*bp.infection_rule())
    sim.step(bp.steps if steps is None else int(steps))
    return bp, sim


def run(text: str, steps: int | None = None):
    """Run a description and return ``(labels, width, height, depth)``, the
    labels flat with x fastest (glazier-py/src/lib.rs:148-163)."""
    bp, sim = _simulate(text, steps)
    with sim:
        return sim.labels().tolist(), bp.width, bp.height, bp.depth


def run_volumes(text: str, steps: int | None = None) -> list:
    """Per-cell volumes after a run, index 0 the medium (glazier-py/src/lib.rs:165-177)."""
    _, sim = _simulate(text, steps)
    with sim:
        return sim.volumes().tolist()


class GpuSession:
    """A run kept on the device between calls, for coupling to another solver
    (glazier-py/src/lib.rs:179-241). Relative ``.npy`` paths in the
    description resolve against ``base``."""

    def __init__(self, text: str, base: str = "."):
        bp = _blueprint(text)
        try:
            start = bp.start(base)
        except BlueprintError as e:
            raise ValueError(str(e)) from None
        self._sim = GpuSimulation.from_start(start)
        if bp.infection_rule() is not None:
            self._sim.set_infection(*bp.infection_rule())
        self._sites = bp.width * bp.height * bp.depth

    def step(self, steps: int) -> None:
        """Run ``steps`` Monte Carlo steps."""
        self._sim.step(steps)

    def labels(self) -> list:
        """The lattice, flat with x fastest."""
        return self._sim.labels().tolist()

    def set_nematic_field(self, flat) -> None:
        """Replace the field from ``2 * sites`` numbers, (Q_xx, Q_xy) per site."""
        flat = list(flat)
        if len(flat) != 2 * self._sites:
            raise ValueError(f"expected {2 * self._sites} numbers, got {len(flat)}")
        self._sim.set_nematic_field(flat)

    def labels_tensor(self):
        """The lattice as a device tensor without a copy (int32, shaped
        (depth, height, width)): the zero-copy ``labels`` for a solver that
        runs on the same GPU. Valid until the session is dropped; read only."""
        return self._sim.labels_tensor()

    def set_nematic_field_tensor(self, field) -> None:
        """``set_nematic_field`` from a CUDA float32 tensor of ``2 * sites``
        values, (Q_xx, Q_xy) per site, without a trip through the host."""
        self._sim.set_nematic_field_tensor(field)

    @property
    def mcs(self) -> int:
        """Monte Carlo steps completed."""
        return self._sim.mcs

    @property
    def simulation(self) -> GpuSimulation:
        """The engine underneath, for numpy or device-pointer access."""
        return self._sim


__all__ += ["GpuError"]
