"""Shared fixtures: the `gpu` marker, starts built the way the reference's
tests build them, and the libraries under test."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from glazier_b200.blueprint import CellType, Model, Species, Start  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200)")


def _has_cuda() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def device():
    """The built engine on a CUDA device; GPU tests fail (not skip) when the
    library is missing, since the device path has no fallback."""
    if not _has_cuda():
        pytest.skip("no CUDA device")
    from glazier_b200 import build

    build.build()
    from glazier_b200 import engine

    return engine


def sheet_model(width=64, height=64, depth=1, seed=1, contact=(0.0, 16.0, 16.0, 8.0), target_volume=64.0,
                lambda_volume=2.0, temperature=10.0, order=2, **type_kw) -> Model:
    """The reference tests' sheet (glazier-tests/tests/gpu_matches_cpu.rs:14-33)."""
    return Model(
        width=width,
        height=height,
        depth=depth,
        contact=list(contact),
        types=[CellType(), CellType(target_volume=target_volume, lambda_volume=lambda_volume, **type_kw)],
        temperature=temperature,
        neighbour_order=order,
        seed=seed,
    )


def tiled(model: Model, side: int = 8, nx=None, ny=None, nz=None) -> Start:
    if nx is None:
        return Start.tiled(model, side)
    return Start.tiled_grid(model, side, nx, ny, nz or 1)


def with_species(model: Model, species, secretion, uptake, chemotaxis) -> Model:
    model.species = [Species(*s) for s in species]
    model.secretion = [list(r) for r in secretion]
    model.uptake = [list(r) for r in uptake]
    model.chemotaxis = [list(r) for r in chemotaxis]
    return model


def spread(volumes, target: float) -> float:
    v = np.asarray(volumes, dtype=np.float64)
    return float(np.sqrt(np.mean((v - target) ** 2)))


def recount_volumes(labels, n_labels: int) -> np.ndarray:
    return np.bincount(np.asarray(labels, dtype=np.int64), minlength=n_labels).astype(np.uint32)


def pieces(labels, width, height, depth=1) -> int:
    """Pieces each label falls into under the Moore (26) ring
    (glazier-tests/tests/connectivity.rs:31-55)."""
    lab = np.asarray(labels).reshape(depth, height, width)
    seen = np.zeros_like(lab, dtype=bool)
    total = 0
    ring = [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)
            if (dx, dy, dz) != (0, 0, 0) and (depth > 1 or dz == 0)]
    for z in range(depth):
        for y in range(height):
            for x in range(width):
                if lab[z, y, x] == 0 or seen[z, y, x]:
                    continue
                total += 1
                label = lab[z, y, x]
                stack = [(x, y, z)]
                seen[z, y, x] = True
                while stack:
                    cx, cy, cz = stack.pop()
                    for dx, dy, dz in ring:
                        nx, ny, nz = (cx + dx) % width, (cy + dy) % height, (cz + dz) % depth
                        if not seen[nz, ny, nx] and lab[nz, ny, nx] == label:
                            seen[nz, ny, nx] = True
                            stack.append((nx, ny, nz))
    return total
