"""Synthetic starts with the shapes of the scaling, ensemble and field runs.

No public dataset is involved: every start is a tiling of square (or cubic)
cells, built the way the reference's own benchmark builds its lattices
(glazier/examples/bench.rs, Lattice::tile_grid in lattice.rs:169-196), with
parameters drawn from a counter hash of (seed, index) so a run is the same on
every machine.
"""

from __future__ import annotations

import math

import numpy as np

from .blueprint import CellType, Model, Species, Start

_M64 = (1 << 64) - 1


def _mix(z: int) -> int:
    """SplitMix64's finaliser, the mixer of the engine's counter hash."""
    z = (z + 0x9E3779B97F4A7C15) & _M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def uniform01(seed: int, index: int, draw: int) -> float:
    """A float in [0, 1) from (seed, index, draw), top 53 bits."""
    return (_mix(seed ^ ((index * 0xD1B54A32D192ED03) & _M64) ^ ((draw * 0xA0761D6478BD642F) & _M64)) >> 11) / 2.0**53


def monolayer(size: int, depth: int = 1, contact: float = 10.0, lambda_volume: float = 1.0,
              target_volume: float | None = None, lambda_surface: float = 0.0, target_surface: float = 0.0,
              temperature: float = 10.0, seed: int = 1, side: int = 8, order: int | None = None) -> Start:
    """A periodic lattice tiled by cubes (squares in a plane) of `side`, one
    cell type, no medium: the plain monolayer and its scaling sweep."""
    if target_volume is None:
        target_volume = float(side**2 if depth == 1 else side**3)
    model = Model(
        width=size,
        height=size,
        depth=depth,
        contact=[0.0, contact, contact, contact],
        types=[CellType(), CellType(target_volume=target_volume, lambda_volume=lambda_volume,
                                    target_surface=target_surface, lambda_surface=lambda_surface)],
        temperature=temperature,
        neighbour_order=order if order is not None else (2 if depth == 1 else 3),
        seed=seed,
    )
    return Start.tiled(model, side)


def initial_surface(side: int, depth: int = 1) -> float:
    """Unlike-bond count of one isolated square (cube) of `side` under the
    Moore (26) neighbourhood: what a tiled cell starts with."""
    if depth == 1:
        edge = 4 * (side - 2)
        return float(4 * 5 + edge * 3)
    # a cube: count neighbours outside for every boundary site
    n = 0
    rng = range(side)
    for z in rng:
        for y in rng:
            for x in rng:
                for dz in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        for dx in (-1, 0, 1):
                            if (dx, dy, dz) == (0, 0, 0):
                                continue
                            if not (0 <= x + dx < side and 0 <= y + dy < side and 0 <= z + dz < side):
                                n += 1
    return float(n)


def ensemble_starts(count: int = 64, seed: int = 1, side: int = 8, low: int = 128, high: int = 1024) -> list:
    """`count` monolayer replicas with lattice sides log-uniform from `low` to
    `high` (rounded to whole cells), temperature uniform in [5, 20], contact
    energy uniform in [6, 16] on a 1/64 grid, volume constraint uniform in
    [0.5, 2], each with its own seed."""
    starts = []
    for i in range(count):
        u = [uniform01(seed, i, k) for k in range(4)]
        size = side * round(2 ** (math.log2(low) + u[0] * (math.log2(high) - math.log2(low))) / side)
        size += size % 2
        temperature = 5.0 + 15.0 * u[1]
        contact = 6.0 + round(10.0 * u[2] * 64) / 64
        lambda_volume = 0.5 + 1.5 * u[3]
        starts.append(monolayer(size, contact=contact, lambda_volume=lambda_volume, temperature=temperature,
                                seed=(seed * 1_000_003 + i) & _M64, side=side))
    return starts


def mixed_ensemble_starts(count: int = 64, seed: int = 1, side: int = 8, low: int = 128, high: int = 1024) -> list:
    """`count` replicas alternating the plain monolayer (even places, as
    `ensemble_starts` draws them) and the two-field infection model (odd
    places: `infection_start` on a lattice of the drawn side, a centred block
    of cells covering half of it, 32 immune cells, with the drawn temperature,
    cell-cell contact energy and epithelial volume constraint). The infection
    replicas take INFECTION_RULE. Returns (starts, indices of the infection
    replicas)."""
    plain = ensemble_starts(count, seed, side, low, high)
    starts, infected = [], []
    for i, st in enumerate(plain):
        if i % 2 == 0:
            starts.append(st)
            continue
        size = st.model.width
        inf = infection_start(seed=(seed * 1_000_003 + i) & _M64, size=size, side=side, grid=size // (2 * side))
        m = inf.model
        u = [uniform01(seed, i, k) for k in range(4)]
        m.temperature = 5.0 + 15.0 * u[1]
        j = 6.0 + round(10.0 * u[2] * 64) / 64
        n = m.n_types
        m.contact = [j if (a != 0 and b != 0) else m.contact[a * n + b] for a in range(n) for b in range(n)]
        for t in (1, 2):
            m.types[t].lambda_volume = 0.5 + 1.5 * u[3]
        m.validate()
        starts.append(inf)
        infected.append(i)
    return starts, infected


def adjoint_start(seed: int = 1, size: int = 512, side: int = 8) -> Start:
    """The field-adjoint workload: a periodic `size` lattice tiled by cells of
    `side` (512^2: 4096 cells), types medium, healthy, infected and immune,
    with the infection model's two fields: virus (D 0.05, decay 0.01) and
    interferon (D 0.1, decay 0.005). Infected cells secrete virus at 1.0 and
    interferon at 0.5 per site per MCS, healthy cells take up virus at 0.02;
    immune cells climb interferon (chemotaxis 50) under a length term
    (lambda_L 2, L_target 12). One cell in 16 is infected and 32 are immune,
    picked by the hash of (seed, cell). J is 10 between cells, 16 against the
    medium; lambda_V 1 at the tile volume; T 10."""
    vt = float(side * side)
    cell = dict(target_volume=vt, lambda_volume=1.0)
    n = 4
    contact = [0.0 if (a == 0 and b == 0) else (16.0 if (a == 0 or b == 0) else 10.0)
               for a in range(n) for b in range(n)]
    model = Model(
        width=size,
        height=size,
        contact=contact,
        types=[CellType(), CellType(**cell), CellType(**cell),
               CellType(target_length=12.0, lambda_length=2.0, **cell)],
        temperature=10.0,
        neighbour_order=2,
        seed=seed,
        species=[Species("virus", 0.05, 0.01, 0.0), Species("interferon", 0.1, 0.005, 0.0)],
        secretion=[[0.0, 0.0], [0.0, 0.0], [1.0, 0.5], [0.0, 0.0]],
        uptake=[[0.0, 0.0], [0.02, 0.0], [0.0, 0.0], [0.0, 0.0]],
        chemotaxis=[[0.0, 0.0], [0.0, 0.0], [0.0, 0.0], [0.0, 50.0]],
    )
    start = Start.tiled(model, side)
    cells = start.n_cells
    order = sorted(range(1, cells + 1), key=lambda c: uniform01(seed, c, 7))
    start.cell_type[1:] = 1
    for c in order[: cells // 16]:
        start.cell_type[c] = 2
    for c in order[cells // 16: cells // 16 + 32]:
        start.cell_type[c] = 3
    return start


# The infection rule of the two-field infection model, for set_infection:
# (field, from type, to type, threshold) -- a healthy cell that has taken up
# 5 units of virus is infected.
INFECTION_RULE = (0, 1, 2, 5.0)


def infection_start(seed: int = 1, size: int = 256, side: int = 8, grid: int = 16, immune: int = 32,
                    immune_side: int = 6) -> Start:
    """The two-field infection model on a periodic `size` lattice: a centred
    `grid` x `grid` block of square cells of `side` (healthy, the centre one
    infected), medium elsewhere, and `immune` squares of `immune_side` placed
    uniformly at random in the medium (no overlap) by the hash of (seed,
    attempt). Types: medium, healthy, infected, immune. Fields: virus (D 0.05,
    decay 0.01) and interferon (D 0.1, decay 0.005). Infected cells secrete
    virus at 1.0 and interferon at 0.5 per site per MCS and die at 0.005 per
    MCS; healthy cells take up virus at 0.02; healthy and infected cells divide
    at volume 128; immune cells climb interferon (chemotaxis 50) under a
    length term (lambda_L 2, L_target 12). J is 10 between cells and 16
    against the medium, every cell type keeps its cells in one piece, T 10.
    The switch from healthy to infected is INFECTION_RULE, set on the engine
    (or the replay) separately."""
    vt = float(side * side)
    epithelial = dict(target_volume=vt, lambda_volume=2.0, division_volume=2.0 * vt, connected=True)
    n = 4
    contact = [0.0 if (a == 0 and b == 0) else (16.0 if (a == 0 or b == 0) else 10.0)
               for a in range(n) for b in range(n)]
    model = Model(
        width=size,
        height=size,
        contact=contact,
        types=[CellType(), CellType(**epithelial), CellType(death_rate=0.005, **epithelial),
               CellType(target_volume=float(immune_side * immune_side), lambda_volume=2.0, target_length=12.0,
                        lambda_length=2.0, connected=True)],
        temperature=10.0,
        neighbour_order=2,
        seed=seed,
        species=[Species("virus", 0.05, 0.01, 0.0), Species("interferon", 0.1, 0.005, 0.0)],
        secretion=[[0.0, 0.0], [0.0, 0.0], [1.0, 0.5], [0.0, 0.0]],
        uptake=[[0.0, 0.0], [0.02, 0.0], [0.0, 0.0], [0.0, 0.0]],
        chemotaxis=[[0.0, 0.0], [0.0, 0.0], [0.0, 0.0], [0.0, 50.0]],
    )
    model.validate()
    labels = np.zeros((size, size), dtype=np.uint32)
    origin = (size - grid * side) // 2
    for gy in range(grid):
        for gx in range(grid):
            y0, x0 = origin + gy * side, origin + gx * side
            labels[y0:y0 + side, x0:x0 + side] = 1 + gy * grid + gx
    types = [1] * (grid * grid)
    types[(grid // 2) * grid + grid // 2] = 2
    placed, attempt = 0, 0
    while placed < immune:
        x0 = int(uniform01(seed, attempt, 11) * (size - immune_side + 1))
        y0 = int(uniform01(seed, attempt, 12) * (size - immune_side + 1))
        attempt += 1
        if attempt > 100000:
            raise ValueError("no room for the immune cells")
        if labels[y0:y0 + immune_side, x0:x0 + immune_side].any():
            continue
        placed += 1
        labels[y0:y0 + immune_side, x0:x0 + immune_side] = grid * grid + placed
        types.append(3)
    return Start(model, labels.reshape(-1), np.array([1] + types, dtype=np.uint8))
