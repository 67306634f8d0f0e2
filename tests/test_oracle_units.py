"""The reference's own unit tests and known answers, run on the oracle.

Each test restates a test of glazier-core (file:line given) so the oracle is
held to the same fixtures the reference holds itself to.
"""

from __future__ import annotations

import numpy as np

from conftest import sheet_model, tiled, with_species
from oracle import serial as S


def test_a_plane_and_a_volume_take_their_neighbour_counts():
    # lattice.rs:258-270
    assert len(S.offsets(2, 1)) == 8 and len(S.offsets(1, 1)) == 4 and len(S.offsets(3, 1)) == 8
    assert len(S.offsets(1, 4)) == 6 and len(S.offsets(2, 4)) == 18 and len(S.offsets(3, 4)) == 26


def test_a_seed_reproduces_its_stream_and_below_covers_its_range():
    # rng.rs:78-96
    assert np.array_equal(S.xoshiro_stream(3, 100), S.xoshiro_stream(3, 100))
    counts = np.bincount(S.xoshiro_below(11, 5, 10_000).astype(np.int64), minlength=5)
    assert counts.size == 5 and (counts > 1500).all()


def test_the_xoshiro_stream_matches_the_published_generator():
    # xoshiro256++ seeded through SplitMix64 (rng.rs:17-45), restated in numpy.
    def splitmix(z):
        out = []
        for _ in range(4):
            z = (z + 0x9E3779B97F4A7C15) & (2**64 - 1)
            x = z
            x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & (2**64 - 1)
            x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & (2**64 - 1)
            out.append(x ^ (x >> 31))
        return out

    def rotl(x, k):
        return ((x << k) | (x >> (64 - k))) & (2**64 - 1)

    s = splitmix(123456789)
    want = []
    for _ in range(16):
        want.append((rotl((s[0] + s[3]) & (2**64 - 1), 23) + s[0]) & (2**64 - 1))
        t = (s[1] << 17) & (2**64 - 1)
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t
        s[3] = rotl(s[3], 45)
    assert S.xoshiro_stream(123456789, 16).tolist() == want


def _filled(w, h, d):
    return [(x, y, z) for z in range(d) for y in range(h) for x in range(w)]


def test_a_strip_reads_about_its_own_extent():
    # moments.rs:218-223: a 1 by 16 strip has length 4 sqrt((16^2 - 1)/12) = 18.47
    length, _, _ = S.moments_of(_filled(1, 16, 1))
    assert abs(length - 18.47) < 0.05


def test_rectangles_squares_and_columns_read_their_lengths():
    # moments.rs:205-231
    square, _, _ = S.moments_of(_filled(8, 8, 1))
    wide, _, _ = S.moments_of(_filled(16, 4, 1))
    tall, _, _ = S.moments_of(_filled(4, 16, 1))
    assert square > 0 and wide > square and abs(wide - tall) < 1e-6
    column, _, axis = S.moments_of(_filled(1, 1, 16))
    strip, _, _ = S.moments_of(_filled(1, 16, 1))
    assert abs(column - strip) < 1e-6 and abs(axis[2]) > 0.99


def test_anisotropy_points_along_the_long_axis():
    # moments.rs:271-278
    _, (a, b), _ = S.moments_of(_filled(8, 8, 1))
    assert abs(a) < 1e-12 and abs(b) < 1e-12
    _, (a, b), _ = S.moments_of(_filled(16, 2, 1))
    assert a > 0.9 and abs(b) < 1e-12
    _, (a, _), _ = S.moments_of(_filled(2, 16, 1))
    assert a < -0.9


def test_unwrapping_pulls_a_site_across_the_edge():
    # moments.rs:254-268
    x, y, _ = S.unwrap_about((1.0, 1.0, 0.0), (63.0, 1.0, 0.0), (64.0, 64.0, 1.0))
    assert abs(x + 1.0) < 1e-12 and abs(y - 1.0) < 1e-12
    _, _, z = S.unwrap_about((1.0, 1.0, 0.0), (0.0, 0.0, 0.0), (64.0, 64.0, 1.0))
    assert z == 0.0


def _plane_with(pattern):
    lab = np.zeros(81, dtype=np.uint32)
    for x, y in pattern:
        lab[(4 + y) * 9 + (4 + x)] = 1
    return lab


def test_local_connectivity_patterns():
    # connectivity.rs:99-152
    target = 4 * 9 + 4
    solid = [(-1, -1), (0, -1), (1, -1), (-1, 0), (1, 0), (-1, 1), (0, 1), (1, 1)]
    assert S.locally_connected(_plane_with(solid), 9, 9, 1, target, 1)
    assert not S.locally_connected(_plane_with([(-1, 0), (1, 0)]), 9, 9, 1, target, 1)
    assert S.locally_connected(_plane_with([(1, 0)]), 9, 9, 1, target, 1)
    assert S.locally_connected(_plane_with([(1, 0), (1, 1)]), 9, 9, 1, target, 1)
    vol = np.zeros(9 * 9 * 9, dtype=np.uint32)
    idx = lambda x, y, z: (z * 9 + y) * 9 + x  # noqa: E731
    vol[idx(4, 4, 3)] = vol[idx(4, 4, 5)] = 1
    assert not S.locally_connected(vol, 9, 9, 9, idx(4, 4, 4), 1)
    vol[idx(5, 4, 4)] = 1
    assert S.locally_connected(vol, 9, 9, 9, idx(4, 4, 4), 1)


def test_substeps_follow_the_stability_limit():
    # field.rs:255-270
    assert [S.substeps_for(d, 2) for d in (0.0, 0.25, 0.26, 2.0)] == [1, 1, 2, 8]
    assert S.substeps_for(1.0, 2) == 4 and S.substeps_for(1.0, 3) == 6


def _field_sheet(w, h, diffusion, decay, initial, secretion=0.0, uptake=0.0, all_medium=True):
    m = sheet_model(width=w, height=h)
    with_species(m, [("a", diffusion, decay, initial)], [[0.0], [secretion]], [[0.0], [uptake]], [[0.0], [0.0]])
    labels = np.zeros(w * h, dtype=np.uint32)
    labels[0] = 1  # a cell somewhere so the start is valid
    o = S.SerialOracle(m, labels=labels, cell_type=[0, 1])
    return o


def test_a_uniform_field_stays_uniform_and_a_point_source_conserves():
    # field.rs:178-215: driven through whole steps with a frozen lattice (T tiny)
    o = _field_sheet(16, 16, 0.2, 0.0, 3.0)
    o.step(1)
    assert np.allclose(o.field(0), 3.0, atol=1e-12)
    o = _field_sheet(16, 16, 0.2, 0.0, 0.0)
    f = np.zeros(256)
    f[8 * 16 + 8] = 100.0
    o.set_field(0, f)
    o.step(20)
    assert abs(o.field(0).sum() - 100.0) < 1e-9


def test_decay_removes_its_fraction_and_exchange_follows_the_owner():
    # field.rs:240-253 and 319-345: 1 + 2 = 3, less half of it, is 1.5
    o = _field_sheet(8, 8, 0.0, 0.1, 1.0)
    o.step(1)
    assert abs(o.field(0)[5] - 0.9) < 1e-12
    o = _field_sheet(8, 8, 0.0, 0.0, 1.0, secretion=2.0, uptake=0.5)
    o.step(1)
    f = o.field(0)
    owned = o.labels() == 1
    assert np.allclose(f[owned], 1.5, atol=1e-12) and np.allclose(f[~owned], 1.0, atol=1e-12)


def _energy_check(model, rng_seed, steps, probes):
    start = tiled(model, 8)
    o = S.SerialOracle.from_start(start)
    rng = np.random.default_rng(rng_seed)
    checked = 0
    for _ in range(steps):
        o.step(1)
        labels = o.labels()
        volumes = o.volumes()
        for _ in range(probes):
            target = int(rng.integers(labels.size))
            source = int(rng.integers(labels.size))
            old, new = labels[target], labels[source]
            if old == new or (old != 0 and volumes[old] <= 1):
                continue
            predicted = o.delta_energy(target, int(new))
            before = o.energy()
            after = S.SerialOracle(model, labels=np.where(np.arange(labels.size) == target, new, labels),
                                   cell_type=o.cell_types())
            measured = after.energy() - before
            assert abs(predicted - measured) < 1e-9, (predicted, measured)
            checked += 1
    assert checked > 20


def test_the_incremental_delta_matches_a_full_recomputation():
    # cpu_reference.rs:31-65 (contact and volume) and 77-110 (surface)
    _energy_check(sheet_model(32, 32, seed=42), 5, 6, 15)
    _energy_check(sheet_model(32, 32, seed=42, target_surface=28.0, lambda_surface=1.0), 9, 6, 15)


def test_surface_bookkeeping_survives_a_run():
    # cpu_reference.rs:113-119
    o = S.SerialOracle.from_start(tiled(sheet_model(48, 48, seed=42, target_surface=28.0, lambda_surface=1.0)))
    o.step(60)
    assert np.array_equal(o.surfaces(), o.recounted_surfaces())
