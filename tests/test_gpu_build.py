"""Grid index builds on the GPU (radix sort by cell id, then the cell-offset
table) on dense clumps, a single crowded cell, odd and very large grids, and
the README-scale file.  The counts must equal the oracle's (which is pinned
to the reference's own outputs)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle
from spatialjoincountovershells_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _counts(ctx, p, h, r2, grid=None, hint=5.0, periodic=True):
    q = ctx.query(h, r2, periodic=periodic)
    idx = ctx.build_index(p, radius_hint=hint, grid=grid)
    q.count(idx)
    out = q.read_counts()
    idx.destroy()
    q.destroy()
    return out


def _halos_around(rng, centre, spread, n_near, n_far):
    near = centre + rng.normal(0, spread, size=(n_near, 3))
    far = rng.uniform(0, 1000, size=(n_far, 3))
    return np.concatenate([near, far, [[0, 0, 0], [999.99, 0.5, 500]]]).astype(np.float32) % np.float32(1000)


def test_dense_buckets(ctx):
    """600k particles, 80 % in a ball of radius 1: a few cells hold most of
    the particles."""
    rng = np.random.default_rng(61)
    n = 600_000
    p = rng.uniform(0, 1000, size=(n, 3))
    k = int(0.8 * n)
    d = rng.normal(size=(k, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    p[:k] = np.array([500.0, 500.0, 500.0]) + d * rng.uniform(0, 1, size=(k, 1)) ** (1 / 3)
    p = p.astype(np.float32)
    h = _halos_around(rng, np.array([500.0, 500.0, 500.0]), 2.0, 300, 700)
    r2 = nat.radius_table(0.001, 5.0, 40)
    assert np.array_equal(_counts(ctx, p, h, r2), oracle.count(p, h, r2))


def test_one_cell_holds_every_particle(ctx):
    rng = np.random.default_rng(62)
    p = np.empty((300_000, 3), np.float32)
    p[:] = (123.25, 456.5, 789.75)
    p[:100] = rng.uniform(0, 1000, size=(100, 3))
    h = np.array([[123.25, 456.5, 789.75], [123.0, 456.0, 790.0], [500, 500, 500], [0, 0, 0]], np.float32)
    r2 = nat.radius_table(0.01, 5.0, 12)
    got = _counts(ctx, p, h, r2)
    want = oracle.count(p, h, r2)
    assert np.array_equal(got, want)
    assert got[0].sum() >= 299_900


def test_clustered_file_matches_oracle(ctx):
    p = nat.gen_clustered_particles(63, 2_000_000)
    h = nat.gen_clustered_halos(64, 4000)
    r2 = nat.radius_table(0.01, 20.0, 64)
    assert np.array_equal(_counts(ctx, p, h, r2, hint=20.0), oracle.count(p, h, r2))


@pytest.mark.parametrize("grid", [(2048, 512, 512), (4096, 512, 600), (1, 1, 1), (3, 1, 70001 // 3), (5, 1, 1)])
def test_large_tiny_and_odd_grids(grid, ctx):
    """2^29 and more than 2^30 cells (31-bit cell ids: four 8-bit passes); one
    cell; small and odd cell counts."""
    rng = np.random.default_rng(65)
    p = rng.uniform(0, 1000, size=(120_000, 3)).astype(np.float32)
    h = rng.uniform(0, 1000, size=(1500, 3)).astype(np.float32)
    h[:20] = rng.choice([0.0, 1000.0, 4.0, 996.0], size=(20, 3))
    r2 = nat.radius_table(0.01, 12.0, 30)
    assert np.array_equal(_counts(ctx, p, h, r2, grid=grid, hint=12.0), oracle.count(p, h, r2))


def test_build_at_the_automatic_readme_scale_grid(ctx):
    """1e8 uniform particles (the README-scale file): 1000 x 400 x 400 cells
    (28-bit cell ids: segments of 1024 cells under two 9-bit partition
    passes); 20000 halos including face and corner halos checked against the
    oracle."""
    import torch
    n = 100_000_000
    p = nat.gen_uniform_particles(1, 1, n)
    dp = torch.from_numpy(p).cuda()
    idx = ctx.build_index(dp, radius_hint=5.0)
    assert idx.grid == (1000, 400, 400)
    rng = np.random.default_rng(66)
    h = nat.gen_uniform_halos(2, 20000)["point"].copy()
    h[:600] = rng.choice([0.0, 999.999, 1.5, 998.5, 4.99, 995.01], size=(600, 3))
    r2 = nat.radius_table(0.001, 5.0, 40)
    q = ctx.query(h, r2)
    q.count(idx)
    got = q.read_counts()
    q.destroy()
    idx.destroy()
    del dp
    torch.cuda.empty_cache()
    assert np.array_equal(got, oracle.count(p, h, r2))
