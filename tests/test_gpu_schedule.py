"""Count schedules on the GPU: the persistent work queue and the autotuner.

A schedule decides only which warp counts which halo (or which piece of a
heavy halo); the counts must be bit-identical to the static schedule's and to
the oracle's for every piece size, including pieces so small that every
halo is split across many warps.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import oracle
from spatialjoincountovershells_b200 import _native as nat

pytestmark = pytest.mark.gpu

QUEUES = [dict(piece=8192, max_pieces=64), dict(piece=1, max_pieces=7, single=1), dict(piece=64, max_pieces=65536),
          dict(piece=1 << 30, max_pieces=1, single=1 << 30), dict(piece=256, max_pieces=3, single=2)]


def counts(ctx, p, h, r2, periodic=True, grid=None, **sched):
    q = ctx.query(h, r2, periodic=periodic)
    q.set_schedule(**sched)
    hint = math.sqrt(float(r2[-1])) if np.isfinite(r2[-1]) else 10.0
    idx = ctx.build_index(p, radius_hint=hint, grid=grid)
    q.count(idx)
    out = q.read_counts()
    idx.destroy()
    q.destroy()
    return out


@pytest.mark.parametrize("qs", QUEUES)
def test_queue_matches_oracle_on_clustered_data(qs, ctx):
    p = nat.gen_clustered_particles(7, 300000)
    h = nat.gen_clustered_halos(8, 5000)
    r2 = nat.radius_table(0.01, 20, 64)
    want = oracle.count(p, h, r2)
    got = counts(ctx, p, h, r2, mode=nat.SCHED_QUEUE, **qs)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("qs", QUEUES)
@pytest.mark.parametrize("seed", [31, 32])
def test_queue_matches_static_on_random_inputs(seed, qs, ctx):
    rng = np.random.default_rng(seed)
    p = rng.uniform(0, 1000, size=(int(rng.integers(1, 80000)), 3)).astype(np.float32)
    p[: len(p) // 3] = (rng.normal(200, 3, size=(len(p) // 3, 3)) % 1000).astype(np.float32)
    nh = int(rng.integers(1, 4000))
    h = rng.uniform(0, 1000, size=(nh, 3)).astype(np.float32)
    h[: nh // 3] = rng.normal(200, 2, size=(nh // 3, 3)).astype(np.float32) % 1000
    h[: nh // 10] = rng.choice([0.0, 1000.0, 2.0, 998.0, 999.99994], size=(nh // 10, 3))
    r2 = nat.radius_table(0.001, 15, 40)
    for periodic in (True, False):
        want = counts(ctx, p, h, r2, periodic=periodic, mode=nat.SCHED_STATIC)
        got = counts(ctx, p, h, r2, periodic=periodic, mode=nat.SCHED_QUEUE, **qs)
        assert np.array_equal(got, want), (seed, periodic)
        if seed == 31:
            assert np.array_equal(want, oracle.count(p, h, r2, periodic=periodic))


def test_queue_with_tables_outside_the_fast_path_and_odd_grids(ctx):
    rng = np.random.default_rng(33)
    p = rng.uniform(-20, 1020, size=(20000, 3)).astype(np.float32)
    p[:4] = [[np.nan, 1, 1], [np.inf, 2, 2], [0, np.nan, 0], [1e30, 4, 4]]
    h = rng.uniform(0, 1000, size=(300, 3)).astype(np.float32)
    h[:4] = [[np.nan, 500, 500], [np.inf, 500, 500], [-5, -5, -5], [1005, 1005, 1005]]
    for r2 in [np.array([400.0, 100.0, 2500.0], np.float32), np.linspace(1, 3000, 2000).astype(np.float32),
               nat.radius_table(0.5, 40, 12)]:
        for grid in [None, (7, 3, 5), (300, 300, 300)]:
            want = oracle.count(p, h, r2, brute=True)
            got = counts(ctx, p, h, r2, grid=grid, mode=nat.SCHED_QUEUE, piece=32, max_pieces=5, single=4)
            assert np.array_equal(got, want), (r2[:3], grid)


def test_autotune_keeps_counts_and_remembers_the_choice(ctx):
    p = nat.gen_clustered_particles(9, 400000)
    h = nat.gen_clustered_halos(10, 20000)
    r2 = nat.radius_table(0.01, 20, 64)
    idx = ctx.build_index(p, radius_hint=20.0)
    q = ctx.query(h, r2)
    q.count(idx)
    before = q.read_counts()
    res = ctx.autotune(q, idx)
    assert len(res["trial_ms"]) == 6 and all(t > 0 for t in res["trial_ms"])
    assert res["chosen"]["mode"] in (nat.SCHED_STATIC, nat.SCHED_QUEUE)
    assert q.schedule() == res["chosen"]
    assert np.array_equal(q.read_counts(), before)  # tuning did not touch the counts
    q.count(idx)
    assert np.array_equal(q.read_counts(), 2 * before)
    # a new query of the same shape on AUTO picks the tuned schedule and counts the same
    q2 = ctx.query(h, r2)
    assert q2.schedule()["mode"] == nat.SCHED_AUTO
    q2.count(idx)
    assert np.array_equal(q2.read_counts(), before)
    for o in (q, q2, idx):
        o.destroy()


def test_schedule_arguments_are_validated(ctx):
    q = ctx.query(np.zeros((1, 3), np.float32), nat.radius_table(0.1, 1, 4))
    for kw in [dict(mode=3), dict(mode=-1), dict(mode=nat.SCHED_QUEUE, max_pieces=70000),
               dict(mode=nat.SCHED_QUEUE, piece=(1 << 30) + 1)]:
        with pytest.raises(nat.SjcsError):
            q.set_schedule(**kw)
    q.destroy()


def test_autotune_on_morton_indexes(ctx):
    rng = np.random.default_rng(34)
    p = rng.uniform(0, 1000, size=(50000, 3)).astype(np.float32)
    h = rng.uniform(0, 1000, size=(2000, 3)).astype(np.float32)
    r2 = nat.radius_table(0.001, 5, 40)
    for kind in (nat.INDEX_MORTON, nat.INDEX_LEARNED):
        idx = ctx.build_index(p, radius_hint=5.0, kind=kind)
        q = ctx.query(h, r2)
        res = ctx.autotune(q, idx)
        assert len(res["trial_ms"]) == 6 and res["chosen"]["mode"] in (nat.SCHED_STATIC, nat.SCHED_QUEUE)
        q.count(idx)
        assert np.array_equal(q.read_counts(), oracle.count(p, h, r2))
        idx.destroy()
        q.destroy()


@pytest.mark.parametrize("kind", [nat.INDEX_MORTON, nat.INDEX_LEARNED])
@pytest.mark.parametrize("qs", QUEUES)
def test_queue_on_morton_forms_matches_oracle(kind, qs, ctx):
    p = nat.gen_clustered_particles(17, 200000)
    h = nat.gen_clustered_halos(18, 3000)
    rng = np.random.default_rng(19)
    h["point"][:30] = rng.choice([0.0, 1000.0, 2.0, 998.0], size=(30, 3))
    for r2, per in [(nat.radius_table(0.01, 20, 64), True), (nat.radius_table(0.001, 5, 40), False),
                    (np.array([400.0, 100.0, 2500.0], np.float32), True)]:
        q = ctx.query(h, r2, periodic=per)
        q.set_schedule(nat.SCHED_QUEUE, **qs)
        idx = ctx.build_index(p, radius_hint=10.0, kind=kind)
        q.count(idx)
        got = q.read_counts()
        idx.destroy()
        q.destroy()
        assert np.array_equal(got, oracle.count(p, h, r2, periodic=per, brute=len(r2) < 10)), (kind, r2[:3])
