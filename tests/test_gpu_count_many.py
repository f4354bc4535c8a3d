"""Several indexes counted in one pass (sjcs_query_count_many): the counts must
be the oracle's sum over the files -- the reference's += over its file loop
(src/astr_rcount/main.c:651) -- whether the run is fused (grid indexes of one
cell grid, static schedule) or falls back to one count per index."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle
from spatialjoincountovershells_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _files(seeds, n):
    out = []
    for s in seeds:
        rng = np.random.default_rng(s)
        out.append(rng.uniform(0, 1000, size=(n, 3)).astype(np.float32))
    return out


def _halos(seed, m):
    rng = np.random.default_rng(seed)
    h = rng.uniform(0, 1000, size=(m, 3)).astype(np.float32)
    h[:40] = rng.choice([0.0, 999.99, 3.0, 997.0, 500.0], size=(40, 3))
    return h


@pytest.fixture(scope="module")
def six_files():
    files = _files(range(700, 706), 40000)
    h = _halos(699, 3000)
    r2 = nat.radius_table(0.01, 12.0, 30)
    per_file = [oracle.count(f, h, r2) for f in files]
    return files, h, r2, per_file


def _count_many(ctx, files, h, r2, hint=12.0, sched=None, fold_limit=None, **build):
    q = ctx.query(h, r2)
    if sched is not None:
        q.set_schedule(sched)
    if fold_limit is not None:
        q.set_fold_limit(fold_limit)
    idx = [ctx.build_index(f, radius_hint=hint, **build) for f in files]
    q.count_many(idx)
    out = q.read_counts()
    folds = q.folds
    for i in idx:
        i.destroy()
    q.destroy()
    return out, folds


def test_fused_three_files_equal_the_oracle_sum(six_files, ctx):
    files, h, r2, per_file = six_files
    got, _ = _count_many(ctx, files[:3], h, r2, sched=nat.SCHED_STATIC)
    assert np.array_equal(got, sum(per_file[:3]))


def test_six_files_run_as_four_and_two(six_files, ctx):
    files, h, r2, per_file = six_files
    got, _ = _count_many(ctx, files, h, r2, sched=nat.SCHED_STATIC)
    assert np.array_equal(got, sum(per_file))


def test_mixed_grids_and_kinds_fall_back(six_files, ctx):
    """A file of another size has another automatic grid, and a Morton index
    is not a grid index: each is counted on its own, the rest fused."""
    files, h, r2, per_file = six_files
    small = files[5][:17000]
    q = ctx.query(h, r2)
    q.set_schedule(nat.SCHED_STATIC)
    idx = [ctx.build_index(files[0], radius_hint=12.0), ctx.build_index(small, radius_hint=12.0),
           ctx.build_index(files[1], radius_hint=12.0),
           ctx.build_index(files[2], radius_hint=12.0, kind=nat.INDEX_MORTON),
           ctx.build_index(files[3], radius_hint=12.0), ctx.build_index(files[4], radius_hint=12.0)]
    q.count_many(idx)
    got = q.read_counts()
    for i in idx:
        i.destroy()
    q.destroy()
    want = per_file[0] + oracle.count(small, h, r2) + per_file[1] + per_file[2] + per_file[3] + per_file[4]
    assert np.array_equal(got, want)


def test_fused_runs_split_at_the_fold_limit(six_files, ctx):
    """Two files fit under the lowered limit, a third would not: the run is
    split and the query folds between runs; totals stay exact."""
    files, h, r2, per_file = six_files
    got, folds = _count_many(ctx, files, h, r2, sched=nat.SCHED_STATIC, fold_limit=90000)
    assert folds >= 2
    assert np.array_equal(got, sum(per_file))


def test_queue_schedule_counts_each_index(six_files, ctx):
    files, h, r2, per_file = six_files
    got, _ = _count_many(ctx, files[:3], h, r2, sched=nat.SCHED_QUEUE)
    assert np.array_equal(got, sum(per_file[:3]))


@pytest.mark.parametrize("kind", ["big", "first_match", "nonperiodic"])
def test_fused_other_kernel_variants(kind, ctx):
    """Tables past the shared-memory limit (global counters), a
    non-monotone table (first-match scan) and the non-periodic entry."""
    files = _files(range(710, 713), 25000)
    h = _halos(709, 1500)
    periodic = True
    if kind == "big":
        r2 = nat.radius_table(0.01, 10.0, 1500)
    elif kind == "first_match":
        r2 = nat.radius_table(0.01, 10.0, 20)
        r2[[3, 11]] = r2[[11, 3]]
    else:
        r2 = nat.radius_table(0.01, 10.0, 20)
        periodic = False
    q = ctx.query(h, r2, periodic=periodic)
    q.set_schedule(nat.SCHED_STATIC)
    idx = [ctx.build_index(f, radius_hint=10.0) for f in files]
    q.count_many(idx)
    got = q.read_counts()
    for i in idx:
        i.destroy()
    q.destroy()
    want = sum(oracle.count(f, h, r2, periodic=periodic) for f in files)
    assert np.array_equal(got, want)


def test_fresh_query_reads_zeros_and_fused_passes_add(six_files, ctx):
    """Every read of a new query before a count gives zeros (host uint64,
    host uint32 and the device pointer), and fused passes add up and
    restart after a reset."""
    import torch
    files, h, r2, per_file = six_files
    q = ctx.query(h, r2)
    assert not q.read_counts().any()
    buf = nat.PinnedBuffer((len(h), len(r2)), np.uint32)
    buf.array[:] = 7
    q.read_counts32_async(buf.array)
    q.wait_read()
    assert not buf.array.any()
    q.destroy()
    q = ctx.query(h, r2)
    m = len(h) * len(r2)

    class _U32:  # the accumulators as a CUDA array for torch to copy
        __cuda_array_interface__ = {"shape": (m,), "typestr": "<i4", "data": (q.device_counts_ptr, False),
                                    "version": 3}

    dev = torch.as_tensor(_U32(), device="cuda").clone()
    torch.cuda.synchronize()
    assert not dev.any()
    q.destroy()
    q = ctx.query(h, r2)
    q.set_schedule(nat.SCHED_STATIC)
    idx = [ctx.build_index(f, radius_hint=12.0) for f in files[:3]]
    q.count_many(idx)
    assert np.array_equal(q.read_counts(), sum(per_file[:3]))
    q.count_many(idx)
    assert np.array_equal(q.read_counts(), 2 * sum(per_file[:3]))
    q.reset()
    q.count_many(idx)
    assert np.array_equal(q.read_counts(), sum(per_file[:3]))
    for i in idx:
        i.destroy()
    q.destroy()
    buf.free()
