"""64-bit count totals on the device (the reference's ulong_t counts over any
number of particle files, src/astr_rcount/main.c:651).

A query accumulates in uint32 and folds into 64-bit totals before a count call
could carry an accumulator past its fold limit.  A lowered limit (the test
hook sjcs_query_set_fold_limit) makes folds happen every few files on small
inputs, and the totals must stay equal to the oracle's; one case takes a
single accumulator past 2^32 for real.
"""
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


@pytest.fixture(scope="module")
def many_files():
    files = _files(range(300, 310), 30000)
    rng = np.random.default_rng(299)
    h = rng.uniform(0, 1000, size=(2000, 3)).astype(np.float32)
    h[:30] = rng.choice([0.0, 999.99, 2.0, 998.0], size=(30, 3))
    r2 = nat.radius_table(0.01, 20.0, 30)
    per_file = [oracle.count(f, h, r2) for f in files]
    return files, h, r2, per_file


@pytest.mark.parametrize("sched", [nat.SCHED_STATIC, nat.SCHED_QUEUE])
def test_folds_keep_totals_exact_across_many_files(many_files, ctx, sched):
    files, h, r2, per_file = many_files
    q = ctx.query(h, r2)
    q.set_schedule(sched)
    q.set_fold_limit(70000)  # R = 20: each file adds at most 30000 -> a fold every second file
    for k, f in enumerate(files):
        idx = ctx.build_index(f, radius_hint=20.0)
        q.count(idx)
        idx.destroy()
        if k == 4:
            assert np.array_equal(q.read_counts(), sum(per_file[:5]))
    assert q.folds == 4
    want = sum(per_file)
    assert np.array_equal(q.read_counts(), want)
    buf = nat.PinnedBuffer((len(h), len(r2)), np.uint64)
    q.read_counts_async(buf.array)
    q.wait_read()
    assert np.array_equal(buf.array, want)
    acc = np.ones_like(want)
    q.read_counts(out=acc, accumulate=True)
    assert np.array_equal(acc, want + 1)
    buf.free()
    q.reset()
    assert q.folds == 0
    idx = ctx.build_index(files[0], radius_hint=20.0)
    q.count(idx)
    assert np.array_equal(q.read_counts(), per_file[0])
    idx.destroy()
    q.destroy()


def test_uint32_read_is_exact_until_a_fold(many_files, ctx):
    """The uint32 read-back copies the accumulators as they are: equal to the
    oracle's totals while no fold has happened, refused after one."""
    files, h, r2, per_file = many_files
    q = ctx.query(h, r2)
    q.set_fold_limit(70000)
    buf = nat.PinnedBuffer((len(h), len(r2)), np.uint32)
    for k in range(2):
        idx = ctx.build_index(files[k], radius_hint=20.0)
        q.count(idx)
        idx.destroy()
    assert q.folds == 0
    q.read_counts32_async(buf.array)
    q.wait_read()
    assert np.array_equal(buf.array, per_file[0] + per_file[1])
    idx = ctx.build_index(files[2], radius_hint=20.0)
    q.count(idx)
    idx.destroy()
    assert q.folds == 1
    with pytest.raises(nat.SjcsError):
        q.read_counts32_async(buf.array)
    assert np.array_equal(q.read_counts(), sum(per_file[:3]))
    buf.free()
    q.destroy()


def test_fold_with_radius_beyond_half_box(ctx):
    """R >= 499: a particle can lie in several images' boxes, so one file may add
    8n to an accumulator; the query folds on that bound."""
    files = _files((320, 321, 322), 4000)
    rng = np.random.default_rng(323)
    h = rng.uniform(0, 1000, size=(60, 3)).astype(np.float32)
    r2 = nat.radius_table(1.0, 600.0, 12)
    q = ctx.query(h, r2)
    q.set_fold_limit(8 * 4000 + 5)  # every file needs a fold first
    want = np.zeros((len(h), len(r2)), np.uint64)
    for f in files:
        idx = ctx.build_index(f, radius_hint=600.0)
        q.count(idx)
        idx.destroy()
        want += oracle.count(f, h, r2)
    assert q.folds == 2
    assert np.array_equal(q.read_counts(), want)
    q.destroy()


def test_captured_steps_fold_too(many_files, ctx):
    files, h, r2, per_file = many_files
    n = len(files[0])
    q = ctx.query(h, r2)
    q.set_fold_limit(70000)
    st = ctx.step(q, n, radius_hint=20.0)
    for f in files[:6]:
        st.buffer[:] = f
        st.launch().wait()
    assert q.folds == 2
    assert np.array_equal(q.read_counts(), sum(per_file[:6]))
    st.destroy()
    q.destroy()


def test_one_call_beyond_the_limit_is_refused(many_files, ctx):
    files, h, r2, _ = many_files
    q = ctx.query(h, r2)
    q.set_fold_limit(1000)
    idx = ctx.build_index(files[0], radius_hint=20.0)
    with pytest.raises(nat.SjcsError) as e:
        q.count(idx)
    assert e.value.code == 1
    with pytest.raises(nat.SjcsError):
        q.set_fold_limit(0)
    with pytest.raises(nat.SjcsError):
        q.set_fold_limit(1 << 32)
    idx.destroy()
    q.destroy()


def test_an_accumulator_past_two_to_the_32(ctx):
    """65 passes over 2^26 particles that all land in one shell of one halo:
    65 * 2^26 = 4362076160 > 2^32 - 1, so a 32-bit accumulator alone would
    have wrapped to 2^26."""
    import torch
    n = 1 << 26
    g = torch.Generator(device="cuda").manual_seed(7)
    p = torch.rand((n, 3), device="cuda", dtype=torch.float32, generator=g) * 800.0 + 100.0
    idx = ctx.build_index(p, radius_hint=0.0)
    h = np.array([[500.0, 500.0, 500.0]], np.float32)
    r2 = np.array([1.0e6], np.float32)  # every particle is within 700 of the halo
    q = ctx.query(h, r2, periodic=False)
    q.set_schedule(nat.SCHED_QUEUE, piece=8192, max_pieces=8192)
    for _ in range(65):
        q.count(idx)
    assert q.folds == 1
    got = q.read_counts()
    assert got.dtype == np.uint64 and int(got[0, 0]) == 65 * n
    idx.destroy()
    q.destroy()
    del p
    torch.cuda.empty_cache()
