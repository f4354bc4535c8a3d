"""Asynchronous count read-back (sjcs_query_read_counts_async / sjcs_query_wait_read).

A queued read must deliver exactly the counts accumulated when it was queued:
what sjcs_query_read_counts returns at that point, whatever is queued on the
query afterwards (counts, resets, captured steps, destroy), and it must refuse
host memory that a copy engine cannot write asynchronously.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle
from spatialjoincountovershells_b200 import _native as nat

pytestmark = pytest.mark.gpu

NR = 30


def _case(seed, n=60000, nh=3000):
    rng = np.random.default_rng(seed)
    p = rng.uniform(0, 1000, size=(n, 3)).astype(np.float32)
    h = rng.uniform(0, 1000, size=(nh, 3)).astype(np.float32)
    return p, h


@pytest.fixture(scope="module")
def case():
    p1, h = _case(50)
    p2, _ = _case(51)
    r2 = nat.radius_table(0.01, 20, NR)
    return p1, p2, h, r2, oracle.count(p1, h, r2), oracle.count(p2, h, r2)


def _pinned(nh):
    buf = nat.PinnedBuffer((nh, NR), np.uint64)
    buf.array[:] = 0xdeadbeef  # a read that did not land shows
    return buf


def test_async_read_equals_blocking_read(case, ctx):
    p1, _, h, r2, c1, _ = case
    q = ctx.query(h, r2)
    idx = ctx.build_index(p1, radius_hint=20)
    q.count(idx)
    buf = _pinned(len(h))
    q.read_counts_async(buf.array)
    q.wait_read()
    assert np.array_equal(buf.array, c1)
    assert np.array_equal(q.read_counts(), c1)
    assert q.timing()["d2h_ms"] > 0
    idx.destroy()
    q.destroy()


def test_later_counts_and_resets_wait_for_the_read(case, ctx):
    p1, p2, h, r2, c1, c2 = case
    q = ctx.query(h, r2)
    i1 = ctx.build_index(p1, radius_hint=20)
    i2 = ctx.build_index(p2, radius_hint=20)
    a, b, c = _pinned(len(h)), _pinned(len(h)), _pinned(len(h))
    q.count(i1)
    q.read_counts_async(a.array)  # after file 1
    q.count(i2)                   # queued at once; runs after the read
    q.read_counts_async(b.array)  # after files 1 and 2
    q.reset()
    q.count(i2)
    q.read_counts_async(c.array)  # file 2 only
    q.wait_read()
    assert np.array_equal(a.array, c1)
    assert np.array_equal(b.array, c1 + c2)
    assert np.array_equal(c.array, c2)
    for x in (i1, i2, q):
        x.destroy()


def test_destroy_with_a_read_in_flight(case, ctx):
    p1, _, h, r2, c1, _ = case
    q = ctx.query(h, r2)
    idx = ctx.build_index(p1, radius_hint=20)
    q.count(idx)
    idx.destroy()
    buf = _pinned(len(h))
    q.read_counts_async(buf.array)
    q.destroy()  # frees the counts only after the read
    assert np.array_equal(buf.array, c1)


def test_captured_step_after_a_read(case, ctx):
    p1, p2, h, r2, c1, c2 = case
    q = ctx.query(h, r2)
    st = ctx.step(q, len(p1), radius_hint=20.0)
    st.buffer[:] = p1
    st.launch().wait()
    buf = _pinned(len(h))
    q.read_counts_async(buf.array)
    st.buffer[:] = p2  # the previous replay is done; the buffer is free
    st.launch().wait()
    q.wait_read()
    assert np.array_equal(buf.array, c1)
    assert np.array_equal(q.read_counts(), c1 + c2)
    st.destroy()
    q.destroy()


def test_pageable_memory_is_refused_and_empty_queries_pass(case, ctx):
    p1, _, h, r2, _, _ = case
    q = ctx.query(h, r2)
    with pytest.raises(nat.SjcsError):
        q.read_counts_async(np.zeros((len(h), NR), np.uint64))
    q.wait_read()  # nothing pending
    q.destroy()
    e = ctx.query(np.zeros((0, 3), np.float32), r2)
    e.read_counts_async(np.zeros((0, NR), np.uint64))  # nothing to copy
    e.wait_read()
    e.destroy()


def test_reads_of_two_queries_in_flight(case, ctx):
    p1, p2, h, r2, c1, c2 = case
    qa, qb = ctx.query(h, r2), ctx.query(h, r2)
    i1 = ctx.build_index(p1, radius_hint=20)
    i2 = ctx.build_index(p2, radius_hint=20)
    qa.count(i1)
    qb.count(i2)
    a, b = _pinned(len(h)), _pinned(len(h))
    qa.read_counts_async(a.array)
    qb.read_counts_async(b.array)
    qa.count(i2)  # waits on the device for qa's read only
    qb.wait_read()
    qa.wait_read()
    assert np.array_equal(a.array, c1)
    assert np.array_equal(b.array, c2)
    assert np.array_equal(qa.read_counts(), c1 + c2)
    for x in (i1, i2, qa, qb):
        x.destroy()
