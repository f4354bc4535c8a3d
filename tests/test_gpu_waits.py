"""Bounded waits of the count kernel.

The static schedule waits for each halo's staged candidate copies on an
mbarrier with a bound of about a second.  The test hook makes every staged
copy expect more bytes than it delivers, so the waits run out: the host must
see SJCS_ERR_TIMEOUT once, and the context must stay usable, giving exact
counts once the hook is off.  No fault, trap or endless wait is involved.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle
from spatialjoincountovershells_b200 import _native as nat

pytestmark = pytest.mark.gpu


def test_a_wait_that_runs_out_is_reported_and_the_context_recovers():
    rng = np.random.default_rng(71)
    p = rng.uniform(0, 1000, size=(40000, 3)).astype(np.float32)
    h = rng.uniform(0, 1000, size=(6, 3)).astype(np.float32)
    r2 = nat.radius_table(0.01, 20.0, 16)
    want = oracle.count(p, h, r2)
    with nat.Context(0) as ctx:
        idx = ctx.build_index(p, radius_hint=20.0)
        q = ctx.query(h, r2)
        q.set_schedule(nat.SCHED_STATIC)
        nat._check(nat.lib().sjcs_ctx_set_wait_test(ctx.handle, 16))
        q.count(idx)
        with pytest.raises(nat.SjcsError) as e:
            q.wait()
        assert e.value.code == 5  # SJCS_ERR_TIMEOUT
        q.wait()  # reported once
        nat._check(nat.lib().sjcs_ctx_set_wait_test(ctx.handle, 0))
        q.reset()
        q.count(idx)
        assert np.array_equal(q.read_counts(), want)
        idx.destroy()
        q.destroy()
