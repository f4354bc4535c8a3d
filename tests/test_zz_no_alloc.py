"""sjcs_count_noalloc, the entry point for callers that must not have the
library allocate device memory (a framework that has reserved the GPU for its
own allocator, a latency-critical loop that cannot absorb cudaMalloc's
synchronisation).  It keeps all scratch in one fixed device array, so two
calls in a row must each give exactly the counts of the allocating path,
whatever the previous call left in that array.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from spatialjoincountovershells_b200 import _native as nat

pytestmark = pytest.mark.gpu

MAX_P = 131072
MAX_H = 32768


def _noalloc(dp, dh, r2, dcounts, periodic=True, stream=0):
    r2 = np.ascontiguousarray(r2, dtype=np.float32)
    return nat.lib().sjcs_count_noalloc(
        ctypes.c_void_p(dp.data_ptr()), dp.shape[0], ctypes.c_void_p(dh.data_ptr()), 12, dh.shape[0],
        ctypes.c_void_p(r2.ctypes.data), len(r2), 1 if periodic else 0, ctypes.c_void_p(dcounts.data_ptr()),
        ctypes.c_void_p(stream))


def _allocating_path(ctx, dp, dh, r2, periodic):
    q = ctx.query(dh, r2, periodic=periodic)
    idx = ctx.build_index(dp, radius_hint=float(np.sqrt(r2[-1])))
    q.count(idx)
    out = q.read_counts()
    idx.destroy()
    q.destroy()
    return out


def test_no_alloc_matches_allocating_path_on_two_calls_in_a_row():
    import torch
    with nat.Context(0) as ctx:
        cases = [
            # (seed, particles, halos, radius schedule, periodic): the second call is
            # smaller, so stale scratch from the first must not leak into it
            (21, MAX_P, 20000, (0.01, 40.0, 40), True),
            (22, 50000, 3000, (0.5, 25.0, 17), False),
        ]
        for seed, n, m, (mn, mx, nr), periodic in cases:
            rng = np.random.default_rng(seed)
            p = rng.uniform(0, 1000, size=(n, 3)).astype(np.float32)
            h = rng.uniform(0, 1000, size=(m, 3)).astype(np.float32)
            h[:40] = rng.choice([0.0, 1000.0, 3.0, 997.0], size=(40, 3))
            r2 = nat.radius_table(mn, mx, nr)
            dp = torch.from_numpy(p).cuda()
            dh = torch.from_numpy(h).cuda()
            dcounts = torch.zeros(m * nr, dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            assert _noalloc(dp, dh, r2, dcounts, periodic) == 0, nat.lib().sjcs_last_error()
            torch.cuda.synchronize()
            got = dcounts.cpu().numpy().view(np.uint32).reshape(m, nr).astype(np.uint64)
            want = _allocating_path(ctx, dp, dh, r2, periodic)
            assert np.array_equal(got, want), seed
            assert want.sum() > 0


def test_no_alloc_rejects_sizes_beyond_its_limits():
    import torch
    r2 = nat.radius_table(0.01, 5.0, 8)
    dp = torch.zeros((MAX_P + 1, 3), dtype=torch.float32, device="cuda")
    dh = torch.zeros((4, 3), dtype=torch.float32, device="cuda")
    dc = torch.zeros(4 * 8, dtype=torch.int32, device="cuda")
    assert _noalloc(dp, dh, r2, dc) == 1
    assert b"limit" in nat.lib().sjcs_last_error()
    dh2 = torch.zeros((MAX_H + 1, 3), dtype=torch.float32, device="cuda")
    assert _noalloc(dp[:10], dh2, r2, dc) == 1
    assert _noalloc(dp[:10], dh, nat.radius_table(0.01, 5.0, 300), dc) == 1
