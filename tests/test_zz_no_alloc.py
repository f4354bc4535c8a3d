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


def _noalloc(dp, dh, r2, dcounts, periodic=True, stream=0, stride=12, nhalos=None, offset=0):
    r2 = np.ascontiguousarray(r2, dtype=np.float32)
    m = dh.shape[0] if nhalos is None else nhalos
    return nat.lib().sjcs_count_noalloc(
        ctypes.c_void_p(dp.data_ptr()), dp.shape[0], ctypes.c_void_p(dh.data_ptr() + offset), stride, m,
        ctypes.c_void_p(r2.ctypes.data), len(r2), 1 if periodic else 0, ctypes.c_void_p(dcounts.data_ptr()),
        ctypes.c_void_p(stream))


def _u32_counts(dcounts, m, nr):
    return dcounts.cpu().numpy().view(np.uint32).reshape(m, nr).astype(np.uint64)


class _DefaultPool:
    """The device's default stream-ordered memory pool (driver API), where the
    library's allocating entry points take their memory (cudaMallocAsync);
    torch's caching allocator does not use it."""

    USED_HIGH, RESERVED_HIGH, USED_CURRENT = 8, 6, 7  # CUmemPool_attribute

    def __init__(self, device=0):
        self.cu = ctypes.CDLL("libcuda.so.1")
        dev = ctypes.c_int()
        assert self.cu.cuDeviceGet(ctypes.byref(dev), device) == 0
        self.pool = ctypes.c_void_p()
        assert self.cu.cuDeviceGetDefaultMemPool(ctypes.byref(self.pool), dev) == 0

    def get(self, attr):
        v = ctypes.c_uint64()
        assert self.cu.cuMemPoolGetAttribute(self.pool, attr, ctypes.byref(v)) == 0
        return v.value

    def reset_highs(self):
        for attr in (self.USED_HIGH, self.RESERVED_HIGH):
            z = ctypes.c_uint64(0)
            assert self.cu.cuMemPoolSetAttribute(self.pool, attr, ctypes.byref(z)) == 0


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
            got = _u32_counts(dcounts, m, nr)
            want = _allocating_path(ctx, dp, dh, r2, periodic)
            assert np.array_equal(got, want), seed
            assert want.sum() > 0


def test_no_alloc_call_takes_no_device_memory():
    """After a warm-up call, a call changes neither the default pool's high-water
    marks nor the device's free memory."""
    import torch
    rng = np.random.default_rng(24)
    dp = torch.from_numpy(rng.uniform(0, 1000, size=(100000, 3)).astype(np.float32)).cuda()
    dh = torch.from_numpy(rng.uniform(0, 1000, size=(5000, 3)).astype(np.float32)).cuda()
    r2 = nat.radius_table(0.01, 10.0, 24)
    dcounts = torch.zeros(5000 * 24, dtype=torch.int32, device="cuda")
    assert _noalloc(dp, dh, r2, dcounts) == 0, nat.lib().sjcs_last_error()
    torch.cuda.synchronize()
    pool = _DefaultPool()
    pool.reset_highs()
    used0 = pool.get(pool.USED_CURRENT)
    free0 = torch.cuda.mem_get_info()[0]
    assert _noalloc(dp, dh, r2, dcounts) == 0, nat.lib().sjcs_last_error()
    torch.cuda.synchronize()
    assert pool.get(pool.USED_HIGH) <= used0
    assert pool.get(pool.RESERVED_HIGH) <= pool.get(5)  # high mark = what the pool already held
    assert torch.cuda.mem_get_info()[0] == free0


def test_no_alloc_edge_inputs_match_the_allocating_path():
    """Strided halos read in place, an empty particle set, no halos, radius
    tables outside the fast path, and a call on a side stream."""
    import torch
    rng = np.random.default_rng(25)
    n, m = 60000, 2500
    p = rng.uniform(0, 1000, size=(n, 3)).astype(np.float32)
    h = rng.uniform(0, 1000, size=(m, 3)).astype(np.float32)
    h[:20] = rng.choice([0.0, 999.5, 1.0], size=(20, 3))
    dp = torch.from_numpy(p).cuda()
    dh = torch.from_numpy(h).cuda()
    with nat.Context(0) as ctx:
        # the reference's Halo records (u64 id, f32 mass, f32 point[3]): stride 24, point at byte 12
        rec = np.zeros(m, nat.HALO_DTYPE)
        rec["id"] = np.arange(m)
        rec["point"] = h
        drec = torch.from_numpy(rec.view(np.uint8).copy()).cuda()
        r2 = nat.radius_table(0.01, 15.0, 33)
        want = _allocating_path(ctx, dp, dh, r2, True)
        dc = torch.zeros(m * 33, dtype=torch.int32, device="cuda")
        assert _noalloc(dp, drec, r2, dc, stride=24, nhalos=m, offset=12) == 0, nat.lib().sjcs_last_error()
        torch.cuda.synchronize()
        assert np.array_equal(_u32_counts(dc, m, 33), want)

        # a side stream: the work is queued there and seen after that stream alone is synchronised
        side = torch.cuda.Stream()
        dc.zero_()
        torch.cuda.synchronize()
        assert _noalloc(dp, dh, r2, dc, stream=side.cuda_stream) == 0, nat.lib().sjcs_last_error()
        side.synchronize()
        assert np.array_equal(_u32_counts(dc, m, 33), want)

        # radius tables outside the fast path: unsorted with a repeat, and one with a NaN
        for tab in (np.array([4.0, 1.0, 9.0, 9.0, 25.0, 16.0, 100.0], np.float32),
                    np.array([1.0, np.nan, 30.0, 120.0], np.float32)):
            w = _allocating_path(ctx, dp, dh, tab, True)
            dc2 = torch.zeros(m * len(tab), dtype=torch.int32, device="cuda")
            assert _noalloc(dp, dh, tab, dc2) == 0, nat.lib().sjcs_last_error()
            torch.cuda.synchronize()
            assert np.array_equal(_u32_counts(dc2, m, len(tab)), w)
            assert w.sum() > 0

        # no particles: counts stay as they were; no halos: nothing to do
        dc.fill_(3)
        torch.cuda.synchronize()
        assert _noalloc(dp[:0], dh, r2, dc) == 0, nat.lib().sjcs_last_error()
        assert _noalloc(dp, dh[:0], r2, dc, nhalos=0) == 0, nat.lib().sjcs_last_error()
        torch.cuda.synchronize()
        assert bool((dc == 3).all())


def test_no_alloc_call_replays_from_a_cuda_graph():
    """A call captured into a CUDA graph (after the warm-up call that loads the
    scratch array) replays with its radius table baked into the graph: each
    replay adds the same counts as a direct call, the oracle-pinned
    allocating path's."""
    import torch
    with nat.Context(0) as ctx:
        rng = np.random.default_rng(27)
        n, m = 60000, 2500
        p = rng.uniform(0, 1000, size=(n, 3)).astype(np.float32)
        h = rng.uniform(0, 1000, size=(m, 3)).astype(np.float32)
        h[:30] = rng.choice([0.0, 999.99, 4.0, 996.0], size=(30, 3))
        r2 = nat.radius_table(0.05, 30.0, 24)
        nr = len(r2)
        dp = torch.from_numpy(p).cuda()
        dh = torch.from_numpy(h).cuda()
        dcounts = torch.zeros(m * nr, dtype=torch.int32, device="cuda")
        want = _allocating_path(ctx, dp, dh, r2, True)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            assert _noalloc(dp, dh, r2, dcounts, stream=side.cuda_stream) == 0, nat.lib().sjcs_last_error()
        side.synchronize()
        assert np.array_equal(_u32_counts(dcounts, m, nr), want)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=side):
            rc = _noalloc(dp, dh, r2, dcounts, stream=side.cuda_stream)
        assert rc == 0, nat.lib().sjcs_last_error()
        # the table the graph holds must not depend on this host array
        r2[:] = np.float32(1.0)
        dcounts.zero_()
        torch.cuda.synchronize()
        graph.replay()
        torch.cuda.synchronize()
        assert np.array_equal(_u32_counts(dcounts, m, nr), want)
        graph.replay()
        torch.cuda.synchronize()
        assert np.array_equal(_u32_counts(dcounts, m, nr), 2 * want)
        del graph


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
