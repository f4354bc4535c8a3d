"""Serving loop on the GPU: requests of uneven size, admitted by memory, overlapping.

Each request's counts must be the same when it runs alone and when it runs in
a mix of concurrent requests (bit-identical: the counts are integers), and the
same as the oracle's sum over the resident particle files.
"""
from __future__ import annotations

import math
import time

import numpy as np
import pytest

from oracle import oracle
from spatialjoincountovershells_b200 import _native as nat

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def resident(ctx):
    files = [nat.gen_clustered_particles(s, 120000) for s in (61, 62)]
    idx = [ctx.build_index(f, radius_hint=10.0) for f in files]
    for i in idx:
        i.wait()
    yield files, idx
    for i in idx:
        i.destroy()


def make_requests(seed, count):
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(count):
        n = int(round(10 ** rng.uniform(0, 3.7)))  # 1 .. 5000 halos
        h = nat.gen_clustered_halos(1000 + k, n)
        nr = int(rng.integers(8, 65))
        r2 = nat.radius_table(0.001, float(rng.uniform(1, 10)), nr)
        reqs.append((h, r2, bool(rng.integers(0, 4) > 0)))
    return reqs


def test_each_result_is_the_same_alone_and_in_the_mix(ctx, resident):
    files, idx = resident
    reqs = make_requests(71, 40)
    # alone: one request in flight at a time
    alone = []
    with nat.Server(ctx, idx, slots=1) as srv:
        for h, r2, per in reqs:
            out, info = srv.wait(srv.submit(h, r2, periodic=per))
            alone.append(out.copy())
            assert info["status"] == 0 and info["latency_ms"] >= info["service_ms"] >= 0
    # mix: everything submitted at once, 6 slots
    with nat.Server(ctx, idx, slots=6) as srv:
        tickets = [srv.submit(h, r2, periodic=per) for h, r2, per in reqs]
        mixed = [srv.wait(t)[0] for t in tickets]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["max_inflight"] > 1
    for k, (a, b) in enumerate(zip(alone, mixed)):
        assert np.array_equal(a, b), k
    # and both equal the oracle summed over the resident files
    for k in (0, 7, 19):
        h, r2, per = reqs[k]
        want = np.zeros((len(h), len(r2)), np.uint64)
        for f in files:
            oracle.count(f, h, r2, periodic=per, counts=want)
        assert np.array_equal(alone[k].astype(np.uint64), want), k


def request_bytes(n, stride, nrads):
    # the server's estimate of a request's device memory
    return n * (stride + 16 + 40 + 4 * nrads + 13) + 65536 + 8 * nrads


def test_admission_waits_for_memory(ctx, resident):
    _, idx = resident
    reqs = [(nat.gen_clustered_halos(2000 + k, 4000), nat.radius_table(0.001, 8.0, 64), True) for k in range(10)]
    per_req = request_bytes(4000, 24, 64)
    # a budget for one request at a time: the rest wait in the queue
    with nat.Server(ctx, idx, slots=8, mem_budget=int(per_req * 1.5)) as srv:
        tickets = [srv.submit(h, r2, periodic=per) for h, r2, per in reqs]
        outs = [srv.wait(t) for t in tickets]
        st = srv.stats()
    assert st["peak_bytes"] <= st["budget_bytes"]
    assert st["max_inflight"] == 1
    with nat.Server(ctx, idx, slots=8) as srv:
        for (h, r2, per), (out, _) in zip(reqs, outs):
            assert np.array_equal(srv.wait(srv.submit(h, r2, periodic=per))[0], out)


def test_requests_arriving_during_others_are_admitted(ctx, resident):
    _, idx = resident
    reqs = make_requests(73, 30)
    rng = np.random.default_rng(51)
    with nat.Server(ctx, idx, slots=4) as srv:
        tickets = []
        for h, r2, per in reqs:
            time.sleep(float(rng.exponential(0.002)))  # Poisson arrivals
            tickets.append(srv.submit(h, r2, periodic=per))
        infos = [srv.wait(t)[1] for t in tickets]
    lat = sorted(i["latency_ms"] for i in infos)
    assert all(i["status"] == 0 for i in infos)
    assert lat[len(lat) // 2] <= lat[int(math.ceil(0.99 * len(lat))) - 1]


def test_request_too_big_for_the_budget_is_refused(ctx, resident):
    _, idx = resident
    with nat.Server(ctx, idx, slots=2, mem_budget=100_000) as srv:
        with pytest.raises(nat.SjcsError):
            srv.submit(np.zeros((2000, 3), np.float32), nat.radius_table(0.1, 2, 8))
        # empty requests are fine
        out, info = srv.wait(srv.submit(np.zeros((0, 3), np.float32), nat.radius_table(0.1, 2, 8)))
        assert out.shape == (0, 8) and info["status"] == 0


def test_server_over_learned_indexes_and_odd_tables(ctx):
    rng = np.random.default_rng(74)
    files = [rng.uniform(-5, 1005, size=(30000, 3)).astype(np.float32) for _ in range(2)]
    files[0][:3] = [[np.nan, 1, 1], [np.inf, 2, 2], [0, 0, 0]]
    idx = [ctx.build_index(f, radius_hint=10.0, kind=nat.INDEX_LEARNED, verify=True) for f in files]
    h = rng.uniform(0, 1000, size=(700, 3)).astype(np.float32)
    h[:4] = [[0, 0, 0], [1000, 1000, 1000], [np.nan, 5, 5], [999.99994, 0, 500]]
    tables = [np.array([400.0, 100.0, 2500.0], np.float32), np.linspace(1, 3000, 2000).astype(np.float32),
              nat.radius_table(0.01, 8.0, 33)]
    with nat.Server(ctx, idx, slots=3) as srv:
        tickets = [(srv.submit(h, r2, periodic=per), r2, per) for r2 in tables for per in (True, False)]
        for t, r2, per in tickets:
            out, info = srv.wait(t)
            want = np.zeros((len(h), len(r2)), np.uint64)
            for f in files:
                oracle.count(f, h, r2, periodic=per, counts=want, brute=len(r2) < 10)
            assert np.array_equal(out.astype(np.uint64), want), (r2[:3], per)
    for i in idx:
        i.destroy()


def test_destroy_finishes_pending_requests(ctx, resident):
    _, idx = resident
    reqs = make_requests(75, 12)
    srv = nat.Server(ctx, idx, slots=2)
    outs = [np.zeros((len(hh), len(r2)), np.uint32) for hh, r2, _ in reqs]
    for (hh, r2, per), o in zip(reqs, outs):
        srv.submit(hh, r2, periodic=per, out=o)
    srv.close()  # drains every submitted request before returning
    with nat.Server(ctx, idx, slots=2) as s2:
        for (hh, r2, per), o in zip(reqs, outs):
            assert np.array_equal(s2.wait(s2.submit(hh, r2, periodic=per))[0], o)
