"""Captured file steps (copy + build + count as one CUDA graph) on the GPU.

A replayed step must add exactly what the uncaptured calls add: the same
counts for every index kind and schedule, file after file through the same
pinned buffer, and mixed freely with ordinary count calls on the query.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from oracle import oracle
from spatialjoincountovershells_b200 import _native as nat

pytestmark = pytest.mark.gpu


def plain_counts(ctx, files, h, r2, kind, sched):
    q = ctx.query(h, r2)
    q.set_schedule(sched)
    for f in files:
        idx = ctx.build_index(f, radius_hint=20.0, kind=kind)
        q.count(idx)
        idx.destroy()
    out = q.read_counts()
    q.destroy()
    return out


@pytest.mark.parametrize("kind,sched", [(nat.INDEX_GRID, nat.SCHED_STATIC), (nat.INDEX_GRID, nat.SCHED_QUEUE),
                                        (nat.INDEX_LEARNED, nat.SCHED_AUTO), (nat.INDEX_MORTON, nat.SCHED_AUTO)])
def test_step_replays_match_uncaptured_calls(kind, sched, ctx):
    n = 150000
    files = [nat.gen_clustered_particles(s, n) for s in (41, 42, 43)]
    h = nat.gen_clustered_halos(44, 3000)
    r2 = nat.radius_table(0.01, 20, 64)
    want = plain_counts(ctx, files, h, r2, kind, sched)
    q = ctx.query(h, r2)
    q.set_schedule(sched)
    st = ctx.step(q, n, radius_hint=20.0, kind=kind)
    before = nat.launch_counter()
    for f in files:
        st.buffer[:] = f
        st.launch().wait()
        assert st.time_ms() > 0
    assert nat.launch_counter() - before >= 3 * 5  # the graph's kernels are counted
    assert np.array_equal(q.read_counts(), want)
    # an ordinary count call on the same query adds on top of the replays
    idx = ctx.build_index(files[0], radius_hint=20.0, kind=kind)
    q.count(idx)
    st.buffer[:] = files[1]
    st.launch()
    q.count(idx)
    got = q.read_counts()
    single0 = plain_counts(ctx, files[:1], h, r2, kind, sched)
    single1 = plain_counts(ctx, files[1:2], h, r2, kind, sched)
    assert np.array_equal(got, want + 2 * single0 + single1)
    idx.destroy()
    st.destroy()
    q.destroy()


def test_step_needs_pinned_memory(ctx):
    q = ctx.query(np.ones((4, 3), np.float32), nat.radius_table(0.1, 5, 8))
    pageable = np.zeros((100, 3), np.float32)
    h = ctypes.c_void_p()
    rc = nat.lib().sjcs_step_create(ctx._h, q._h, ctypes.c_void_p(pageable.ctypes.data), 100,
                                     ctypes.byref(nat.sjcs_index_opts()), ctypes.byref(h))
    assert rc == 1 and b"pinned" in nat.lib().sjcs_last_error()
    q.destroy()


DRIVER_OPTIONS = [["--index", "learned"], ["--index", "morton"], ["--schedule", "queue"], ["--autotune"],
                  ["--graph"], ["--graph", "--index", "learned", "--autotune"]]


@pytest.mark.parametrize("extra", DRIVER_OPTIONS, ids=lambda e: " ".join(e))
@pytest.mark.parametrize("name", ["multi_file", "edge", "c1"])
def test_driver_gpu_options_keep_the_reference_text(name, extra, case_dirs, manifest, tmp_path):
    import hashlib
    import subprocess

    from golden import cases
    from test_gpu_parity import DRIVER
    d, spec = case_dirs[name]
    out = tmp_path / "result.txt"
    r = subprocess.run([str(DRIVER), *cases.cli_args(spec, str(out)), *extra], cwd=d, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert hashlib.sha256(out.read_bytes()).hexdigest() == manifest[name]["sha256"]
    if "--graph" in extra:
        assert "step time" in r.stdout
    if "--autotune" in extra:
        assert "autotune: schedule" in r.stdout


def test_step_with_odd_tables_and_non_periodic_queries(ctx):
    rng = np.random.default_rng(45)
    n = 40000
    files = [rng.uniform(0, 1000, size=(n, 3)).astype(np.float32) for _ in range(2)]
    h = rng.uniform(0, 1000, size=(500, 3)).astype(np.float32)
    h[:3] = [[0, 0, 0], [1000, 1000, 1000], [2, 998, 500]]
    for r2, per in [(np.array([400.0, 100.0, 2500.0], np.float32), True),
                    (np.linspace(1, 3000, 2000).astype(np.float32), False), (nat.radius_table(0.5, 30, 17), False)]:
        q = ctx.query(h, r2, periodic=per)
        st = ctx.step(q, n, radius_hint=10.0)
        for f in files:
            st.buffer[:] = f
            st.launch().wait()
        want = np.zeros((len(h), len(r2)), np.uint64)
        for f in files:
            oracle.count(f, h, r2, periodic=per, counts=want, brute=len(r2) < 10)
        assert np.array_equal(q.read_counts(), want), (r2[:3], per)
        st.destroy()
        q.destroy()


def test_driver_graph_with_files_of_different_sizes(tmp_path):
    import hashlib
    import subprocess

    from test_gpu_parity import DRIVER
    rng = np.random.default_rng(46)
    sizes = [20000, 35000, 20000, 5000]
    for k, m in enumerate(sizes):
        nat.write_particle_file(tmp_path / f"p{k}.dat", rng.uniform(0, 1000, size=(m, 3)).astype(np.float32))
    nat.write_halo_file(tmp_path / "h.list", nat.gen_uniform_halos(47, 800, 0))
    outs = []
    for extra in ([], ["--graph"]):
        out = tmp_path / f"r{len(extra)}.txt"
        args = ["--thread", "2", "--next-setup", "2", "--particle-files", *[f"p{k}.dat" for k in range(len(sizes))],
                "--halo-file", "h.list", "--radius", "0.01:25:20", "--output-file", str(out), *extra]
        r = subprocess.run([str(DRIVER), *args], cwd=tmp_path, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        outs.append(hashlib.sha256(out.read_bytes()).hexdigest())
    assert outs[0] == outs[1]
