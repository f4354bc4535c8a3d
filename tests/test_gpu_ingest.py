"""Particle file ingest (sjcs_index_build_file): chunked reads through the
context's staging slots, each chunk uploaded as it is read.

The index must be the one the host-buffer build makes from the same file
(same counts), for files that end inside a chunk, span several chunks per
reader thread, carry trailing bytes (count = file size / 12, as
readDecodedParticles) or are empty; a missing file is refused.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle
from spatialjoincountovershells_b200 import _native as nat

pytestmark = pytest.mark.gpu

CHUNK_PARTICLES = (8 << 20) / 12  # particles per staging chunk (not whole)


def _counts(ctx, build, h, r2):
    q = ctx.query(h, r2)
    idx = build()
    q.count(idx)
    out = q.read_counts()
    t = idx.timing()
    idx.destroy()
    q.destroy()
    return out, t


@pytest.mark.parametrize("n", [1, 5, 100_003, int(CHUNK_PARTICLES) + 1, 12_000_001])
def test_file_build_matches_host_build(n, ctx, tmp_path):
    rng = np.random.default_rng(n)
    p = rng.uniform(0, 1000, size=(n, 3)).astype(np.float32)
    h = rng.uniform(0, 1000, size=(2000, 3)).astype(np.float32)
    r2 = nat.radius_table(0.01, 10, 24)
    path = tmp_path / "part.dat"
    nat.write_particle_file(path, p)
    got, t = _counts(ctx, lambda: ctx.build_index_file(path, radius_hint=10), h, r2)
    if n <= 100_003:
        want = oracle.count(p, h, r2)
    else:
        want, _ = _counts(ctx, lambda: ctx.build_index(p, radius_hint=10), h, r2)
    assert np.array_equal(got, want)
    assert t["h2d_ms"] > 0


def test_trailing_bytes_are_ignored_and_empty_files_build(ctx, tmp_path):
    rng = np.random.default_rng(7)
    p = rng.uniform(0, 1000, size=(5000, 3)).astype(np.float32)
    h = rng.uniform(0, 1000, size=(300, 3)).astype(np.float32)
    r2 = nat.radius_table(0.01, 30, 16)
    path = tmp_path / "odd.dat"
    path.write_bytes(p.tobytes() + b"\x01\x02\x03\x04\x05")  # 5 bytes past the last particle
    got, _ = _counts(ctx, lambda: ctx.build_index_file(path, radius_hint=30), h, r2)
    assert np.array_equal(got, oracle.count(p, h, r2))
    empty = tmp_path / "empty.dat"
    empty.write_bytes(b"")
    got, _ = _counts(ctx, lambda: ctx.build_index_file(empty, radius_hint=30), h, r2)
    assert not got.any()


def test_missing_file_is_refused(ctx, tmp_path):
    with pytest.raises(nat.SjcsError, match="not found"):
        ctx.build_index_file(tmp_path / "nope.dat")


def test_concurrent_file_builds_from_several_threads(ctx, tmp_path):
    # host threads share the context's staging slots one file at a time; every
    # index must still hold its own file
    import threading
    rng = np.random.default_rng(11)
    files = []
    for k in range(4):
        p = rng.uniform(0, 1000, size=(2_000_000 + 777 * k, 3)).astype(np.float32)
        path = tmp_path / f"part{k}.dat"
        nat.write_particle_file(path, p)
        files.append((path, p))
    h = rng.uniform(0, 1000, size=(1500, 3)).astype(np.float32)
    r2 = nat.radius_table(0.01, 12, 20)
    built, errors = [None] * len(files), []

    def work(k):
        try:
            built[k] = ctx.build_index_file(files[k][0], radius_hint=12)
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append(e)

    th = [threading.Thread(target=work, args=(k,)) for k in range(len(files))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors
    for k, (_, p) in enumerate(files):
        q = ctx.query(h, r2)
        q.count(built[k])
        got = q.read_counts()
        q.destroy()
        built[k].destroy()
        want, _ = _counts(ctx, lambda p=p: ctx.build_index(p, radius_hint=12), h, r2)
        assert np.array_equal(got, want), k


def test_prepared_context_builds_the_same(tmp_path):
    # a fresh context prepared for the files: same index as an unprepared one
    rng = np.random.default_rng(21)
    p = rng.uniform(0, 1000, size=(300_001, 3)).astype(np.float32)
    h = rng.uniform(0, 1000, size=(800, 3)).astype(np.float32)
    r2 = nat.radius_table(0.01, 15, 12)
    path = tmp_path / "part.dat"
    nat.write_particle_file(path, p)
    with nat.Context(0) as c:
        c.prepare_files(len(p))
        c.prepare_files(0)  # nothing to do
        got, _ = _counts(c, lambda: c.build_index_file(path, radius_hint=15), h, r2)
    assert np.array_equal(got, oracle.count(p, h, r2))
