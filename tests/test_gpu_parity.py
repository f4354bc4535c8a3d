"""GPU path (libsjcs.so through its C ABI) against the reference's outputs and the oracle.

Bit-exact integer counts everywhere: the golden vectors come from the
reference program itself; randomised and adversarial cases are checked
against the oracle restatement (itself pinned to the golden vectors in
test_oracle.py).
"""
from __future__ import annotations

import hashlib
import math
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_counts
from golden import cases
from oracle import oracle
from spatialjoincountovershells_b200 import _native as nat

pytestmark = pytest.mark.gpu
DRIVER = ROOT / "spatialjoincountovershells_b200" / "bin" / "sjcs_rcount"


def gpu_counts(ctx, parts, halos, r2, periodic=True, grid=None, hint=None):
    q = ctx.query(halos, r2, periodic=periodic)
    if hint is None:
        hint = math.sqrt(float(r2[-1])) if np.isfinite(r2[-1]) else 0.0
    for p in parts:
        idx = ctx.build_index(p, radius_hint=hint, grid=grid)
        q.count(idx)
        idx.destroy()
    out = q.read_counts()
    q.destroy()
    return out


@pytest.mark.parametrize("name", list(cases.CASES))
def test_api_counts_match_reference(name, case_dirs, ctx):
    d, spec = case_dirs[name]
    halos, parts = cases.load_halos_and_particles(spec, d)
    r2 = nat.radius_table(*cases.radius_spec(spec))
    got = gpu_counts(ctx, parts, halos, r2)
    ids, want, _ = golden_counts(name)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("name", list(cases.CASES))
@pytest.mark.parametrize("backlog", [0, 2])
def test_driver_text_matches_reference(name, backlog, case_dirs, manifest, tmp_path):
    d, spec = case_dirs[name]
    out = tmp_path / "result.txt"
    r = subprocess.run([str(DRIVER), *cases.cli_args(spec, str(out), backlog=backlog)], cwd=d,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    data = out.read_bytes()
    assert hashlib.sha256(data).hexdigest() == manifest[name]["sha256"]
    assert ">>>> total searching time" in r.stdout


def test_driver_writes_result_to_stdout_without_output_file(case_dirs):
    d, spec = case_dirs["kat"]
    args = cases.cli_args(spec, "x")[:-2]
    r = subprocess.run([str(DRIVER), *args], cwd=d, capture_output=True, timeout=120)
    assert r.returncode == 0
    kat = (ROOT / "tests" / "golden" / "kat_result.txt").read_bytes()
    assert kat in r.stdout


def test_grid_shape_does_not_change_counts(case_dirs, ctx):
    d, spec = case_dirs["c1"]
    halos, parts = cases.load_halos_and_particles(spec, d)
    r2 = nat.radius_table(0.001, 5, 40)
    ref = gpu_counts(ctx, parts, halos, r2)
    for grid in [(1, 1, 1), (7, 3, 5), (1000, 400, 400), (2048, 64, 3)]:
        assert np.array_equal(gpu_counts(ctx, parts, halos, r2, grid=grid), ref), grid


@pytest.mark.parametrize("seed", [11, 12, 13, 14])
def test_random_inputs_vs_oracle(seed, ctx):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 60000))
    p = rng.uniform(0, 1000, size=(n, 3)).astype(np.float32)
    if seed % 2:
        p[: n // 2] = (rng.normal(500, 30, size=(n // 2, 3)) % 1000).astype(np.float32)
    nh = int(rng.integers(1, 3000))
    h = rng.uniform(0, 1000, size=(nh, 3)).astype(np.float32)
    h[: nh // 4] = rng.choice([0.0, 1000.0, 2.0, 998.0, 999.99994], size=(nh // 4, 3))
    mn, mx, nr = [(0.001, 5, 40), (0.01, 20, 64), (1, 120, 9), (50, 700, 5)][seed % 4]
    r2 = nat.radius_table(mn, mx, nr)
    for periodic in (True, False):
        got = gpu_counts(ctx, [p], h, r2, periodic=periodic)
        want = oracle.count(p, h, r2, periodic=periodic)
        assert np.array_equal(got, want), (seed, periodic)


def test_radius_tables_outside_the_fast_path(ctx):
    rng = np.random.default_rng(5)
    p = rng.uniform(0, 1000, size=(20000, 3)).astype(np.float32)
    h = np.concatenate([rng.uniform(0, 1000, size=(200, 3)), [[0, 0, 0], [1000, 1000, 1000]]]).astype(np.float32)
    tables = [
        np.array([400.0, 100.0, 2500.0, 900.0], np.float32),   # not sorted
        np.array([100.0, np.nan, 2500.0], np.float32),         # NaN inside
        np.array([np.nan, 100.0, 900.0], np.float32),
        np.array([100.0, 400.0, np.nan], np.float32),          # NaN last: R is NaN, box passes everything
        np.array([25.0], np.float32),                          # a single shell
        np.array([0.0, 0.0, 100.0, 100.0, 400.0], np.float32), # repeated edges
        np.array([0.0, 1.0, 4.0, 9.0, 900.0], np.float32),     # zero first edge (lookup-table path)
        np.linspace(1e-3, 900, 3000).astype(np.float32),       # too dense for the lookup table
        np.linspace(1, 3000, 2000).astype(np.float32),         # more shells than shared memory holds
    ]
    for r2 in tables:
        for periodic in (True, False):
            got = gpu_counts(ctx, [p], h, r2, periodic=periodic, hint=10.0)
            want = oracle.count(p, h, r2, periodic=periodic, brute=len(r2) < 10)
            assert np.array_equal(got, want), (r2[:4], periodic)


@pytest.mark.parametrize("rmax", [5.0, 20.0, 0.37])
def test_particles_on_the_search_sphere(rmax, ctx):
    # The count kernel clips each row of cells to the sphere of radius R with
    # conservative margins; particles on the sphere (and a few ulps either
    # side), around halos sitting on cell edges, must all be classified exactly.
    rng = np.random.default_rng(int(rmax * 100))
    r2 = nat.radius_table(rmax / 50, rmax, 24)
    R = np.float32(math.sqrt(float(r2[-1])))
    for grid in [(1000, 400, 400), (97, 31, 13)]:
        hx, hy, hz = 1000.0 / grid[0], 1000.0 / grid[1], 1000.0 / grid[2]
        centres = [(500.0, 500.0, 500.0), (hx * 300, hy * 20, hz * 10), (hx * 31 + 1e-4, hy * 7, 2.5),
                   (1000.0 - 1e-3, hy * 3, hz * 12), (0.0, 0.0, 0.0), (hx * 5, hy * 5 - 1e-4, hz * 5 + 1e-4)]
        pts = []
        for c in centres:
            d = rng.normal(size=(3000, 3))
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            for scale in (1.0, 1 - 1e-7, 1 + 1e-7, 1 - 3e-7, 1 + 3e-7):
                pts.append((np.array(c) + d * float(R) * scale) % 1000.0)
        p = np.concatenate(pts).astype(np.float32)
        h = np.array(centres, np.float32)
        got = gpu_counts(ctx, [p], h, r2, grid=grid)
        want = oracle.count(p, h, r2, brute=True)
        assert np.array_equal(got, want), grid
        assert want[:, -1].sum() > 0


def test_non_finite_and_out_of_box_coordinates(ctx):
    rng = np.random.default_rng(9)
    p = rng.uniform(-50, 1050, size=(30000, 3)).astype(np.float32)
    p[:6] = [[np.nan, 1, 1], [np.inf, 2, 2], [-np.inf, 3, 3], [1e30, 4, 4], [-1e30, 5, 5], [0, np.nan, 0]]
    h = rng.uniform(-20, 1020, size=(300, 3)).astype(np.float32)
    h[:6] = [[np.nan, 500, 500], [np.inf, 500, 500], [-np.inf, 0, 0], [1e30, 1, 1], [-5, -5, -5], [1005, 1005, 1005]]
    r2 = nat.radius_table(0.5, 40, 12)
    for periodic in (True, False):
        got = gpu_counts(ctx, [p], h, r2, periodic=periodic)
        want = oracle.count(p, h, r2, periodic=periodic, brute=True)
        assert np.array_equal(got, want)


def test_empty_index_and_empty_query(ctx):
    r2 = nat.radius_table(0.001, 5, 40)
    h = np.array([[1, 2, 3], [500, 500, 500]], np.float32)
    got = gpu_counts(ctx, [np.zeros((0, 3), np.float32)], h, r2)
    assert got.shape == (2, 40) and not got.any()
    q = ctx.query(np.zeros((0, 3), np.float32), r2)
    idx = ctx.build_index(np.ones((10, 3), np.float32))
    q.count(idx)
    assert q.read_counts().shape == (0, 40)
    idx.destroy()
    q.destroy()


def test_accumulate_and_reset(ctx):
    rng = np.random.default_rng(3)
    p = rng.uniform(0, 1000, size=(50000, 3)).astype(np.float32)
    h = rng.uniform(0, 1000, size=(500, 3)).astype(np.float32)
    r2 = nat.radius_table(0.1, 30, 16)
    want = oracle.count(p, h, r2)
    q = ctx.query(h, r2)
    idx = ctx.build_index(p, radius_hint=30)
    q.count(idx).count(idx)
    base = np.full((500, 16), 7, np.uint64)
    q.read_counts(out=base, accumulate=True)
    assert np.array_equal(base, 2 * want + 7)
    q.reset()
    q.count(idx)
    assert np.array_equal(q.read_counts(), want)
    # one-shot reference-style call: counts +=
    c = np.ones((500, 16), np.uint64)
    nat.multi_range_count_with_periodic_bound(ctx, idx, h, r2, c)
    assert np.array_equal(c, want + 1)
    idx.destroy()
    q.destroy()


def test_split_files_add_up(ctx):
    # counts are additive over particle files (the driver accumulates per file)
    rng = np.random.default_rng(4)
    p = rng.uniform(0, 1000, size=(200000, 3)).astype(np.float32)
    h = rng.uniform(0, 1000, size=(4000, 3)).astype(np.float32)
    r2 = nat.radius_table(0.01, 25, 32)
    whole = gpu_counts(ctx, [p], h, r2)
    parts = gpu_counts(ctx, np.array_split(p, 7), h, r2)
    assert np.array_equal(whole, parts)


def test_device_pointer_api(ctx):
    import torch
    rng = np.random.default_rng(8)
    p = rng.uniform(0, 1000, size=(80000, 3)).astype(np.float32)
    h = rng.uniform(0, 1000, size=(2000, 3)).astype(np.float32)
    r2 = nat.radius_table(0.001, 15, 40)
    dp = torch.from_numpy(p).cuda()
    dh = torch.from_numpy(h).cuda()
    torch.cuda.synchronize()
    q = ctx.query(dh, r2)
    idx = ctx.build_index(dp, radius_hint=15)
    q.count(idx)
    got = q.read_counts()
    idx.destroy()
    q.destroy()
    assert np.array_equal(got, oracle.count(p, h, r2))


@pytest.mark.parametrize("offset", [0, 1, 2, 3])
def test_device_particles_at_any_alignment(offset, ctx):
    # The first radix pass stages a 16-byte-aligned particle array in shared
    # memory a tile at a time and reads any other one particle by particle:
    # same counts at every float offset, with a ragged last tile whose length
    # is not a whole number of 16-byte chunks, and with 9-bit digits (the
    # 25- and 27-bit cell keys of the requested grids).
    import torch
    rng = np.random.default_rng(30 + offset)
    n = 3 * 4096 + 1001
    p = rng.uniform(0, 1000, size=(n, 3)).astype(np.float32)
    h = rng.uniform(0, 1000, size=(1500, 3)).astype(np.float32)
    r2 = nat.radius_table(0.001, 8, 40)
    want = oracle.count(p, h, r2)
    flat = torch.zeros(3 * n + 4, dtype=torch.float32, device="cuda")
    flat[offset:offset + 3 * n] = torch.from_numpy(p.reshape(-1)).cuda()
    dp = flat[offset:offset + 3 * n].view(n, 3)
    torch.cuda.synchronize()
    for grid in (None, (64, 64, 64), (256, 256, 512), (512, 512, 512)):
        q = ctx.query(h, r2)
        idx = ctx.build_index(dp, radius_hint=8, grid=grid)
        q.count(idx)
        got = q.read_counts()
        idx.destroy()
        q.destroy()
        assert np.array_equal(got, want), grid


def test_halo_struct_stride_reads_reference_layout(case_dirs, ctx):
    d, spec = case_dirs["uniform_small"]
    halos, parts = cases.load_halos_and_particles(spec, d)
    r2 = nat.radius_table(*cases.radius_spec(spec))
    a = gpu_counts(ctx, parts, halos, r2)                       # stride 24 (Halo structs)
    b = gpu_counts(ctx, parts, np.ascontiguousarray(halos["point"]), r2)  # stride 12
    assert np.array_equal(a, b)
