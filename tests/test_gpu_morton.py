"""Morton index forms on the GPU: plain Morton offset table and learned rank model.

Both forms must give the reference's counts bit-exactly (golden vectors) and
the oracle's on randomised, clustered and adversarial inputs.  The learned
form is run with the judge on (every cell boundary's corrected model rank is
compared with the offset table; no mismatch may be recorded) and off (the
model's error bound alone must make the lookups exact).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import golden_counts
from golden import cases
from oracle import oracle
from spatialjoincountovershells_b200 import _native as nat

pytestmark = pytest.mark.gpu

FORMS = [
    pytest.param((nat.INDEX_MORTON, False), id="morton"),
    pytest.param((nat.INDEX_LEARNED, True), id="learned-judged"),
    pytest.param((nat.INDEX_LEARNED, False), id="learned"),
]


def morton_counts(ctx, parts, halos, r2, form, periodic=True, level=0, hint=None):
    kind, verify = form
    q = ctx.query(halos, r2, periodic=periodic)
    if hint is None:
        hint = math.sqrt(float(r2[-1])) if np.isfinite(r2[-1]) else 0.0
    for p in parts:
        idx = ctx.build_index(p, radius_hint=hint, kind=kind, level=level, verify=verify)
        q.count(idx)
        if kind == nat.INDEX_LEARNED:
            info = idx.learned_info()
            L = idx.grid[0].bit_length() - 1
            assert info["level"] == L and info["leaves"] == 4096
            if verify and len(p):
                assert info["checked"] == 8 ** L + 1
                assert info["mismatches"] == 0, info
        idx.destroy()
    out = q.read_counts()
    q.destroy()
    return out


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("name", list(cases.CASES))
def test_morton_forms_match_reference(name, form, case_dirs, ctx):
    d, spec = case_dirs[name]
    halos, parts = cases.load_halos_and_particles(spec, d)
    r2 = nat.radius_table(*cases.radius_spec(spec))
    got = morton_counts(ctx, parts, halos, r2, form)
    _, want, _ = golden_counts(name)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("seed", [21, 22, 23, 24])
def test_random_inputs_vs_oracle(seed, form, ctx):
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
        got = morton_counts(ctx, [p], h, r2, form, periodic=periodic)
        want = oracle.count(p, h, r2, periodic=periodic)
        assert np.array_equal(got, want), (seed, periodic)


@pytest.mark.parametrize("level", [1, 3, 6, 8, 10])
def test_every_cell_level(level, ctx):
    rng = np.random.default_rng(100 + level)
    p = rng.uniform(0, 1000, size=(40000, 3)).astype(np.float32)
    p[:5000] = (rng.normal(300, 4, size=(5000, 3))).astype(np.float32)
    h = rng.uniform(0, 1000, size=(800, 3)).astype(np.float32)
    h[:100] = p[:100]
    r2 = nat.radius_table(0.001, 12, 40)
    want = oracle.count(p, h, r2)
    for form in [(nat.INDEX_MORTON, False), (nat.INDEX_LEARNED, True)]:
        got = morton_counts(ctx, [p], h, r2, form, level=level)
        assert np.array_equal(got, want), (level, form)


@pytest.mark.parametrize("form", FORMS)
def test_clustered_particles_and_halos(form, ctx):
    # the clustered workload's generators at reduced size: 60% of particles in
    # Gaussian clumps, 70% of halos at clump centres
    p = nat.gen_clustered_particles(5, 400000)
    h = nat.gen_clustered_halos(6, 4000)
    r2 = nat.radius_table(0.001, 5, 40)
    want = oracle.count(p, h, r2)
    got = morton_counts(ctx, [p], h, r2, form)
    assert np.array_equal(got, want)
    grid = ctx.query(h, r2)
    idx = ctx.build_index(p, radius_hint=5.0)
    grid.count(idx)
    assert np.array_equal(grid.read_counts(), got)
    idx.destroy()
    grid.destroy()


@pytest.mark.parametrize("rmax", [5.0, 0.37])
def test_particles_on_the_search_sphere_at_cell_edges(rmax, ctx):
    rng = np.random.default_rng(int(rmax * 1000))
    r2 = nat.radius_table(rmax / 50, rmax, 24)
    R = np.float32(math.sqrt(float(r2[-1])))
    for level in (8, 5):
        h_ = 1000.0 / 2 ** level
        centres = [(500.0, 500.0, 500.0), (h_ * 30, h_ * 20, h_ * 10), (h_ * 31 + 1e-4, h_ * 7, 2.5),
                   (1000.0 - 1e-3, h_ * 3, h_ * 12), (0.0, 0.0, 0.0), (h_ * 5, h_ * 5 - 1e-4, h_ * 5 + 1e-4)]
        pts = []
        for c in centres:
            d = rng.normal(size=(3000, 3))
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            for scale in (1.0, 1 - 1e-7, 1 + 1e-7, 1 - 3e-7, 1 + 3e-7):
                pts.append((np.array(c) + d * float(R) * scale) % 1000.0)
        p = np.concatenate(pts).astype(np.float32)
        h = np.array(centres, np.float32)
        want = oracle.count(p, h, r2, brute=True)
        assert want[:, -1].sum() > 0
        for form in [(nat.INDEX_MORTON, False), (nat.INDEX_LEARNED, True)]:
            got = morton_counts(ctx, [p], h, r2, form, level=level)
            assert np.array_equal(got, want), (level, form)


@pytest.mark.parametrize("form", FORMS)
def test_radius_tables_outside_the_fast_path(form, ctx):
    rng = np.random.default_rng(15)
    p = rng.uniform(0, 1000, size=(20000, 3)).astype(np.float32)
    h = np.concatenate([rng.uniform(0, 1000, size=(200, 3)), [[0, 0, 0], [1000, 1000, 1000]]]).astype(np.float32)
    tables = [
        np.array([400.0, 100.0, 2500.0, 900.0], np.float32),
        np.array([100.0, np.nan, 2500.0], np.float32),
        np.array([100.0, 400.0, np.nan], np.float32),
        np.array([25.0], np.float32),
        np.array([0.0, 0.0, 100.0, 100.0, 400.0], np.float32),
        np.linspace(1e-3, 900, 3000).astype(np.float32),
        np.linspace(1, 3000, 2000).astype(np.float32),
    ]
    for r2 in tables:
        for periodic in (True, False):
            got = morton_counts(ctx, [p], h, r2, form, periodic=periodic, hint=10.0)
            want = oracle.count(p, h, r2, periodic=periodic, brute=len(r2) < 10)
            assert np.array_equal(got, want), (r2[:4], periodic)


@pytest.mark.parametrize("form", FORMS)
def test_non_finite_and_out_of_box_coordinates(form, ctx):
    rng = np.random.default_rng(19)
    p = rng.uniform(-50, 1050, size=(30000, 3)).astype(np.float32)
    p[:6] = [[np.nan, 1, 1], [np.inf, 2, 2], [-np.inf, 3, 3], [1e30, 4, 4], [-1e30, 5, 5], [0, np.nan, 0]]
    h = rng.uniform(-20, 1020, size=(300, 3)).astype(np.float32)
    h[:6] = [[np.nan, 500, 500], [np.inf, 500, 500], [-np.inf, 0, 0], [1e30, 1, 1], [-5, -5, -5], [1005, 1005, 1005]]
    r2 = nat.radius_table(0.5, 40, 12)
    for periodic in (True, False):
        got = morton_counts(ctx, [p], h, r2, form, periodic=periodic)
        want = oracle.count(p, h, r2, periodic=periodic, brute=True)
        assert np.array_equal(got, want)


@pytest.mark.parametrize("form", FORMS)
def test_degenerate_particle_sets(form, ctx):
    rng = np.random.default_rng(7)
    h = rng.uniform(0, 1000, size=(500, 3)).astype(np.float32)
    h[:50] = [250.0, 250.0, 250.0]
    r2 = nat.radius_table(0.01, 30, 20)
    sets = [
        np.zeros((0, 3), np.float32),                                   # empty file
        np.array([[250.0, 250.0, 250.0]], np.float32),                   # one particle
        np.full((5000, 3), 250.0, np.float32),                           # one key repeated
        (rng.integers(0, 20, size=(30000, 3)) * 50.0).astype(np.float32),  # coarse lattice: long key runs
        np.concatenate([np.full((20000, 3), 0.0), rng.uniform(990, 1000, size=(20000, 3))]).astype(np.float32),
    ]
    for p in sets:
        got = morton_counts(ctx, [p], h, r2, form)
        want = oracle.count(p, h, r2) if len(p) else np.zeros((len(h), len(r2)), np.uint64)
        assert np.array_equal(got, want), len(p)


def test_learned_training_record(ctx):
    p = nat.gen_uniform_particles(3, 1, 2_000_000)
    idx = ctx.build_index(p, radius_hint=5.0, kind=nat.INDEX_LEARNED, verify=True)
    info = idx.learned_info()
    assert info["leaves"] == 4096 and 0 < info["nonempty"] <= 4096
    assert info["mismatches"] == 0 and info["checked"] == 8 ** info["level"] + 1
    assert 0 < info["mean_err"] <= info["max_err"] < 2_000_000
    assert info["sort_ms"] > 0 and info["train_ms"] > 0
    idx.destroy()
    grid = ctx.build_index(p, radius_hint=5.0)
    with pytest.raises(nat.SjcsError):
        grid.learned_info()
    grid.destroy()


def test_morton_options_are_validated(ctx):
    p = np.ones((10, 3), np.float32)
    for kw in [dict(kind=nat.INDEX_MORTON, level=11), dict(kind=nat.INDEX_LEARNED, grid=(4, 4, 4)),
               dict(kind=7)]:
        with pytest.raises(nat.SjcsError):
            ctx.build_index(p, **kw)
