"""The oracle (CPU restatement) pinned against the reference's own outputs.

The golden vectors were produced by the reference program compiled from its
own sources (tests/golden/make_golden.py).  If the restatement agrees with
them on the known-answer fixture, on shell edges, box faces, R > 500 and the
1e6 x 10.5k workload, it is trusted as the checker for the GPU path.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, golden_counts
from golden import cases
from oracle import oracle
from spatialjoincountovershells_b200 import _native as nat


@pytest.mark.parametrize("name", list(cases.CASES))
def test_oracle_matches_reference_golden(name, case_dirs):
    d, spec = case_dirs[name]
    halos, parts = cases.load_halos_and_particles(spec, d)
    r2 = oracle.radius_table(*cases.radius_spec(spec))
    counts = np.zeros((len(halos), len(r2)), dtype=np.uint64)
    for p in parts:
        oracle.count(p, halos, r2, periodic=True, counts=counts)
    ids, want, totals = golden_counts(name)
    assert np.array_equal(halos["id"], ids)
    assert np.array_equal(counts, want)
    # the reference's Total row: sum over halos plus halo 0 again
    assert np.array_equal(counts.sum(axis=0) + counts[0], totals)


def test_known_answer_periodic_corners(case_dirs):
    # TestData4PB: per halo 1, 3, 3, 1 particles at squared distances 0, 1, 2, 3
    d, spec = case_dirs["kat"]
    halos, parts = cases.load_halos_and_particles(spec, d)
    r2 = oracle.radius_table(0.001, 5, 40)
    c = oracle.count(parts[0], halos, r2)
    for h in range(2):
        nz = {int(i): int(v) for i, v in enumerate(c[h]) if v}
        bins = [int(np.searchsorted(r2, dd, side="right")) for dd in (0.0, 1.0, 2.0, 3.0)]
        assert nz == {bins[0]: 1, bins[1]: 3, bins[2]: 3, bins[3]: 1}


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("periodic", [True, False])
def test_grid_oracle_equals_brute_force(seed, periodic, built):
    rng = np.random.default_rng(seed)
    p = rng.uniform(0, 1000, size=(3000, 3)).astype(np.float32)
    p[:20] = rng.choice([0.0, 1000.0, 999.99994, 0.5], size=(20, 3))
    h = np.concatenate([rng.uniform(0, 1000, size=(60, 3)), rng.choice([0.0, 1000.0, 3.0, 997.0], size=(20, 3))])
    h = h.astype(np.float32)
    r2 = oracle.radius_table(0.5, 90.0, 17)
    a = oracle.count(p, h, r2, periodic=periodic)
    b = oracle.count(p, h, r2, periodic=periodic, brute=True)
    assert np.array_equal(a, b)
    assert a.sum() > 0


def test_nonmonotone_and_nan_tables_follow_first_match(built):
    rng = np.random.default_rng(7)
    p = rng.uniform(0, 1000, size=(4000, 3)).astype(np.float32)
    h = rng.uniform(0, 1000, size=(50, 3)).astype(np.float32)
    for r2 in (np.array([400.0, 100.0, 2500.0, 900.0], np.float32),
               np.array([np.nan, 100.0, 2500.0], np.float32),
               np.array([100.0, np.nan, 2500.0], np.float32)):
        a = oracle.count(p, h, r2)
        b = oracle.count(p, h, r2, brute=True)
        assert np.array_equal(a, b)


def test_radius_table_fma_and_plain_agree_on_workload_schedules(built):
    for spec in [(0.001, 5, 40), (0.01, 20, 64), (0.5, 20, 16), (600, 1, 12), (0.001, 9.37, 57)]:
        assert np.array_equal(oracle.radius_table(*spec, use_fma=True), oracle.radius_table(*spec, use_fma=False))
        assert np.array_equal(oracle.radius_table(*spec), nat.radius_table(*spec))


def test_radius_labels_match_reference_text(built):
    # The reference prints (float)sqrt(r2[i]) with %f; the KAT text holds all 40 labels.
    text = (cases.pathlib.Path(__file__).parent / "golden" / "kat_result.txt").read_text().splitlines()
    r2 = nat.radius_table(0.001, 5, 40)
    rad = np.sqrt(r2.astype(np.float64)).astype(np.float32)
    want = ["  [0.0 ~ %f]: " % rad[0]] + ["  [%f ~ %f]: " % (rad[i - 1], rad[i]) for i in range(1, 40)]
    got = [ln[: ln.rindex(":") + 2] for ln in text[1:41]]
    assert got == want


def test_compressed_decode_matches_the_reference_decoder():
    # golden/compressed_decode.npz holds the output of the reference's own
    # decodeCompressedParticle (oracle/_ref/ref_decode.exe) per decode set
    import hashlib

    from golden import cases
    from spatialjoincountovershells_b200 import _native as nat
    z = np.load(GOLDEN / "compressed_decode.npz")
    for k, (seed, n1d, box, dmin, dmax, bits, id0, n) in enumerate(cases.DECODE_SETS):
        hdr, uv = nat.gen_compressed(seed, n1d, box, dmin, dmax, bits, id0, n)
        pos = oracle.decode_compressed(hdr, uv)
        assert hashlib.sha256(pos.tobytes()).hexdigest() == z["sha256"][k], k
        assert np.array_equal(pos[:512].view(np.uint32), z["heads"][k].view(np.uint32)), k


def test_compressed_file_round_trip(tmp_path):
    from spatialjoincountovershells_b200 import _native as nat
    hdr, uv = nat.gen_compressed(9, 20, 500.0, -1.5, 2.5, 10, 11, 5000)
    nat.write_compressed_file(tmp_path / "c.dat", hdr, uv)
    h2, uv2 = nat.read_compressed(tmp_path / "c.dat")
    assert h2 == hdr and np.array_equal(uv, uv2)
    assert int.from_bytes(hdr[4:8], "little") == 5000           # npart[1]
    assert int.from_bytes(hdr[100:104], "little") == 20 ** 3    # npartTotal[1]
    assert (tmp_path / "c.dat").stat().st_size == 4 + 256 + 4 + 4 + 6 * 5000 + 4
