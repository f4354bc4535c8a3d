"""Host-side formats: generators, readers and the result writer (CPU only)."""
from __future__ import annotations

import hashlib
import pathlib

import numpy as np
import pytest

from conftest import golden_counts
from golden import cases
from oracle import oracle
from spatialjoincountovershells_b200 import _native as nat

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference binaries not built")


@needs_ref
def test_particle_generator_matches_reference(tmp_path, built):
    r = oracle.run_ref(["-f", "a.dat", "b.dat", "-n", "5000", "-s", "17"], exe=oracle.REF_PGEN, cwd=tmp_path)
    assert r.returncode == 0
    ref = np.concatenate([np.fromfile(tmp_path / "a.dat", np.float32), np.fromfile(tmp_path / "b.dat", np.float32)])
    ours = nat.gen_uniform_particles(17, 2, 5000).reshape(-1)
    assert np.array_equal(ref.view(np.uint32), ours.view(np.uint32))


@needs_ref
def test_halo_generator_matches_reference(tmp_path, built):
    r = oracle.run_ref(["-f", "h.list", "-n", "3000", "-s", "23"], exe=oracle.REF_HGEN, cwd=tmp_path)
    assert r.returncode == 0
    nat.gen_uniform_halo_file(tmp_path / "mine.list", 23, 3000)
    assert (tmp_path / "h.list").read_bytes() == (tmp_path / "mine.list").read_bytes()


def test_generator_checksums_pinned(tmp_path, built):
    # pins the generators where the reference binaries are absent
    p = nat.gen_uniform_particles(1, 1, 1000)
    assert hashlib.sha256(p.tobytes()).hexdigest()[:16] == _PIN_PARTICLES
    nat.gen_uniform_halo_file(tmp_path / "h.list", 2, 500)
    assert hashlib.sha256((tmp_path / "h.list").read_bytes()).hexdigest()[:16] == _PIN_HALOS


_PIN_PARTICLES = "35967606d4eb08e1"  # sha256 prefix, uniform_decoded_particle_generator -n 1000 -s 1
_PIN_HALOS = "27c0f3b7ccdfbbb6"  # sha256 prefix, uniform_halo_generator -n 500 -s 2


def test_in_memory_halos_equal_parsed_file(tmp_path, built):
    nat.gen_uniform_halo_file(tmp_path / "h.list", 29, 4000, 10)
    parsed = nat.read_halos(tmp_path / "h.list")
    mem = nat.gen_uniform_halos(29, 4000, 10)
    assert parsed.tobytes() == mem.tobytes()
    face = nat.gen_face_halos(3, 300, 0, margin=5.0)
    nat.write_halo_file(tmp_path / "f.list", face)
    assert nat.read_halos(tmp_path / "f.list").tobytes() == face.tobytes()


def _halo_text(lines, header=16):
    return "".join(f"# dummy header {k}\n" for k in range(header)) + "".join(lines)


REC = "7 0 1.5e+11 0 0 0 0 0 1.5 2.5 3.5 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0\n"


def test_halo_reader_acceptance_rules(tmp_path, built):
    f = tmp_path / "h.list"
    # a last line without a newline is ignored (fgets reaches end of file)
    f.write_text(_halo_text([REC, REC.rstrip("\n")]))
    h = nat.read_halos(f)
    assert len(h) == 1 and h[0]["id"] == 7 and tuple(h[0]["point"]) == (1.5, 2.5, 3.5)
    assert h[0]["mass"] == np.float32(1.5e11)
    # fewer than 16 header lines
    f.write_text(_halo_text([], header=15))
    with pytest.raises(nat.SjcsError, match="does not contain headers"):
        nat.read_halos(f)
    # 16th header line without newline also counts as missing
    f.write_text(_halo_text([], header=15) + "# dummy header 15")
    with pytest.raises(nat.SjcsError, match="does not contain headers"):
        nat.read_halos(f)
    # exactly 16 header lines and nothing else: zero halos
    f.write_text(_halo_text([]))
    assert len(nat.read_halos(f)) == 0
    # a record with too few fields
    f.write_text(_halo_text([REC, "1 2 3\n"]))
    with pytest.raises(nat.SjcsError, match="may be incorrect"):
        nat.read_halos(f)
    # an empty line is a bad record too
    f.write_text(_halo_text([REC, "\n", REC]))
    with pytest.raises(nat.SjcsError, match="may be incorrect"):
        nat.read_halos(f)
    with pytest.raises(nat.SjcsError, match="not found"):
        nat.read_halos(tmp_path / "missing.list")


def test_halo_reader_long_lines_split_like_fgets(tmp_path, built):
    # A line longer than the reference's 16 KiB fgets buffer is read as several
    # records; the reader falls back to the literal fgets loop for such files.
    f = tmp_path / "h.list"
    long_rec = REC.rstrip("\n") + " 0" * 9000 + "\n"
    f.write_text(_halo_text([REC, long_rec, REC]))
    h = nat.read_halos(f)
    # long record: first piece parses as a halo; the remaining pieces are "0 0 0 ..." records
    pieces = -(-len(long_rec) // 16383)
    assert len(h) == 2 + pieces
    assert h[0]["id"] == 7 and h[1]["id"] == 7 and h[-1]["id"] == 7


def test_halo_reader_parallel_equals_serial(tmp_path, built):
    nat.gen_uniform_halo_file(tmp_path / "h.list", 31, 50000)
    a = nat.read_halos(tmp_path / "h.list", nthreads=1)
    b = nat.read_halos(tmp_path / "h.list", nthreads=8)
    assert a.tobytes() == b.tobytes() and len(a) == 50000


def test_filter_reader_intended_merge_join(tmp_path, built):
    # The reference never stores the filter count (ConstructFilterIdList,
    # src/Gadget/BufHalo.c:132-180), so its result depends on heap contents.
    # The reader implements the evident intent: sort the ids, keep every halo
    # whose id is listed (halo ids ascending, as the merge-join assumes).
    nat.gen_uniform_halo_file(tmp_path / "h.list", 14, 200)
    (tmp_path / "f.txt").write_text("150\n5\n7\n7\n100\n3\n199\n1000")
    h = nat.read_halos(tmp_path / "h.list", filter_path=tmp_path / "f.txt")
    assert list(h["id"]) == [3, 5, 7, 100, 150, 199]
    allh = nat.read_halos(tmp_path / "h.list")
    assert h.tobytes() == allh[[3, 5, 7, 100, 150, 199]].tobytes()


def test_particle_reader(tmp_path, built):
    p = nat.gen_uniform_particles(3, 1, 777)
    nat.write_particle_file(tmp_path / "p.dat", p)
    with open(tmp_path / "p.dat", "ab") as fh:  # trailing partial record is ignored (size / 12)
        fh.write(b"\x00" * 7)
    q = nat.read_particles(tmp_path / "p.dat")
    assert np.array_equal(p, q)
    with pytest.raises(nat.SjcsError, match="not found"):
        nat.read_particles(tmp_path / "nope.dat")


@pytest.mark.parametrize("name", list(cases.CASES))
def test_result_writer_reproduces_reference_text(name, case_dirs, manifest, tmp_path):
    d, spec = case_dirs[name]
    halos, _ = cases.load_halos_and_particles(spec, d)
    ids, counts, _ = golden_counts(name)
    r2 = nat.radius_table(*cases.radius_spec(spec))
    out = tmp_path / "r.txt"
    nat.write_result(out, halos, r2, counts, nthreads=3)
    data = out.read_bytes()
    assert hashlib.sha256(data).hexdigest() == manifest[name]["sha256"]
    if name == "kat":
        assert data == (cases.pathlib.Path(__file__).parent / "golden" / "kat_result.txt").read_bytes()


def _libc_strtof():
    import ctypes
    libc = ctypes.CDLL(None)
    f = libc.strtof
    f.restype = ctypes.c_float
    f.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    return f


def test_halo_reader_floats_equal_strtof(tmp_path, built):
    # The reader converts the plain decimal tokens itself and hands everything
    # else to strtof; either way each value must be strtof's, bit for bit.
    # Tokens: random widths and signs, exponents, hex, inf/nan, 20+ digits,
    # and shortest double representations of float midpoints (whose double
    # conversion lands exactly on the midpoint while their exact value is
    # just beside it).
    rng = np.random.default_rng(12)
    toks = []
    for _ in range(6000):
        ip = str(rng.integers(0, 10 ** rng.integers(1, 12)))
        fp = "".join(rng.choice(list("0123456789"), size=rng.integers(0, 14)))
        t = ip + ("." + fp if rng.random() < 0.9 else "")
        toks.append(("-" if rng.random() < 0.2 else "") + t)
    f32 = rng.uniform(0.0, 1000.0, 6000).astype(np.float32)
    nxt = np.nextafter(f32, np.float32(np.inf))
    for a, b in zip(f32.astype(np.float64), nxt.astype(np.float64)):
        toks.append(repr((a + b) / 2.0))  # exact midpoint as a double, shortest round-trip digits
    # 16 significant digits (< 2^53 as an integer): their double conversion
    # is often exactly the float midpoint they approximate
    f32 = rng.uniform(1.0, 9.0, 6000).astype(np.float32)
    nxt = np.nextafter(f32, np.float32(np.inf))
    for a, b in zip(f32.astype(np.float64), nxt.astype(np.float64)):
        toks.append("%.15f" % ((a + b) / 2.0))
    toks += ["0", "-0", "+3.5", "1e3", "2.5E-1", "0x1p3", "inf", "-nan", "1.", "007.250",
             "12345678901234567890.5", "0.0000000000000000000001", "340282356779733661637539395458142568448",
             "16777217", "16777217.0", "9007199254740993", "1.00000005960464477539062500001"]
    lines = [f"{i + 1} 0 {t} 0 0 0 0 0 {t} {toks[-1 - (i % len(toks))]} 1.5\n" for i, t in enumerate(toks)]
    f = tmp_path / "h.list"
    f.write_text(_halo_text(lines))
    h = nat.read_halos(f, nthreads=1)
    strtof = _libc_strtof()
    want = np.array([strtof(t.encode(), None) for t in toks], np.float32)
    want_y = np.array([strtof(toks[-1 - (i % len(toks))].encode(), None) for i in range(len(toks))], np.float32)
    assert np.array_equal(h["mass"].view(np.uint32), want.view(np.uint32))
    assert np.array_equal(h["point"][:, 0].view(np.uint32), want.view(np.uint32))
    assert np.array_equal(h["point"][:, 1].view(np.uint32), want_y.view(np.uint32))
    assert np.array_equal(h["id"], np.arange(1, len(toks) + 1, dtype=np.uint64))


def test_mapped_and_buffered_writers_agree(tmp_path, built):
    # a regular file goes through the mapped writer, stdout through the
    # buffered one; both must give the same text
    import subprocess
    import sys
    rng = np.random.default_rng(3)
    halos = nat.gen_uniform_halos(4, 3000)
    counts = rng.integers(0, 10 ** 9, size=(3000, 24)).astype(np.uint64)
    r2 = nat.radius_table(0.01, 7.0, 24)
    np.save(tmp_path / "c.npy", counts)
    np.save(tmp_path / "h.npy", halos)
    nat.write_result(tmp_path / "mapped.txt", halos, r2, counts, nthreads=5)
    code = ("import sys, numpy as np; sys.path.insert(0, sys.argv[1]); "
            "from spatialjoincountovershells_b200 import _native as nat; "
            "nat.write_result(None, np.load(sys.argv[2]), nat.radius_table(0.01, 7.0, 24), np.load(sys.argv[3]), "
            "nthreads=5)")
    root = str(pathlib.Path(__file__).resolve().parents[1])
    out = subprocess.run([sys.executable, "-c", code, root, str(tmp_path / "h.npy"), str(tmp_path / "c.npy")],
                         capture_output=True, check=True).stdout
    assert out == (tmp_path / "mapped.txt").read_bytes()
