"""Input fixtures of the golden cases, regenerated deterministically from seeds.

Every case writes its particle files and halo file into a directory and
returns the astr_rcount command-line arguments that go with them.  The
expected outputs in this directory were produced by running the reference
program (compiled from its own sources) on exactly these inputs -- see
make_golden.py.  Uniform particle and halo files come from the project's
generators, which reproduce the reference generators byte for byte
(tests/test_host_formats.py checks that).
"""
from __future__ import annotations

import math
import pathlib

import numpy as np

from spatialjoincountovershells_b200 import _native as nat

HALO_HEADER = "".join(f"# dummy header {k}\n" for k in range(16))


def _logspace_r(minrad: float, maxrad: float, n: int) -> np.ndarray:
    """The unsquared radii of the driver's schedule (fp32), for placing particles on shell edges."""
    a, b = math.log2(minrad), math.log2(maxrad)
    c = (b - a) / (n - 1)
    r = [np.float32(math.pow(2.0, a + i * c)) for i in range(n - 1)] + [np.float32(math.pow(2.0, b))]
    return np.array(r, dtype=np.float32)


def _kat(d: pathlib.Path) -> dict:
    # The reference's periodic known-answer fixture (TestData4PB): the 8 corners
    # of {0,999}^3 and two halos at the opposite corners; per halo the periodic
    # squared distances are 0, 1, 2, 3 with multiplicities 1, 3, 3, 1.
    corners = np.array([[x, y, z] for x in (0.0, 999.0) for y in (0.0, 999.0) for z in (0.0, 999.0)],
                       dtype=np.float32)
    nat.write_particle_file(d / "kat_particles.dat", corners)
    rest = " 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0"
    lines = HALO_HEADER
    lines += "0 0 8.51985e+11 0 0 0 0 0 0.0 0.0 0.0" + rest + "\n"
    lines += "0 0 8.51985e+11 0 0 0 0 0 999 999 999" + rest + "\n"
    (d / "kat_halos.list").write_text(lines)
    return dict(particle_files=["kat_particles.dat"], halo_file="kat_halos.list", radius="0.001:5:40")


def _uniform_small(d: pathlib.Path) -> dict:
    nat.write_particle_file(d / "us_p.dat", nat.gen_uniform_particles(1, 1, 20000))
    h = np.concatenate([nat.gen_uniform_halos(2, 300, 0), nat.gen_face_halos(3, 60, 300, margin=60.0)])
    nat.write_halo_file(d / "us_h.list", h)
    return dict(particle_files=["us_p.dat"], halo_file="us_h.list", radius="0.01:60:40")


def _multi_file(d: pathlib.Path) -> dict:
    p = nat.gen_uniform_particles(5, 3, 8000)
    for f in range(3):
        nat.write_particle_file(d / f"mf_p{f}.dat", p[f * 8000:(f + 1) * 8000])
    h = np.concatenate([nat.gen_uniform_halos(6, 200, 0), nat.gen_face_halos(7, 40, 200, margin=30.0)])
    nat.write_halo_file(d / "mf_h.list", h)
    return dict(particle_files=[f"mf_p{f}.dat" for f in range(3)], halo_file="mf_h.list", radius="0.05:30:24")


def _edge(d: pathlib.Path) -> dict:
    r = _logspace_r(0.5, 20.0, 16)
    pts = []
    # on every shell edge around the origin halo: dist == r2[i] exactly
    for ri in r:
        pts += [[ri, 0, 0], [0, ri, 0], [0, 0, ri], [np.nextafter(ri, np.float32(0)), 0, 0],
                [np.nextafter(ri, np.float32(100)), 0, 0]]
        # and across the periodic boundary (999.x wraps to -0.x)
        pts += [[np.float32(1000.0) - ri, 0, 0], [0, np.float32(1000.0) - ri, 0]]
    # exactly on the query box of the centre halo (R = 20): 480 and 520
    for v in (480.0, 520.0, np.nextafter(np.float32(480.0), np.float32(0)), np.nextafter(np.float32(520.0), np.float32(1e4))):
        pts += [[v, 500, 500], [500, v, 500], [500, 500, v]]
    # box faces, corners, and the top of [0, 1000]
    for v in (0.0, 1000.0, np.float32(999.99994), np.float32(1e-6), 5.0, 995.0, 20.0, 980.0):
        pts += [[v, v, v], [v, 0, 1000.0], [1000.0, v, 0], [500, 500, v]]
    pts += [[500, 500, 500], [500.5, 500, 500], [500, 500.5, 500.5]]
    rng_p = nat.gen_uniform_particles(11, 1, 6000)
    p = np.concatenate([np.array(pts, dtype=np.float32), rng_p]).astype(np.float32)
    nat.write_particle_file(d / "edge_p.dat", p)
    halos = [(0, 0, 0), (1000, 1000, 1000), (500, 500, 500), (999.99994, 0.0, 500), (5.0, 995.0, 20.0),
             (20, 20, 20), (0.5, 999.5, 0.5), (980, 20, 500), (1000, 0, 500), (0, 1000, 1000)]
    h = np.zeros(len(halos) + 40, dtype=nat.HALO_DTYPE)
    h["id"] = np.arange(len(h))
    h["mass"] = 1e12
    h["point"][: len(halos)] = np.array(halos, dtype=np.float32)
    h[len(halos):] = nat.gen_face_halos(13, 40, len(halos), margin=20.0)
    nat.write_halo_file(d / "edge_h.list", h)
    return dict(particle_files=["edge_p.dat"], halo_file="edge_h.list", radius="0.5:20:16")


def _big_radius(d: pathlib.Path) -> dict:
    # R = 600 > 500: the query box crosses both faces of an axis; the minimum
    # side takes precedence and particles are counted once per image.
    nat.write_particle_file(d / "br_p.dat", nat.gen_uniform_particles(7, 1, 2000))
    h = np.concatenate([nat.gen_uniform_halos(8, 30, 0), nat.gen_face_halos(9, 10, 30, margin=5.0)])
    nat.write_halo_file(d / "br_h.list", h)
    return dict(particle_files=["br_p.dat"], halo_file="br_h.list", radius="600:1:12")


def _c1(d: pathlib.Path) -> dict:
    # The CPU-runnable workload: 1e6 uniform particles (seed 1), 1e4 uniform
    # halos (seed 2) plus 500 halos within 5 of the faces (seed 3), 40 shells.
    nat.write_particle_file(d / "c1_p.dat", nat.gen_uniform_particles(1, 1, 1_000_000))
    h = np.concatenate([nat.gen_uniform_halos(2, 10000, 0), nat.gen_face_halos(3, 500, 10000, margin=5.0)])
    nat.write_halo_file(d / "c1_h.list", h)
    return dict(particle_files=["c1_p.dat"], halo_file="c1_h.list", radius="0.001:5:40", threads=4)


def _compressed(d: pathlib.Path) -> dict:
    # Two compressed (Gadget-encoded) files of one 100^3 lattice, ids 1.. and
    # 500001.., displacements in [-4, 4) at 16 bits; --compressed.
    for k, (seed, id0) in enumerate([(41, 1), (42, 500_001)]):
        hdr, uv = nat.gen_compressed(seed, 100, 1000.0, -4.0, 4.0, 16, id0, 500_000)
        nat.write_compressed_file(d / f"cp_{k}.dat", hdr, uv)
    h = np.concatenate([nat.gen_uniform_halos(43, 3000, 0), nat.gen_face_halos(44, 200, 3000, margin=5.0)])
    nat.write_halo_file(d / "cp_h.list", h)
    return dict(particle_files=["cp_0.dat", "cp_1.dat"], halo_file="cp_h.list", radius="0.001:5:40",
                extra=["--compressed"], compressed=True)


# Compressed decode vectors: (seed, n1d, box, disp_min, disp_max, pos_bits, id_start, n)
DECODE_SETS = [(1, 60, 1000.0, -3.1, 4.7, 16, 7, None), (2, 37, 1000.0, -11.3, 9.9, 12, 0, 40000),
               (3, 100, 999.7, 0.0, 2.5, 9, 123456, 300000), (4, 128, 1000.0, -6.0, 6.0, 16, 1, 200000)]

# Cases whose particle files are compressed (run with --compressed).
COMPRESSED_CASES = {"compressed": _compressed}

CASES = {
    "kat": _kat,
    "uniform_small": _uniform_small,
    "multi_file": _multi_file,
    "edge": _edge,
    "big_radius": _big_radius,
    "c1": _c1,
}


def materialize(name: str, d: pathlib.Path) -> dict:
    d = pathlib.Path(d)
    d.mkdir(parents=True, exist_ok=True)
    spec = {**CASES, **COMPRESSED_CASES}[name](d)
    spec["nrads"] = int(spec["radius"].split(":")[-1])
    return spec


def cli_args(spec: dict, output: str, backlog: int = 0) -> list:
    t = spec.get("threads", 2)
    args = ["--thread", str(t + (1 if backlog else 0)), "--next-setup", str(t), "--particle-files",
            *spec["particle_files"], "--halo-file", spec["halo_file"], "--radius", spec["radius"],
            "--output-file", output]
    if backlog:
        args += ["--backlog", str(backlog)]
    return args + spec.get("extra", [])


def load_halos_and_particles(spec: dict, d: pathlib.Path):
    """(halos as the reader sees them, list of particle arrays) for API-level tests."""
    d = pathlib.Path(d)
    extra = spec.get("extra", [])
    filt = d / extra[1] if "--filter-file" in extra else None
    halos = nat.read_halos(d / spec["halo_file"], filter_path=filt)
    if spec.get("compressed"):
        parts = [nat.read_compressed(d / f) for f in spec["particle_files"]]  # (header, uv) per file
    else:
        parts = [nat.read_particles(d / f) for f in spec["particle_files"]]
    return halos, parts


def radius_spec(spec: dict):
    mn, mx, n = spec["radius"].split(":")
    return float(mn), float(mx), int(n)
