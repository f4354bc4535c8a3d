"""Compressed (Gadget-encoded) particle files on the GPU.

The device decode must reproduce the reference's decodeCompressedParticle bit
for bit (golden vectors from the reference's own decoder), and the counts and
result text of a --compressed run must equal the reference program's.
"""
from __future__ import annotations

import hashlib
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, golden_counts
from golden import cases
from spatialjoincountovershells_b200 import _native as nat
from test_gpu_parity import DRIVER

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def compressed_case(tmp_path_factory, built):
    d = tmp_path_factory.mktemp("compressed")
    return d, cases.materialize("compressed", d)


def test_device_decode_matches_the_reference_decoder(ctx):
    z = np.load(GOLDEN / "compressed_decode.npz")
    for k, (seed, n1d, box, dmin, dmax, bits, id0, n) in enumerate(cases.DECODE_SETS):
        hdr, uv = nat.gen_compressed(seed, n1d, box, dmin, dmax, bits, id0, n)
        pos = ctx.decode_compressed(uv, hdr)
        assert hashlib.sha256(pos.tobytes()).hexdigest() == z["sha256"][k], k
        assert np.array_equal(pos[:512].view(np.uint32), z["heads"][k].view(np.uint32)), k


@pytest.mark.parametrize("kind", [nat.INDEX_GRID, nat.INDEX_LEARNED])
def test_compressed_counts_match_reference(kind, compressed_case, ctx):
    d, spec = compressed_case
    halos, parts = cases.load_halos_and_particles(spec, d)
    r2 = nat.radius_table(*cases.radius_spec(spec))
    q = ctx.query(halos, r2)
    for hdr, uv in parts:
        idx = ctx.build_index_compressed(uv, hdr, radius_hint=float(np.sqrt(r2[-1])), kind=kind)
        q.count(idx)
        idx.destroy()
    got = q.read_counts()
    q.destroy()
    _, want, _ = golden_counts("compressed")
    assert np.array_equal(got, want)


@pytest.mark.parametrize("backlog", [0, 2])
def test_driver_compressed_text_matches_reference(backlog, compressed_case, manifest, tmp_path):
    d, spec = compressed_case
    out = tmp_path / "result.txt"
    r = subprocess.run([str(DRIVER), *cases.cli_args(spec, str(out), backlog=backlog)], cwd=d,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert hashlib.sha256(out.read_bytes()).hexdigest() == manifest["compressed"]["sha256"]
    assert ">>>> particles decoding + index construction time" in r.stdout or backlog


def test_bad_headers_are_rejected(ctx):
    hdr, uv = nat.gen_compressed(5, 10, 1000.0, -1.0, 1.0, 8, 1, 100)
    empty = bytearray(hdr)
    empty[96:120] = bytes(24)  # npartTotal = 0: no lattice
    with pytest.raises(nat.SjcsError):
        ctx.decode_compressed(uv, bytes(empty))
    with pytest.raises(nat.SjcsError):
        ctx.build_index_compressed(uv, bytes(empty))
    assert ctx.decode_compressed(uv[:0], hdr).shape == (0, 3)
