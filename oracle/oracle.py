"""TEST INFRASTRUCTURE ONLY -- the oracle.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, and
nowhere else.  Two checkers:

* ``liboracle.so`` (oracle/sjcs_oracle.c): a CPU restatement of the
  reference's periodic multi-shell count, pinned against the golden vectors
  in tests/golden/ (produced by the reference program itself).
* ``oracle/_ref/*.exe``: the reference program compiled from its own sources
  (oracle/Makefile).  Present wherever the repository was built next to the
  reference sources; it travels with the built libraries.
"""
from __future__ import annotations

import ctypes
import os
import pathlib
import re
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
REF_DIR = HERE / "_ref"
REF_ASTR = REF_DIR / "astr_rcount.exe"
REF_RT = REF_DIR / "rt_rcount.exe"
REF_PGEN = REF_DIR / "uniform_decoded_particle_generator.exe"
REF_HGEN = REF_DIR / "uniform_halo_generator.exe"

_lib = None


def build_port() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE), "port"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build_port()
        L = ctypes.CDLL(str(LIB))
        vp, u64 = ctypes.c_void_p, ctypes.c_uint64
        L.oracle_radius_table.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, vp]
        L.oracle_count.argtypes = [vp, u64, vp, ctypes.c_size_t, u64, vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int]
        L.oracle_count_brute.argtypes = [vp, u64, vp, ctypes.c_size_t, u64, vp, ctypes.c_int, ctypes.c_int, vp]
        L.oracle_decode_compressed.argtypes = [vp, vp, u64, vp]
        _lib = L
    return _lib


def radius_table(minrad: float, maxrad: float, nrads: int, use_fma: bool = True) -> np.ndarray:
    out = np.zeros(nrads, dtype=np.float32)
    if lib().oracle_radius_table(minrad, maxrad, nrads, 1 if use_fma else 0, out.ctypes.data) != 0:
        raise ValueError("bad radius table arguments")
    return out


def _halo_view(halos):
    """(base address, stride, n, keepalive) of halo centres: HALO_DTYPE or (n,3) float32."""
    if isinstance(halos, np.ndarray) and halos.dtype.names and "point" in halos.dtype.names:
        arr = np.ascontiguousarray(halos)
        return arr.ctypes.data + arr.dtype.fields["point"][1], arr.dtype.itemsize, len(arr), arr
    arr = np.ascontiguousarray(halos, dtype=np.float32).reshape(-1, 3)
    return arr.ctypes.data, 12, len(arr), arr


def count(particles, halos, r2, periodic: bool = True, nthreads: int = 0, brute: bool = False,
          counts: np.ndarray | None = None) -> np.ndarray:
    """uint64 [nhalos, nrads] shell counts (added to `counts` if given)."""
    p = np.ascontiguousarray(particles, dtype=np.float32).reshape(-1, 3)
    base, stride, n, keep = _halo_view(halos)
    r2 = np.ascontiguousarray(r2, dtype=np.float32)
    if counts is None:
        counts = np.zeros((n, len(r2)), dtype=np.uint64)
    if brute:
        rc = lib().oracle_count_brute(p.ctypes.data, len(p), base, stride, n, r2.ctypes.data, len(r2),
                                      1 if periodic else 0, counts.ctypes.data)
    else:
        rc = lib().oracle_count(p.ctypes.data, len(p), base, stride, n, r2.ctypes.data, len(r2),
                                1 if periodic else 0, counts.ctypes.data, nthreads)
    if rc != 0:
        raise RuntimeError("oracle_count failed")
    del keep
    return counts


def ref_available() -> bool:
    return REF_ASTR.exists() and os.access(REF_ASTR, os.X_OK)


def run_ref(args, exe=REF_ASTR, cwd=None, timeout=None) -> subprocess.CompletedProcess:
    return subprocess.run([str(exe), *map(str, args)], cwd=cwd, capture_output=True, text=True, timeout=timeout)


_LINE = re.compile(rb"^  \[[^\]]*\]: (\d+)$")


def parse_result_text(data: bytes, nrads: int):
    """Result text -> (ids uint64 [n], counts uint64 [n, nrads], totals uint64 [nrads])."""
    lines = data.split(b"\n")
    ids, rows = [], []
    i = 0
    while i < len(lines) and lines[i].startswith(b"id "):
        ids.append(int(lines[i][3:]))
        rows.append([int(_LINE.match(lines[i + 1 + k]).group(1)) for k in range(nrads)])
        i += 1 + nrads
    assert lines[i] == b"" and lines[i + 1] == b"Total", "unexpected result layout"
    totals = [int(_LINE.match(lines[i + 2 + k]).group(1)) for k in range(nrads)]
    return (np.array(ids, dtype=np.uint64), np.array(rows, dtype=np.uint64).reshape(len(ids), nrads),
            np.array(totals, dtype=np.uint64))


def ref_phase_times(stdout: str) -> dict:
    """Sum of each '>>>> <phase> time: N milli seconds' line of a reference run."""
    out: dict = {}
    for m in re.finditer(r">>>> (.+?) time: (\d+) milli seconds", stdout):
        out[m.group(1)] = out.get(m.group(1), 0) + int(m.group(2))
    return out


def decode_compressed(header_bytes: bytes, uv) -> np.ndarray:
    """(n, 3) float32 positions of compressed particles (oracle restatement)."""
    uv = np.ascontiguousarray(uv, dtype=np.uint16).reshape(-1, 3)
    hdr = ctypes.create_string_buffer(bytes(header_bytes), 256)
    out = np.empty((len(uv), 3), np.float32)
    rc = lib().oracle_decode_compressed(hdr, uv.ctypes.data if len(uv) else None, len(uv),
                                        out.ctypes.data if len(uv) else None)
    if rc != 0:
        raise ValueError("oracle_decode_compressed rejected the header")
    return out


REF_DECODE = REF_DIR / "ref_decode.exe"


def ref_decode(path: str) -> np.ndarray:
    """Positions of a compressed file decoded by the reference's own decoder
    (oracle/ref_decode.c linked with its sources; test-fixture generation only)."""
    r = subprocess.run([str(REF_DECODE), str(path)], capture_output=True, check=True)
    return np.frombuffer(r.stdout, dtype=np.float32).reshape(-1, 3).copy()
