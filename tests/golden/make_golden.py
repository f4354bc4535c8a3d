"""Regenerate the golden vectors from the reference program itself.

Needs oracle/_ref/astr_rcount.exe and rt_rcount.exe, which `make -C oracle ref`
compiles from the reference's own sources.  For every case of cases.py it
writes the inputs into a scratch directory, runs astr_rcount (and rt_rcount,
the reference's independent R-tree implementation, recording whether it
agrees byte for byte), and stores:

  golden/<case>.npz     ids, counts [n, nrads] and the Total row, parsed from the text
  golden/manifest.json  per case: command line, sha256 and size of the result text
  golden/kat_result.txt the full result text of the periodic known-answer case

  golden/compressed_decode.npz  the reference decoder's output for compressed
                        particles (oracle/_ref/ref_decode.exe, see decode_vectors)

Usage:  python tests/golden/make_golden.py [case ... | decode]
"""
from __future__ import annotations

import hashlib
import json
import pathlib
import sys
import tempfile

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE.parent))

import numpy as np  # noqa: E402

from golden import cases  # noqa: E402
from oracle import oracle  # noqa: E402


def main(names):
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/astr_rcount.exe is missing: run `make -C oracle ref` first")
    man_path = HERE / "manifest.json"
    manifest = json.loads(man_path.read_text()) if man_path.exists() else {}
    for name in names:
        with tempfile.TemporaryDirectory() as td:
            d = pathlib.Path(td)
            spec = cases.materialize(name, d)
            args = cases.cli_args(spec, "astr.txt")
            r = oracle.run_ref(args, cwd=d)
            if r.returncode != 0:
                raise SystemExit(f"{name}: astr_rcount failed:\n{r.stderr}")
            r2 = oracle.run_ref(cases.cli_args(spec, "rt.txt"), exe=oracle.REF_RT, cwd=d)
            if r2.returncode != 0:
                raise SystemExit(f"{name}: rt_rcount failed:\n{r2.stderr}")
            text = (d / "astr.txt").read_bytes()
            # rt_rcount skips the rest of a leaf after a particle at distance 0
            # (src/objects/RTree/MultiRangeCount.c:103-104), so it only agrees
            # with astr_rcount when no particle coincides with a halo centre.
            rt_agrees = text == (d / "rt.txt").read_bytes()
            ids, counts, totals = oracle.parse_result_text(text, spec["nrads"])
            np.savez_compressed(HERE / f"{name}.npz", ids=ids, counts=counts, totals=totals)
            manifest[name] = {
                "args": args,
                "radius": spec["radius"],
                "nrads": spec["nrads"],
                "nhalos": int(len(ids)),
                "sha256": hashlib.sha256(text).hexdigest(),
                "bytes": len(text),
                "rt_rcount_agrees": rt_agrees,
            }
            if name == "kat":
                (HERE / "kat_result.txt").write_bytes(text)
            print(f"{name}: {len(ids)} halos, {len(text)} bytes, sum={int(counts.sum())}")
    man_path.write_text(json.dumps(manifest, indent=1, sort_keys=True) + "\n")


def decode_vectors():
    """golden/compressed_decode.npz: per decode set of cases.DECODE_SETS, the
    sha256 of the reference decoder's float32 output (oracle/_ref/ref_decode.exe)
    and its first 512 positions."""
    from spatialjoincountovershells_b200 import _native as nat
    shas, heads = [], []
    for (seed, n1d, box, dmin, dmax, bits, id0, n) in cases.DECODE_SETS:
        hdr, uv = nat.gen_compressed(seed, n1d, box, dmin, dmax, bits, id0, n)
        with tempfile.TemporaryDirectory() as td:
            f = pathlib.Path(td) / "c.dat"
            nat.write_compressed_file(f, hdr, uv)
            pos = oracle.ref_decode(f)
        shas.append(hashlib.sha256(pos.tobytes()).hexdigest())
        heads.append(pos[:512])
        print(f"decode set {seed}: {len(pos)} particles")
    np.savez_compressed(HERE / "compressed_decode.npz", sha256=np.array(shas), heads=np.stack(heads))


if __name__ == "__main__":
    names = sys.argv[1:] or [*cases.CASES, *cases.COMPRESSED_CASES, "decode"]
    if "decode" in names:
        decode_vectors()
    main([n for n in names if n != "decode"])
