"""sjcs_rcount keeps astr_rcount's command line: same validation, same messages,
same execution-info block (src/astr_rcount/main.c:492-626).  These runs stop
at validation, before any GPU call, so they run on CPU."""
from __future__ import annotations

import subprocess

import pytest

from conftest import ROOT
from oracle import oracle

DRIVER = ROOT / "spatialjoincountovershells_b200" / "bin" / "sjcs_rcount"

BAD = [
    [],
    ["--radius", "0.001:5:40"],
    ["--radius", "5:5:10", "--thread", "2", "--next-setup", "2"],
    ["--radius", "5:0.001:40", "--thread", "2", "--next-setup", "3", "--particle-files", "a", "--halo-file", "b"],
    ["--radius", "0.001:5:40", "--thread", "2", "--next-setup", "1", "--backlog", "-1", "--particle-files", "a"],
    ["--radius", "0.001:5:40", "--thread", "4", "--next-setup", "1", "--backlog", "1", "--first-setup", "2:1",
     "--particle-files", "a", "--halo-file", "b"],
    ["--radius", "0.001:5:40", "--thread", "2", "--next-setup", "2", "--backlog", "1", "--particle-files", "a",
     "--halo-file", "b"],
    ["--radius", "0.001:5:40", "--thread", "2", "--next-setup", "2", "--particle-files", "--halo-file", "h"],
    ["--radius", "0.001:5:40", "--thread", "2", "--next-setup", "2", "--particle-files", "p1", "p2"],
    ["--radius", "1", "--thread", "2", "--next-setup", "2", "--particle-files", "p", "--halo-file", "h"],
    ["--radius", "-1:2:3", "--thread", "0", "--next-setup", "0", "--particle-files", "p", "--halo-file", "h"],
    ["--thread", "3", "--thread", "1", "--next-setup", "2", "--radius", "0.1:1:4", "--particle-files", "p",
     "--halo-file", "h", "--compressed"],
]


def _run(exe, args):
    r = subprocess.run([str(exe), *args], capture_output=True, text=True, timeout=60)
    return r.returncode, r.stdout, r.stderr.replace(str(exe), "PROG")


@pytest.mark.parametrize("args", BAD, ids=[str(i) for i in range(len(BAD))])
def test_validation_matches_reference(args, built):
    code, out, err = _run(DRIVER, args)
    assert code == 1
    assert out.startswith("\n--execution info--\n")
    assert "=> " in err and "Usage: PROG" in err
    if oracle.ref_available():
        rcode, rout, rerr = _run(oracle.REF_ASTR, args)
        assert (code, out, err) == (rcode, rout, rerr.replace(str(oracle.REF_ASTR), "PROG"))


def test_compressed_option_is_accepted(tmp_path, built):
    # --compressed passes validation and reaches the run (which, without a
    # GPU, stops at the device; the decode itself is tested on the GPU)
    code, out, err = _run(DRIVER, ["--thread", "1", "--next-setup", "1", "--radius", "0.1:1:4",
                                   "--particle-files", "p", "--halo-file", "h", "--compressed"])
    assert "compressed = true" in out and "not supported" not in err
    assert code == 0 or (code == 1 and "ERROR:" in err)
