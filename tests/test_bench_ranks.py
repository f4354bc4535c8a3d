"""bench.py's multi-rank plumbing on CPU (gloo, world size 2).

The path shards into independent replicas, so ranks meet only at barriers
and in a MAX reduction of the timed region; these tests exercise exactly that
with two real processes, and the reference arm under torchrun (rank 0 runs
the CPU reference, the other rank exits without work).
"""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT
from oracle import oracle


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


WORKER = r"""
import os, sys, json
sys.path.insert(0, {root!r})
import bench
dist, rank, world, local = bench.dist_setup("gloo")
bench.dist_barrier(dist)
t = bench.dist_max(dist, 10.0 + rank * 5.0)
bench.dist_barrier(dist)
print(json.dumps({{"rank": rank, "world": world, "max": t}}), flush=True)
bench.dist_close(dist)
"""


def test_max_over_ranks_with_gloo(tmp_path):
    port = _free_port()
    script = tmp_path / "w.py"
    script.write_text(WORKER.format(root=str(ROOT)))
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e
    res = sorted((json.loads(o.strip().splitlines()[-1]) for o, _ in outs), key=lambda d: d["rank"])
    assert [d["rank"] for d in res] == [0, 1]
    assert all(d["world"] == 2 and d["max"] == 15.0 for d in res)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference binaries not built")
def test_reference_arm_under_torchrun_prints_one_line(built):
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--small"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "halos/s"
    assert d["cpu_baseline"]["kind"] == "reference" and d["e2e"]["h2d_bytes_per_step"] == 0
