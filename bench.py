#!/usr/bin/env python
"""Benchmark of the SJCS hot path (index build + periodic multi-shell count) on B200.

Workload (one "step"): the README-scale run of the reference -- 3 particle
files x 1e8 uniform particles (the reference generator's MT19937 stream,
seed 1), 1e7 uniform halos (seed 2, values as read back from the generated
text), --radius 0.001:5:40, periodic.  A step prepares the halos (upload,
Morton sort), then for every file builds the grid index and counts all
halos' shells into the per-halo accumulators.  Builds of file k+1 run on the
build stream while file k is counted on the count stream.

  value   halo-file passes per second (nhalos * nfiles / step time), inputs
          already resident in HBM; device time from CUDA events.
  e2e     the same through the C ABI with HOST buffers: pinned particle and
          halo buffers copied in, uint64 counts copied back every step.
  roofline  the shell-count kernel: algorithmic bytes per halo-file
          (12 + 8*nrads + 12*density*(2R)^3 = 1532 B) x halos per launch
          over its average launch time (CUDA events on the count stream).
  cpu_baseline  the reference program (oracle/_ref/astr_rcount.exe) on a
          bounded sample of the same workload on this host's cores.

--impl reference times that reference program alone (the reference arm).
Under torchrun with N ranks every rank runs an independent replica
(the path has no exchange step); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "halos/s + build s (1e7 halos×3e8 parts), learned vs plain index, exact counts"
UNIT = "halos/s"
# README.md:137 of the reference: 3 files x 1e7 halos in 84104 ms ("total searching time", 20 threads)
PUBLISHED_HALO_FILES_PER_S = 3 * 10_000_000 / 84.104
ALGO_BYTES_PER_HALO_FILE = 1532.0  # 12 (halo) + 8*40 (u32 counts read+write) + 12*0.1*10^3 (in-box particles)

FULL = dict(nfiles=3, nparticles=100_000_000, nhalos=10_000_000, radius=(0.001, 5.0, 40), pseed=1, hseed=2)
SMALL = dict(nfiles=3, nparticles=2_000_000, nhalos=200_000, radius=(0.001, 5.0, 40), pseed=1, hseed=2)


def workload_name(w) -> str:
    return (f"uniform {w['nfiles']} files x {w['nparticles']:.0e} particles (seed {w['pseed']}), "
            f"{w['nhalos']:.0e} halos (seed {w['hseed']}), --radius {w['radius'][0]}:{w['radius'][1]}:"
            f"{w['radius'][2]} periodic")


# ---------------------------------------------------------------------------
# ranks (replicas only: the path shards without an exchange step)
# ---------------------------------------------------------------------------

def dist_setup(backend: str | None = None):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return None, 0, 1, 0
    import datetime

    import torch.distributed as dist
    if backend is None:
        import torch
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist, dist.get_rank(), dist.get_world_size(), int(os.environ.get("LOCAL_RANK", "0"))


def dist_barrier(dist, device=None):
    if dist is not None:
        if device is not None and dist.get_backend() == "nccl":
            dist.barrier(device_ids=[device])
        else:
            dist.barrier()


def dist_max(dist, value: float, device=None) -> float:
    """Max of a per-rank scalar over all ranks (identity with one rank)."""
    if dist is None:
        return value
    import torch
    dev = f"cuda:{device}" if (device is not None and dist.get_backend() == "nccl") else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_close(dist):
    if dist is not None:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        # nvidia-smi numbers GPUs physically; address ours by UUID so that
        # CUDA_VISIBLE_DEVICES remapping cannot make us sample another GPU
        self.device = str(device)
        try:
            import torch
            u = str(torch.cuda.get_device_properties(device).uuid)
            self.device = u if u.startswith("GPU-") else f"GPU-{u}"
        except Exception:
            pass
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def __enter__(self):
        exe = shutil.which("nvidia-smi")
        if exe:
            self.proc = subprocess.Popen([exe, f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._pump, daemon=True)
            self.thread.start()
        return self

    def _pump(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=5)

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference program on a bounded sample
# ---------------------------------------------------------------------------

def ref_threads() -> int:
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    # the reference's build uses unfenced spin barriers that collapse when every core is busy
    return max(1, min(n - 1, 64))


def reference_sample(w, particles_file0, tmp: pathlib.Path, nhalos_sample: int):
    """Write the reference's inputs for one file and a halo prefix sample."""
    from spatialjoincountovershells_b200 import _native as nat
    pf = tmp / "part0.dat"
    if not pf.exists():
        nat.write_particle_file(pf, particles_file0)
    hf = tmp / "halo_sample.list"
    if not hf.exists():
        nat.gen_uniform_halo_file(hf, w["hseed"], nhalos_sample)
    return pf, hf


def run_reference_once(w, pf, hf, threads: int):
    from oracle import oracle
    mn, mx, nr = w["radius"]
    r = oracle.run_ref(["--thread", threads, "--next-setup", threads, "--particle-files", pf.name,
                        "--halo-file", hf.name, "--radius", f"{mn}:{mx}:{nr}", "--output-file", "/dev/null"],
                       cwd=pf.parent, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(f"reference failed: {r.stderr[-500:]}")
    t = oracle.ref_phase_times(r.stdout)
    return t.get("index construction", 0) / 1e3, t.get("searching", 0) / 1e3


def reference_extrapolate(w, build_s: float, search_s: float, nhalos_sample: int) -> float:
    """Halo-file passes per second of the full workload from one sampled file."""
    full_s = w["nfiles"] * (build_s + search_s * w["nhalos"] / nhalos_sample)
    return w["nhalos"] * w["nfiles"] / full_s


def port_baseline(w, particles_file0, halos_sample, r2):
    """Fallback when the reference program is not built: the oracle port, single thread."""
    from oracle import oracle
    t0 = time.perf_counter()
    oracle.count(particles_file0, halos_sample, r2, nthreads=1)
    dt = time.perf_counter() - t0
    return w["nhalos"] * w["nfiles"] / (w["nfiles"] * dt * w["nhalos"] / len(halos_sample))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def profile_traffic(nhalos: int):
    """DRAM bytes per count launch from the committed ncu summary, scaled to nhalos."""
    p = ROOT / "profiles" / "shell_count_uniform.md"
    if not p.exists():
        return None
    m = re.search(r"dram_bytes_per_halo_file:\s*([0-9.eE+]+)", p.read_text())
    return float(m.group(1)) * nhalos if m else None


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def run_ours(args, w, dist, rank, world, local):
    import numpy as np
    import torch

    from spatialjoincountovershells_b200 import _native as nat

    torch.cuda.set_device(local)
    n, nf, nh = w["nparticles"], w["nfiles"], w["nhalos"]
    mn, mx, nr = w["radius"]
    r2 = nat.radius_table(mn, mx, nr)
    R = math.sqrt(float(r2[-1]))

    # host inputs in pinned memory (the e2e leg copies from these every step)
    parts_h = torch.empty((nf * n, 3), dtype=torch.float32, pin_memory=True)
    pnp = parts_h.numpy()
    from spatialjoincountovershells_b200._native import _hcheck, host_lib
    _hcheck(host_lib().sjcs_gen_uniform_particles(w["pseed"], nf, n, pnp.ctypes.data))
    all_halos = nat.gen_uniform_halos(w["hseed"], nh)
    if args.halo_slab is not None:
        all_halos = all_halos[all_halos["point"][:, 2] < args.halo_slab]
        nh = w["nhalos"] = len(all_halos)
    halos_pinned = torch.empty((nh * 24,), dtype=torch.uint8, pin_memory=True)
    halos_np = halos_pinned.numpy().view(nat.HALO_DTYPE)
    halos_np[:] = all_halos
    del all_halos
    out_h = torch.empty((nh * nr,), dtype=torch.int64, pin_memory=True)
    out_np = out_h.numpy().view(np.uint64).reshape(nh, nr)

    ctx = nat.Context(local)
    # grow the device pool once, so no step takes new memory from the driver:
    # K+1 queries, 4 indexes and one build's scratch
    idx_bytes = n * 16 + int(1.6 * n + 4096) * 4
    ctx.reserve((args.steps + 1) * nh * (16 + 4 * nr + 48) + 4 * idx_bytes + n * 44 + (1 << 30))
    s_build = torch.cuda.ExternalStream(ctx.stream(0))
    s_count = torch.cuda.ExternalStream(ctx.stream(1))

    # resident copies for `value`
    parts_d = [torch.from_numpy(pnp[f * n:(f + 1) * n]).cuda() for f in range(nf)]
    halos_d = torch.from_numpy(np.ascontiguousarray(halos_np["point"])).cuda()
    torch.cuda.synchronize()

    def step_resident():
        q = ctx.query(halos_d, r2)
        for f in range(nf):
            idx = ctx.build_index(parts_d[f], radius_hint=R)
            q.count(idx)
            idx.destroy()
        return q

    def step_e2e():
        q = ctx.query(halos_np, r2)
        for f in range(nf):
            idx = ctx.build_index(pnp[f * n:(f + 1) * n], radius_hint=R)
            q.count(idx)
            idx.destroy()
        q.read_counts(out=out_np, accumulate=False)
        return q

    def timed(step, K, W, keep_queries):
        for _ in range(W):
            q = step()
            ctx.sync()
            q.destroy()
        dist_barrier(dist, local)
        torch.cuda.synchronize()
        ctx.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = nat.launch_counter()
        with ClockSampler(local) as clk:
            e0.record(s_count)
            s_build.wait_event(e0)
            qs = []
            for _ in range(K):
                q = step()
                # a step is one job: the next one starts when this one is done,
                # so builds never run ahead into the next step's files
                q.wait()
                if keep_queries:
                    qs.append(q)
                else:
                    q.destroy()
            e1.record(s_count)
            e1.synchronize()
        launches = nat.launch_counter() - l0
        ctx.sync()
        torch.cuda.synchronize()
        dist_barrier(dist, local)
        ms = e0.elapsed_time(e1) / K
        cnt_ms, calls = 0.0, 0
        for q in qs:
            t = q.timing()
            cnt_ms += t["count_ms"]
            calls += t["count_calls"]
            q.destroy()
        return ms, launches, (cnt_ms / calls if calls else None), clk.summary()

    K, W = args.steps, args.warmup
    ms, launches, count_ms, clocks = timed(step_resident, K, W, keep_queries=True)
    ms = dist_max(dist, ms, local)
    if args.no_e2e:
        ms_e2e, launches_e2e, clocks_e2e = float("nan"), 0, None
    else:
        ms_e2e, launches_e2e, _, clocks_e2e = timed(step_e2e, K, W, keep_queries=False)
        ms_e2e = dist_max(dist, ms_e2e, local)

    # one extra untimed pass for the per-phase split (build vs search)
    q = ctx.query(halos_d, r2)
    bt = []
    for f in range(nf):
        idx = ctx.build_index(parts_d[f], radius_hint=R)
        q.count(idx)
        idx.wait()
        bt.append(idx.timing()["build_ms"])
        idx.destroy()
    qt = q.timing()
    q.destroy()
    # correctness spot-check of the timed path on a halo sample (oracle, file 0)
    check = None
    if rank == 0 and not args.no_check and not args.no_e2e:
        from oracle import oracle
        sample = 2000
        got = out_np[:sample]
        want = np.zeros((sample, nr), np.uint64)
        for f in range(nf):
            oracle.count(pnp[f * n:(f + 1) * n], halos_np[:sample], r2, counts=want)
        check = bool(np.array_equal(got, want))

    units = nh * nf * world
    value = units / (ms / 1e3)
    e2e_value = units / (ms_e2e / 1e3)
    peak, peak_kind = measured_peak()
    roof = None
    if count_ms:
        achieved = ALGO_BYTES_PER_HALO_FILE * nh / (count_ms / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": profile_traffic(nh),
                "kernel": "k_shell_count", "launch_ms": round(count_ms, 3),
                "algorithmic_bytes_per_launch": ALGO_BYTES_PER_HALO_FILE * nh,
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_leg(w, pnp[:n], halos_np, r2)

    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": round(value / PUBLISHED_HALO_FILES_PER_S, 2),
        "vs_baseline_ref": "reference README.md:137, 3 files x 1e7 halos in 84104 ms on 20 CPU threads",
        "dtype": "f32", "data": "synthetic: reference generator streams (MT19937 seeds 1 and 2)",
        "config": {"workload": workload_name(w), "index": "grid (radix-sorted cell table)",
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs larger than L2 (3 x 1.2 GB particle arrays per step)"},
        "build_s_per_file": round(statistics.mean(bt) / 1e3, 5),
        "search_halos_per_s": round(nh * nf / (qt["count_ms"] / 1e3), 1) if qt["count_ms"] else None,
        "e2e": None if args.no_e2e else {
            "value": round(e2e_value, 1), "unit": UNIT, "ms_per_step": round(ms_e2e, 3),
            "h2d_bytes_per_step": int(nf * n * 12 + (nh - 1) * 24 + 12),
            "d2h_bytes_per_step": int(nh * nr * 8)},
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "clocks_e2e": clocks_e2e,
        "gpu_launches": int(launches),
        "gpu_launches_e2e": int(launches_e2e),
        "parity_spot_check": check,
    }
    ctx.close()
    return line


def cpu_baseline_leg(w, particles_file0, halos, r2):
    from oracle import oracle
    nhs = 100_000 if w["nhalos"] >= 1_000_000 else max(1000, w["nhalos"] // 10)
    with tempfile.TemporaryDirectory(prefix="sjcs_ref_") as td:
        tmp = pathlib.Path(td)
        if oracle.ref_available():
            pf, hf = reference_sample(w, particles_file0, tmp, nhs)
            T = ref_threads()
            b, s = run_reference_once(w, pf, hf, T)
            return {"value": round(reference_extrapolate(w, b, s, nhs), 1), "unit": UNIT, "cores": T,
                    "kind": "reference",
                    "sample": f"astr_rcount --thread {T} --next-setup {T} on 1 file of {w['nparticles']:.0e} "
                              f"particles x {nhs} halos (prefix of the halo stream); build {b:.3f} s, search "
                              f"{s:.3f} s; extrapolated to {w['nfiles']} files x {w['nhalos']:.0e} halos"}
        v = port_baseline(w, particles_file0, halos[:nhs], r2)
        return {"value": round(v, 1), "unit": UNIT, "cores": 1, "kind": "port",
                "sample": f"oracle port, 1 thread, 1 file x {nhs} halos, extrapolated"}


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------

def run_reference_arm(args, w):
    from oracle import oracle

    from spatialjoincountovershells_b200 import _native as nat
    if not oracle.ref_available():
        return {"impl": "reference", "metric": METRIC, "unit": UNIT,
                "unavailable": "reference program not built (oracle/_ref/astr_rcount.exe missing)"}
    nhs = 100_000 if w["nhalos"] >= 1_000_000 else max(1000, w["nhalos"] // 10)
    T = ref_threads()
    with tempfile.TemporaryDirectory(prefix="sjcs_refarm_") as td:
        tmp = pathlib.Path(td)
        p0 = nat.gen_uniform_particles(w["pseed"], 1, w["nparticles"])
        pf, hf = reference_sample(w, p0, tmp, nhs)
        del p0
        # warm-up runs on a small file (untimed): page in the binary and the inputs' cache
        small = tmp / "warm"
        small.mkdir()
        wpf, whf = reference_sample(dict(w, nparticles=1_000_000), nat.gen_uniform_particles(w["pseed"], 1, 1_000_000),
                                    small, min(nhs, 10_000))
        for _ in range(args.warmup):
            run_reference_once(w, wpf, whf, T)
        times = [run_reference_once(w, pf, hf, T) for _ in range(args.steps)]
    b = statistics.mean(t[0] for t in times)
    s = statistics.mean(t[1] for t in times)
    v = reference_extrapolate(w, b, s, nhs)
    full_ms = 1e3 * w["nhalos"] * w["nfiles"] / v
    sample = (f"astr_rcount --thread {T} --next-setup {T}: per step 1 file of {w['nparticles']:.0e} particles "
              f"(build {b:.3f} s) and {nhs} halos (search {s:.3f} s), extrapolated to {w['nfiles']} files x "
              f"{w['nhalos']:.0e} halos")
    return {
        "impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": UNIT, "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(full_ms, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": round(v / PUBLISHED_HALO_FILES_PER_S, 3), "dtype": "f32",
        "data": "synthetic: reference generator streams (MT19937 seeds 1 and 2)",
        "config": {"workload": workload_name(w), "index": "reference STR tree (CPU)", "parallelism": "cpu threads"},
        "build_s_per_file": round(b, 3),
        "cpu_baseline": {"value": round(v, 1), "unit": UNIT, "cores": T, "kind": "reference", "sample": sample},
        "e2e": {"value": round(v, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--small", action="store_true", help="a 50x smaller workload (smoke runs, CPU tests)")
    ap.add_argument("--files", type=int, default=None, help="override the number of particle files")
    ap.add_argument("--halos", type=int, default=None, help="override the number of halos (same density)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--halo-slab", type=float, default=None,
                    help="keep only halos with z < SLAB (profiling at full halo density on fewer halos)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-check", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    w = dict(SMALL if args.small else FULL)
    if args.files:
        w["nfiles"] = args.files
    if args.halos:
        w["nhalos"] = args.halos
    if args.impl == "reference":
        # the reference is a CPU program: rank 0 alone runs it, other ranks exit
        if int(os.environ.get("RANK", "0")) != 0:
            return
        print(json.dumps(run_reference_arm(args, w)), flush=True)
        return
    dist, rank, world, local = dist_setup()
    line = run_ours(args, w, dist, rank, world, local)
    dist_close(dist)
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
