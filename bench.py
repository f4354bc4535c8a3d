#!/usr/bin/env python
"""Benchmark of the SJCS hot path (index build + periodic multi-shell count) on B200.

Workload (one "step"): the README-scale run of the reference -- 3 particle
files x 1e8 uniform particles (the reference generator's MT19937 stream,
seed 1), 1e7 uniform halos (seed 2, values as read back from the generated
text), --radius 0.001:5:40, periodic.  A step prepares the halos (upload,
Morton sort), then for every file builds the grid index and counts all
halos' shells into the per-halo accumulators.  File k+1's build is queued on
the build stream behind file k's count (its upload overlaps that count).

  value   halo-file passes per second (nhalos * nfiles / step time), inputs
          already resident in HBM; device time from CUDA events.
  e2e     the same through the C ABI with HOST buffers: pinned particle and
          halo buffers copied in, the counts copied back every step (the
          uint32 accumulators: exact while the query has not folded).
          Steps are independent jobs run as a pipeline: job k's count
          read-back (device to host) overlaps job k+1's uploads (host to
          device); every job's copies are inside the timed region.
  roofline  the shell-count kernel (the fused k_shell_count_multi: one launch
          counts the step's halos against all its files): algorithmic bytes
          per halo-file (12 + 8*nrads + 12*density*(2R)^3 = 1532 B) x
          halo-files per launch over its average launch time (CUDA events on
          the count stream).
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
        self.first = threading.Event()

    def __enter__(self):
        exe = shutil.which("nvidia-smi")
        if exe:
            self.proc = subprocess.Popen([exe, f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._pump, daemon=True)
            self.thread.start()
            # nvidia-smi takes a moment to start: the timed region begins only
            # once it is sampling, so even a short region has samples around it
            self.first.wait(timeout=10)
            self.n_enter = len(self.lines)
        return self

    def _pump(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())
            self.first.set()

    def __exit__(self, *exc):
        if self.proc:
            # a region shorter than the sampling period: take the sample that
            # follows it too (the GPU is still at its loaded clocks)
            t_end = time.time() + 1.0
            while len(self.lines) <= getattr(self, "n_enter", 0) and time.time() < t_end:
                time.sleep(0.02)
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


def write_reference_inputs(tmp: pathlib.Path, particles, nfiles: int, halos):
    """Particle files and a halo file in the reference's formats (our arm:
    written by this package's host library from the arrays it counts)."""
    from spatialjoincountovershells_b200 import _native as nat
    n = len(particles) // nfiles
    files = []
    for f in range(nfiles):
        pf = tmp / f"part{f}.dat"
        nat.write_particle_file(pf, particles[f * n:(f + 1) * n])
        files.append(pf)
    hf = tmp / "halo_sample.list"
    nat.write_halo_file(hf, halos)
    return files, hf


def run_reference(files, hf, radius, threads: int, result: bool, timeout=1800):
    """astr_rcount over the particle files and the halo file (same directory).
    Returns its phase times (seconds per file: build, search), wall time and,
    with result=True, its counts parsed from the result text."""
    from oracle import oracle
    mn, mx, nr = radius
    tmp = files[0].parent
    out = tmp / "ref_result.txt"
    t0 = time.perf_counter()
    r = oracle.run_ref(["--thread", threads, "--next-setup", threads, "--particle-files", *[f.name for f in files],
                        "--halo-file", hf.name, "--radius", f"{mn}:{mx}:{nr}",
                        "--output-file", out.name if result else "/dev/null"], cwd=tmp, timeout=timeout)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"reference failed: {r.stderr[-500:]}")
    t = oracle.ref_phase_times(r.stdout)
    res = {"build_s": t.get("index construction", 0) / 1e3 / len(files),
           "search_s": t.get("searching", 0) / 1e3 / len(files), "wall_s": wall, "counts": None}
    if result:
        _, counts, _ = oracle.parse_result_text(out.read_bytes(), nr)
        res["counts"] = counts
        out.unlink()
    return res


def reference_extrapolate(w, build_s: float, search_s: float, nhalos_sample: int) -> float:
    """Halo-file passes per second of the full workload from sampled files
    (build and search seconds per file; search scaled by the halo count)."""
    full_s = w["nfiles"] * (build_s + search_s * w["nhalos"] / nhalos_sample)
    return w["nhalos"] * w["nfiles"] / full_s


def port_baseline(w, particles_file0, halos_sample, r2):
    """Fallback when the reference program is not built: the oracle port, single thread."""
    from oracle import oracle
    t0 = time.perf_counter()
    oracle.count(particles_file0, halos_sample, r2, nthreads=1)
    dt = time.perf_counter() - t0
    return w["nhalos"] * w["nfiles"] / (w["nfiles"] * dt * w["nhalos"] / len(halos_sample))


def parity_record(ref_counts, forms: dict, workload: str, radius) -> dict:
    """Per index form: are its counts for the sampled halos identical to the reference's?"""
    import numpy as np
    m = len(ref_counts)
    res = {name: bool(np.array_equal(c[:m].astype(np.uint64), ref_counts)) for name, c in forms.items()}
    mn, mx, nr = radius
    return {"identical": all(res.values()), "halo_rows_compared": int(m), "shells": int(nr),
            "counts_compared": int(m * nr * len(forms)), "forms": res,
            "reference_total": int(ref_counts.sum()), "workload": workload,
            "against": "astr_rcount result text (the reference compiled from its sources), all particle files"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def profile_traffic(halo_files: float, fused: bool = False):
    """DRAM bytes per count launch from the committed ncu summary of that
    kernel (bytes per halo-file), scaled to the launch's halo-files."""
    p = ROOT / "profiles" / ("shell_count_multi_uniform.md" if fused else "shell_count_uniform.md")
    if not p.exists():
        return None
    m = re.search(r"dram_bytes_per_halo_file:\s*([0-9.eE+]+)", p.read_text())
    return float(m.group(1)) * halo_files if m else None


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
    # read-back destinations: the uint32 accumulators are the exact totals
    # while the query has not folded (the library refuses the read otherwise)
    out_h = torch.empty((nh * nr,), dtype=torch.int32, pin_memory=True)
    out_np = out_h.numpy().view(np.uint32).reshape(nh, nr)

    ctx = nat.Context(local)
    ctx.set_overlap(args.overlap)
    # grow the device pool once, so no step takes new memory from the driver:
    # 3 queries, a read-back's widened counts, two jobs' indexes, the uploaded
    # files and one build's scratch
    idx_bytes = n * 16 + int(1.6 * n + 4096) * 4
    if not args.no_reserve:
        ctx.reserve(3 * nh * (16 + 4 * nr + 48) + nh * nr * 8 + 2 * nf * idx_bytes + nf * n * 12 + n * 44 + (1 << 30))
    s_build = torch.cuda.ExternalStream(ctx.stream(0))
    s_count = torch.cuda.ExternalStream(ctx.stream(1))

    # resident copies for `value`
    parts_d = [torch.from_numpy(pnp[f * n:(f + 1) * n]).cuda() for f in range(nf)]
    halos_d = torch.from_numpy(np.ascontiguousarray(halos_np["point"])).cuda()
    torch.cuda.synchronize()

    def step_resident():
        # every file's index, then one fused count over them (sjcs_query_count_many)
        q = ctx.query(halos_d, r2)
        idxs = [ctx.build_index(parts_d[f], radius_hint=R) for f in range(nf)]
        q.count_many(idxs)
        for idx in idxs:
            idx.destroy()
        return q

    out_h2 = torch.empty((nh * nr,), dtype=torch.int32, pin_memory=True)
    outs = [out_np, out_h2.numpy().view(np.uint32).reshape(nh, nr)]

    def job_e2e(k):
        q = ctx.query(halos_np, r2)
        idxs = [ctx.build_index(pnp[f * n:(f + 1) * n], radius_hint=R) for f in range(nf)]
        q.count_many(idxs)
        for idx in idxs:
            idx.destroy()
        q.read_counts32_async(outs[k & 1])
        return q

    def run_e2e(jobs):
        # at most two jobs in flight: job k is queued before job k-1's
        # read-back is awaited, so the two overlap on the copy engines
        prev = None
        for k in range(jobs):
            q = job_e2e(k)
            if prev is not None:
                prev.wait_read()
                prev.destroy()
            prev = q
        if prev is not None:
            prev.wait_read()
            prev.destroy()

    def timed_e2e(K, W):
        run_e2e(W)
        dist_barrier(dist, local)
        torch.cuda.synchronize()
        ctx.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = nat.launch_counter()
        with ClockSampler(local) as clk:
            e0.record(s_count)
            s_build.wait_event(e0)
            run_e2e(K)
            # recorded after the last read-back was seen complete on the host
            e1.record(s_count)
            e1.synchronize()
        launches = nat.launch_counter() - l0
        ctx.sync()
        torch.cuda.synchronize()
        dist_barrier(dist, local)
        return e0.elapsed_time(e1) / K, launches, clk.summary()

    def timed(step, K, W):
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
            cnt_ms, calls = 0.0, 0
            files_per_call = None
            for _ in range(K):
                q = step()
                # a step is one job: the next one starts when this one is done,
                # so builds never run ahead into the next step's files
                q.wait()
                t = q.timing()  # event pairs already complete: no wait
                cnt_ms += t["count_ms"]
                calls += t["count_calls"]
                q.destroy()
            e1.record(s_count)
            e1.synchronize()
        launches = nat.launch_counter() - l0
        ctx.sync()
        torch.cuda.synchronize()
        dist_barrier(dist, local)
        ms = e0.elapsed_time(e1) / K
        files_per_call = nf * K / calls if calls else None
        return ms, launches, (cnt_ms / calls if calls else None), files_per_call, clk.summary()

    K, W = args.steps, args.warmup
    ms, launches, count_ms, files_per_call, clocks = timed(step_resident, K, W)
    ms = dist_max(dist, ms, local)
    if args.no_e2e:
        ms_e2e, launches_e2e, clocks_e2e = float("nan"), 0, None
    else:
        ms_e2e, launches_e2e, clocks_e2e = timed_e2e(K, W)
        ms_e2e = dist_max(dist, ms_e2e, local)

    # one extra untimed pass for the per-phase split (build vs search)
    nhs = min(nh, 100_000)  # halos compared with the reference program (a prefix of the halo stream)
    q = ctx.query(halos_d, r2)
    bt = []
    for f in range(nf):
        idx = ctx.build_index(parts_d[f], radius_hint=R)
        q.count(idx)
        idx.wait()
        bt.append(idx.timing()["build_ms"])
        idx.destroy()
    qt = q.timing()
    q.wait()
    grid_counts = device_counts(q)
    sample = {"grid": grid_counts[:nhs * nr].cpu().numpy().view(np.uint32).reshape(nhs, nr)}
    q.destroy()
    # the build kernels alone (no count queued before them), for the build roofline
    bk, ncells = [], None
    for _ in range(2):
        for f in range(nf):
            idx = ctx.build_index(parts_d[f], radius_hint=R)
            idx.wait()
            bk.append(idx.timing()["build_ms"])
            g = idx.grid
            ncells = g[0] * g[1] * g[2]
            idx.destroy()

    def counts_of(kind, mode):
        qq = ctx.query(halos_d, r2)
        qq.set_schedule(mode)
        for f in range(nf):
            ix = ctx.build_index(parts_d[f], radius_hint=R, kind=kind)
            qq.count(ix)
            ix.destroy()
        qq.wait()
        c = device_counts(qq)
        qq.destroy()
        return c

    # the persistent-queue schedule on the same index: same counts on the device
    c = counts_of(nat.INDEX_GRID, nat.SCHED_QUEUE)
    queue_same = bool(torch.equal(c, grid_counts))
    sample["grid-queue"] = c[:nhs * nr].cpu().numpy().view(np.uint32).reshape(nhs, nr)
    del c

    # the other index forms on the same workload (resident leg): the learned
    # index and the plain Morton table, with their counts compared on the device
    forms = None
    if not args.no_forms:
        forms = {}
        for name, kind in (("learned", nat.INDEX_LEARNED), ("morton", nat.INDEX_MORTON)):
            def fstep(kind=kind):
                qq = ctx.query(halos_d, r2)
                for f in range(nf):
                    ix = ctx.build_index(parts_d[f], radius_hint=R, kind=kind)
                    qq.count(ix)
                    ix.destroy()
                return qq
            fms, flaunch, fcount, _ = time_steps(ctx, fstep, K, W, dist, local)
            qq = ctx.query(halos_d, r2)
            fb, info = [], None
            for f in range(nf):
                ix = ctx.build_index(parts_d[f], radius_hint=R, kind=kind)
                qq.count(ix)
                ix.wait()
                fb.append(ix.timing()["build_ms"])
                if kind == nat.INDEX_LEARNED and f == 0:
                    info = ix.learned_info()
                ix.destroy()
            qq.wait()
            c = device_counts(qq)
            same = bool(torch.equal(c, grid_counts))
            sample[name] = c[:nhs * nr].cpu().numpy().view(np.uint32).reshape(nhs, nr)
            del c
            qq.destroy()
            forms[name] = {"value": round(nh * nf * world / (fms / 1e3), 1), "ms_per_step": round(fms, 3),
                           "build_s_per_file": round(statistics.mean(fb) / 1e3, 5),
                           "count_ms_per_file": round(fcount, 3) if fcount else None,
                           "counts_identical_to_grid": same, "gpu_launches": flaunch}
            if info:
                forms[name]["model"] = {"leaves": info["leaves"], "max_err": info["max_err"],
                                        "mean_err": round(info["mean_err"], 1), "level": info["level"]}
    del grid_counts
    torch.cuda.empty_cache()

    units = nh * nf * world
    value = units / (ms / 1e3)
    e2e_value = units / (ms_e2e / 1e3)
    peak, peak_kind = measured_peak()
    roof = None
    if count_ms:
        # one launch counts nh halos against files_per_call indexes
        hf = nh * files_per_call
        achieved = ALGO_BYTES_PER_HALO_FILE * hf / (count_ms / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": profile_traffic(hf, files_per_call > 1),
                "kernel": "k_shell_count_multi" if files_per_call > 1 else "k_shell_count",
                "files_per_launch": round(files_per_call, 3), "launch_ms": round(count_ms, 3),
                "algorithmic_bytes_per_launch": ALGO_BYTES_PER_HALO_FILE * hf,
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind}
    build_ms = statistics.median(bk)
    build_bytes = 24.0 * n + 4.0 * (ncells + 1)  # 12 B read + 12 B written per particle, 4 B per cell
    roof_build = {"bound": "hbm", "achieved": round(build_bytes / (build_ms / 1e3) / 1e9, 1), "peak": peak,
                  "unit": "GB/s", "frac": round(build_bytes / (build_ms / 1e3) / 1e9 / peak, 4),
                  "kernel": "grid index build (partition build: k_pb_top_hist, k_pb_partition x2, k_pb_mid_hist, k_pb_cells)",
                  "build_ms": round(build_ms, 3), "algorithmic_bytes_per_build": build_bytes,
                  "cells": int(ncells)}

    # the reference program on the same host: every particle file of the
    # step and the first nhs halos; its result text is the parity check of
    # every form above at the timed configuration
    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, ref_counts = reference_leg(w, pnp, halos_np[:nhs], r2)
        if ref_counts is not None:
            parity = parity_record(ref_counts, sample, workload_name(w), w["radius"])
    del sample

    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": round(value / PUBLISHED_HALO_FILES_PER_S, 2),
        "vs_baseline_ref": "reference README.md:137, 3 files x 1e7 halos in 84104 ms on 20 CPU threads",
        "dtype": "f32", "data": "synthetic: reference generator streams (MT19937 seeds 1 and 2)",
        "config": {"workload": workload_name(w), "index": "grid (cell table, partition build)",
                   "build_kernels": "beside the counts" if args.overlap else "after the queued counts (copies overlap)",
                   "count": "one fused pass over the step's files (sjcs_query_count_many)",
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": f"inputs larger than L2 ({nf} x {n * 12 / 1e9:.2f} GB particle arrays per step)"},
        "build_s_per_file": round(statistics.mean(bt) / 1e3, 5),
        "search_halos_per_s": round(nh * nf / (qt["count_ms"] / 1e3), 1) if qt["count_ms"] else None,
        "e2e": None if args.no_e2e else {
            "value": round(e2e_value, 1), "unit": UNIT, "ms_per_step": round(ms_e2e, 3),
            "h2d_bytes_per_step": int(nf * n * 12 + (nh - 1) * 24 + 12),
            "d2h_bytes_per_step": int(nh * nr * 4),
            "read_back": "uint32 accumulators, exact without a fold (sjcs_query_read_counts32_async)",
            "pipeline": "job k's read-back overlaps job k+1's uploads (2 jobs in flight)"},
        "roofline": roof,
        "roofline_build": roof_build,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "clocks_e2e": clocks_e2e,
        "gpu_launches": int(launches),
        "gpu_launches_e2e": int(launches_e2e),
        "queue_schedule_counts_identical_to_static": queue_same,
        "forms": forms,
        "parity_at_scale": {"c2": parity} if parity else None,
    }
    ctx.close()
    return line


# ---------------------------------------------------------------------------
# clustered workloads: persistent schedule (config C3), index forms (C4),
# serving (C5).  Each prints its own JSON line; the default line is C2.
# ---------------------------------------------------------------------------

CLUSTERED = dict(workload="clustered", nfiles=3, nparticles=100_000_000, nhalos=10_000_000,
                 radius=(0.01, 20.0, 64), pseed=31, hseed=32)
FORMS = dict(CLUSTERED, workload="learned", radius=(0.001, 5.0, 40))
SERVING = dict(workload="serving", nfiles=3, nparticles=100_000_000, nrequests=2000, size=(1e2, 1e6),
               nrads=(8, 64), rmax=(1.0, 10.0), arrival_seed=51, pseed=31, hseed=32)
IO = dict(workload="io", nfiles=1, nparticles=100_000_000, nhalos=1_000_000, radius=(0.001, 5.0, 40),
          pseed=1, hseed=2)


def clustered_name(w) -> str:
    mn, mx, nr = w["radius"]
    return (f"clustered {w['nfiles']} files x {w['nparticles']:.0e} particles (60% in 1e4 Gaussian clumps, "
            f"sigma log-uniform [2,20], lognormal(0,1.5) weights; seeds {w['pseed']}+file, clumps 31), "
            f"{w['nhalos']:.0e} halos (70% at clump centres, jitter 1; seed {w['hseed']}), "
            f"--radius {mn}:{mx}:{nr} periodic")


class _DeviceU32:
    """A device u32 array seen by torch (zero-copy, via __cuda_array_interface__)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False), "version": 3}


def device_counts(q):
    """A copy of the query's device accumulators (torch, u32 bits as int32).  The
    copy is finished before returning: the query's memory goes back to the
    library's pool when the query is destroyed, and torch's stream is not
    ordered with the library's."""
    import torch
    c = torch.as_tensor(_DeviceU32(q.device_counts_ptr, q.nhalos * q.nrads), device="cuda").clone()
    torch.cuda.synchronize()
    return c


def clustered_inputs(w):
    """Pinned host particles (all files) and halos of a clustered workload."""
    import numpy as np
    import torch

    from spatialjoincountovershells_b200 import _native as nat
    n, nf = w["nparticles"], w["nfiles"]
    parts_h = torch.empty((nf * n, 3), dtype=torch.float32, pin_memory=True)
    for f in range(nf):
        parts_h[f * n:(f + 1) * n] = torch.from_numpy(nat.gen_clustered_particles(w["pseed"] + f, n))
    halos = nat.gen_clustered_halos(w["hseed"], w["nhalos"])
    halos_h = torch.empty((w["nhalos"] * 24,), dtype=torch.uint8, pin_memory=True)
    hnp = halos_h.numpy().view(nat.HALO_DTYPE)
    hnp[:] = halos
    return parts_h, halos_h, hnp, np.ascontiguousarray(halos["point"])


def time_steps(ctx, step, K, W, dist, local):
    """W untimed then K timed steps (one job each) on the context's streams."""
    import torch

    from spatialjoincountovershells_b200 import _native as nat
    s_build = torch.cuda.ExternalStream(ctx.stream(0))
    s_count = torch.cuda.ExternalStream(ctx.stream(1))
    for _ in range(W):
        q = step()
        ctx.sync()
        q.destroy()
    dist_barrier(dist, local)
    torch.cuda.synchronize()
    ctx.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = nat.launch_counter()
    cnt, calls = 0.0, 0
    with ClockSampler(local) as clk:
        e0.record(s_count)
        s_build.wait_event(e0)
        for _ in range(K):
            q = step()
            q.wait()
            # read the count events and release the query at once, so the
            # memory pool holds one step's queries, as in the warm-up
            t = q.timing()
            cnt += t["count_ms"]
            calls += t["count_calls"]
            q.destroy()
        e1.record(s_count)
        e1.synchronize()
    launches = nat.launch_counter() - l0
    ctx.sync()
    dist_barrier(dist, local)
    ms = dist_max(dist, e0.elapsed_time(e1) / K, local)
    return ms, int(launches), (cnt / calls if calls else None), clk.summary()


class ClusteredData:
    """Inputs of the clustered workloads (C3, C4, C5): pinned host copies of
    every file and of the halos, and resident device copies."""

    def __init__(self, w, local):
        import torch

        from spatialjoincountovershells_b200 import _native as nat
        n, nf = w["nparticles"], w["nfiles"]
        self.w = w
        self.parts_h = torch.empty((nf * n, 3), dtype=torch.float32, pin_memory=True)
        self.pnp = self.parts_h.numpy()
        for f in range(nf):
            self.pnp[f * n:(f + 1) * n] = nat.gen_clustered_particles(w["pseed"] + f, n)
        halos = nat.gen_clustered_halos(w["hseed"], w["nhalos"])
        self.halos_h = torch.empty((w["nhalos"] * 24,), dtype=torch.uint8, pin_memory=True)
        self.hnp = self.halos_h.numpy().view(nat.HALO_DTYPE)
        self.hnp[:] = halos
        import numpy as np
        self.parts_d = [torch.from_numpy(self.pnp[f * n:(f + 1) * n]).to(f"cuda:{local}") for f in range(nf)]
        self.halos_d = torch.from_numpy(np.ascontiguousarray(halos["point"])).to(f"cuda:{local}")
        torch.cuda.synchronize()

    def release_device(self):
        import torch
        self.parts_d = None
        self.halos_d = None
        torch.cuda.empty_cache()


def clustered_reference_legs(w, data, legs):
    """astr_rcount on every clustered particle file (written once) for each
    (name, radius, nhalos_sample) leg.  Returns {name: run_reference result}."""
    from oracle import oracle
    if not oracle.ref_available():
        return {}
    from spatialjoincountovershells_b200 import _native as nat
    T = ref_threads()
    out = {}
    with tempfile.TemporaryDirectory(prefix="sjcs_refcl_") as td:
        tmp = pathlib.Path(td)
        n, nf = w["nparticles"], w["nfiles"]
        files = []
        for f in range(nf):
            pf = tmp / f"part{f}.dat"
            nat.write_particle_file(pf, data.pnp[f * n:(f + 1) * n])
            files.append(pf)
        for name, radius, nhs in legs:
            hf = tmp / f"halos_{name}.list"
            nat.write_halo_file(hf, data.hnp[:nhs])
            r = run_reference(files, hf, radius, T, result=True)
            r["threads"] = T
            r["nhs"] = nhs
            out[name] = r
            hf.unlink()
    return out


def clustered_cpu_baseline(w, r) -> dict:
    b, s = r["build_s"], r["search_s"]
    return {"value": round(reference_extrapolate(w, b, s, r["nhs"]), 1), "unit": UNIT, "cores": r["threads"],
            "kind": "reference",
            "sample": f"astr_rcount --thread {r['threads']} --next-setup {r['threads']} on all {w['nfiles']} "
                      f"clustered files of {w['nparticles']:.0e} particles x the first {r['nhs']} halos: build "
                      f"{b:.3f} s and search {s:.3f} s per file (wall {r['wall_s']:.1f} s); extrapolated to "
                      f"{w['nhalos']:.0e} halos"}


def section_c3(args, w, ctx, data, K, W, dist, local, world, nhs):
    """C3: clustered uneven load; autotuned persistent schedule vs static;
    captured file steps; e2e.  Returns (section, counts of the first nhs halos
    per schedule)."""
    import numpy as np

    from spatialjoincountovershells_b200 import _native as nat
    n, nf, nh = w["nparticles"], w["nfiles"], w["nhalos"]
    mn, mx, nr = w["radius"]
    r2 = nat.radius_table(mn, mx, nr)
    R = math.sqrt(float(r2[-1]))
    pnp, hnp, parts_d, halos_d = data.pnp, data.hnp, data.parts_d, data.halos_d
    out_np = np.empty((nh, nr), np.uint64)

    # autotune on file 0 (the choice is cached in the context for this shape)
    idx0 = ctx.build_index(parts_d[0], radius_hint=R)
    qt = ctx.query(halos_d, r2)
    tune = ctx.autotune(qt, idx0)
    qt.destroy()
    idx0.destroy()

    def step_resident(mode):
        def step():
            q = ctx.query(halos_d, r2)
            q.set_schedule(mode)
            for f in range(nf):
                idx = ctx.build_index(parts_d[f], radius_hint=R)
                q.count(idx)
                idx.destroy()
            return q
        return step

    def step_e2e():
        q = ctx.query(hnp, r2)
        for f in range(nf):
            idx = ctx.build_index(pnp[f * n:(f + 1) * n], radius_hint=R)
            q.count(idx)
            idx.destroy()
        q.read_counts(out=out_np)
        return q

    ms, launches, count_ms, clocks = time_steps(ctx, step_resident(nat.SCHED_AUTO), K, W, dist, local)
    ms_static, _, count_static, _ = time_steps(ctx, step_resident(nat.SCHED_STATIC), K, W, dist, local)
    ms_e2e, launches_e2e, _, clocks_e2e = time_steps(ctx, step_e2e, K, W, dist, local)

    sample = {}
    for name, mode in (("grid-queue", nat.SCHED_QUEUE), ("grid-static", nat.SCHED_STATIC)):
        q = step_resident(mode)()
        q.wait()
        c = device_counts(q)
        sample[name] = c[:nhs * nr].cpu().numpy().view(np.uint32).reshape(nhs, nr)
        q.destroy()
        del c

    # captured file steps (graph replays of copy + build + count) against the
    # same query, after W warm-up replays
    q = ctx.query(halos_d, r2)
    st = ctx.step(q, n, radius_hint=R)
    gms = []
    for k in range(W + K):
        st.buffer[:] = pnp[(k % nf) * n:((k % nf) + 1) * n]
        st.launch().wait()
        if k >= W:
            gms.append(st.time_ms())
    st.destroy()
    q.destroy()

    units = nh * nf * world
    sec = {
        "metric": "halos/s (clustered uneven load, persistent schedule)", "value": round(units / (ms / 1e3), 1),
        "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": round(ms, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: project generators (clumped particles and halos, MT19937 block streams)",
        "config": {"workload": clustered_name(w), "index": "grid", "schedule": tune["chosen"],
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": f"inputs larger than L2 ({nf} x {n * 12 / 1e9:.2f} GB particle arrays per step)"},
        "autotune_trial_ms": [round(t, 2) for t in tune["trial_ms"]],
        "count_ms_per_file": round(count_ms, 2) if count_ms else None,
        "static_schedule": {"value": round(units / (ms_static / 1e3), 1), "ms_per_step": round(ms_static, 3),
                            "count_ms_per_file": round(count_static, 2) if count_static else None},
        "captured_step_ms_per_file": round(statistics.mean(gms), 3),
        "e2e": {"value": round(units / (ms_e2e / 1e3), 1), "unit": UNIT, "ms_per_step": round(ms_e2e, 3),
                "h2d_bytes_per_step": int(nf * n * 12 + (nh - 1) * 24 + 12), "d2h_bytes_per_step": int(nh * nr * 8)},
        "roofline": None, "clocks": clocks, "clocks_e2e": clocks_e2e,
        "gpu_launches": launches, "gpu_launches_e2e": launches_e2e,
    }
    return sec, sample


def section_c4(args, w, ctx, data, K, W, dist, local, world, nhs):
    """C4: learned index vs plain forms on the clustered data, each form's
    counts compared on the device with the first form's.  Returns (section,
    counts of the first nhs halos per form)."""
    import numpy as np
    import torch

    from spatialjoincountovershells_b200 import _native as nat
    n, nf, nh = w["nparticles"], w["nfiles"], w["nhalos"]
    mn, mx, nr = w["radius"]
    r2 = nat.radius_table(mn, mx, nr)
    R = math.sqrt(float(r2[-1]))
    parts_d, halos_d = data.parts_d, data.halos_d
    # every form gets its own autotuned schedule (cached in the context per index kind)
    tunes = {}
    for kind in (nat.INDEX_GRID, nat.INDEX_MORTON, nat.INDEX_LEARNED):
        idx0 = ctx.build_index(parts_d[0], radius_hint=R, kind=kind)
        qt = ctx.query(halos_d, r2)
        tunes[kind] = ctx.autotune(qt, idx0)
        qt.destroy()
        idx0.destroy()

    forms = [("grid", nat.INDEX_GRID, nat.SCHED_AUTO), ("grid-static", nat.INDEX_GRID, nat.SCHED_STATIC),
             ("morton", nat.INDEX_MORTON, nat.SCHED_AUTO), ("morton-static", nat.INDEX_MORTON, nat.SCHED_STATIC),
             ("learned", nat.INDEX_LEARNED, nat.SCHED_AUTO), ("learned-static", nat.INDEX_LEARNED, nat.SCHED_STATIC)]
    res, first, info, sample = {}, None, None, {}
    for name, kind, mode in forms:
        def step(kind=kind, mode=mode):
            q = ctx.query(halos_d, r2)
            q.set_schedule(mode)
            for f in range(nf):
                idx = ctx.build_index(parts_d[f], radius_hint=R, kind=kind)
                q.count(idx)
                idx.destroy()
            return q
        ms, launches, count_ms, clocks = time_steps(ctx, step, K, W, dist, local)
        # one more pass for the build split and the counts
        q = ctx.query(halos_d, r2)
        q.set_schedule(mode)
        bts = []
        for f in range(nf):
            idx = ctx.build_index(parts_d[f], radius_hint=R, kind=kind)
            q.count(idx)
            idx.wait()
            bts.append(idx.timing()["build_ms"])
            if kind == nat.INDEX_LEARNED and f == 0:
                info = idx.learned_info()
            idx.destroy()
        q.wait()
        c = device_counts(q)
        sample[name] = c[:nhs * nr].cpu().numpy().view(np.uint32).reshape(nhs, nr)
        if first is None:
            first = c
            same = True
        else:
            same = bool(torch.equal(c, first))
        del c
        q.destroy()
        res[name] = {"value": round(nh * nf * world / (ms / 1e3), 1), "ms_per_step": round(ms, 3),
                     "build_s_per_file": round(statistics.mean(bts) / 1e3, 5),
                     "count_ms_per_file": round(count_ms, 3) if count_ms else None,
                     "counts_identical_to_grid": same, "gpu_launches": launches, "clocks": clocks,
                     "schedule": tunes[kind]["chosen"] if mode == nat.SCHED_AUTO else "static"}
    del first
    torch.cuda.empty_cache()
    sec = {
        "metric": METRIC, "value": res["learned"]["value"], "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": res["learned"]["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: project generators (clumped particles and halos, MT19937 block streams)",
        "config": {"workload": clustered_name(w), "index": "learned (63-bit Morton, 2-level PLM, 4096 leaves)",
                   "parallelism": "replicas" if world > 1 else "single",
                   "grid_schedule": tunes[nat.INDEX_GRID]["chosen"]},
        "plain_value": res["grid"]["value"],
        "learned_over_plain": round(res["learned"]["value"] / res["grid"]["value"], 3),
        "forms": res,
        "learned_info": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in (info or {}).items()},
        "gpu_launches": res["learned"]["gpu_launches"], "clocks": res["learned"]["clocks"],
    }
    return sec, sample


C3_SAMPLE, C4_SAMPLE = 2000, 100_000  # halos of the clustered workloads compared with the reference


def clustered_context(args, w, local, extra_per_particle):
    from spatialjoincountovershells_b200 import _native as nat
    n, nh = w["nparticles"], w["nhalos"]
    nr = w["radius"][2]
    ctx = nat.Context(local)
    ctx.set_overlap(args.overlap)
    if not args.no_reserve:
        ctx.reserve(4 * (n * 16 + int(1.6 * n + 4096) * 4) + n * extra_per_particle + 4 * nh * (16 + 4 * nr + 64)
                    + (2 << 30))
    return ctx


def run_clustered(args, w, dist, rank, world, local):
    """C3 on its own line (--workload clustered)."""
    import torch
    torch.cuda.set_device(local)
    data = ClusteredData(w, local)
    ctx = clustered_context(args, w, local, 44)
    sec, sample = section_c3(args, w, ctx, data, args.steps, args.warmup, dist, local, world, C3_SAMPLE)
    ctx.close()
    data.release_device()
    sec["cpu_baseline"] = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        refs = clustered_reference_legs(w, data, [("c3", w["radius"], C3_SAMPLE)])
        if "c3" in refs:
            sec["cpu_baseline"] = clustered_cpu_baseline(w, refs["c3"])
            sec["parity_at_scale"] = {"c3_sample": parity_record(refs["c3"]["counts"], sample, clustered_name(w),
                                                                 w["radius"])}
    return sec


def run_forms(args, w, dist, rank, world, local):
    """C4 on its own line (--workload learned)."""
    import torch
    torch.cuda.set_device(local)
    data = ClusteredData(w, local)
    ctx = clustered_context(args, w, local, 60)
    sec, sample = section_c4(args, w, ctx, data, args.steps, args.warmup, dist, local, world, C4_SAMPLE)
    ctx.close()
    data.release_device()
    sec["cpu_baseline"] = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        refs = clustered_reference_legs(w, data, [("c4", w["radius"], C4_SAMPLE)])
        if "c4" in refs:
            sec["cpu_baseline"] = clustered_cpu_baseline(w, refs["c4"])
            sec["parity_at_scale"] = {"c4_sample": parity_record(refs["c4"]["counts"], sample, clustered_name(w),
                                                                 w["radius"])}
    return sec


def run_extras(args, dist, rank, world, local, K, W, small):
    """Configs 3-5 for the headline line: C3 and C4 on one clustered data set
    (reference parity samples for both), then C5 over resident indexes of the
    same particles.  K timed and W warm-up steps per leg."""
    import torch
    c3, c4 = dict(CLUSTERED), dict(FORMS)
    sv = dict(SERVING, nrequests=SERVING_IN_HEADLINE)
    if small:
        for d in (c3, c4, sv):
            d["nparticles"] //= 50
            if "nhalos" in d:
                d["nhalos"] //= 50
        sv["nrequests"] //= 10
        sv["size"] = (sv["size"][0], sv["size"][1] / 50)
    data = ClusteredData(c3, local)
    out = {}
    ctx = clustered_context(args, c3, local, 60)
    out["clustered_c3"], s3 = section_c3(args, c3, ctx, data, K, W, dist, local, world, min(C3_SAMPLE, c3["nhalos"]))
    out["forms_clustered_c4"], s4 = section_c4(args, c4, ctx, data, K, W, dist, local, world,
                                               min(C4_SAMPLE, c4["nhalos"]))
    ctx.close()
    torch.cuda.empty_cache()
    parity = {}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        refs = clustered_reference_legs(c3, data, [("c3", c3["radius"], min(C3_SAMPLE, c3["nhalos"])),
                                                   ("c4", c4["radius"], min(C4_SAMPLE, c4["nhalos"]))])
        if refs:
            out["clustered_c3"]["cpu_baseline"] = clustered_cpu_baseline(c3, refs["c3"])
            out["forms_clustered_c4"]["cpu_baseline"] = clustered_cpu_baseline(c4, refs["c4"])
            parity["c3_sample"] = parity_record(refs["c3"]["counts"], s3, clustered_name(c3), c3["radius"])
            parity["c4_sample"] = parity_record(refs["c4"]["counts"], s4, clustered_name(c4), c4["radius"])
    out["serving_c5"] = run_serving(args, sv, dist, rank, world, local, data=data)
    data.release_device()
    del data
    return out, parity


def run_io(args, w, dist, rank, world, local):
    """The host phases around the GPU path, as the driver runs them: halo text
    ingest (readHalos), particle file read (readDecodedParticles) and result
    text output (outputResult), from the phase lines sjcs_rcount prints like
    astr_rcount does, on the same files.  The reference program's own phase
    lines on this host's cores are the cpu_baseline."""
    import subprocess

    from spatialjoincountovershells_b200 import _native as nat
    driver = ROOT / "spatialjoincountovershells_b200" / "bin" / "sjcs_rcount"
    if not driver.exists():
        raise RuntimeError(f"{driver} is missing; run python -m spatialjoincountovershells_b200.build")
    if rank != 0:
        return None
    T = ref_threads()
    mn, mx, nr = w["radius"]
    phases = ["halo data reading", "particles reading", "result writing"]

    def run(cmd, cwd):
        t0 = time.time()
        r = subprocess.run([str(c) for c in cmd], cwd=cwd, capture_output=True, text=True, timeout=3600)
        wall = time.time() - t0
        if r.returncode != 0:
            raise RuntimeError(f"{cmd[0]} failed: {r.stderr[-500:]}")
        t = {}
        for m in re.finditer(r">>>> (.+?) time: (\d+) milli seconds", r.stdout):
            t[m.group(1)] = t.get(m.group(1), 0) + int(m.group(2))
        return t, wall

    with tempfile.TemporaryDirectory(prefix="sjcs_io_") as td:
        d = pathlib.Path(td)
        pf, hf = d / "part0.dat", d / "halos.list"
        nat.write_particle_file(pf, nat.gen_uniform_particles(w["pseed"], 1, w["nparticles"]))
        nat.gen_uniform_halo_file(hf, w["hseed"], w["nhalos"])
        cli = ["--thread", T, "--next-setup", T, "--particle-files", pf.name, "--halo-file", hf.name,
               "--radius", f"{mn}:{mx}:{nr}"]
        ours, ours_wall = run([driver, *cli, "--output-file", "ours.txt"], d)
        out_bytes = (d / "ours.txt").stat().st_size
        (d / "ours.txt").unlink()
        cpu = None
        if not args.no_cpu_baseline:
            from oracle import oracle
            if oracle.ref_available():
                ref, ref_wall = run([oracle.REF_ASTR, *cli, "--output-file", "ref.txt"], d)
                cpu = {"value": sum(ref.get(k, 0) for k in phases), "unit": "ms", "cores": T, "kind": "reference",
                       "sample": "the whole workload", "phases_ms": {k: ref.get(k) for k in phases},
                       "wall_s": round(ref_wall, 2)}
    total = sum(ours.get(k, 0) for k in phases)
    return {
        "metric": "host phases of one driver run: halo text read + particle file read + result text write",
        "value": total, "unit": "ms", "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": total,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32 / text",
        "data": "synthetic: reference generator streams",
        "config": {"workload": f"io: {w['nfiles']} file x {w['nparticles']:.0e} uniform particles "
                               f"(seed {w['pseed']}), {w['nhalos']:.0e} halos (seed {w['hseed']}), "
                               f"--radius {mn}:{mx}:{nr}, --thread {T}", "parallelism": "host threads"},
        "phases_ms": {k: ours.get(k) for k in phases}, "all_phases_ms": ours, "wall_s": round(ours_wall, 2),
        "result_text_bytes": out_bytes, "cpu_baseline": cpu,
    }


SERVING_IN_HEADLINE = 400  # requests of the serving leg inside the headline line (a prefix of the stream)


def run_serving(args, w, dist, rank, world, local, data=None):
    """C5: request loop over resident clustered indexes, Poisson arrivals, p50/p99.
    data: resident clustered particles to index (else generated here)."""
    import numpy as np
    import torch

    from spatialjoincountovershells_b200 import _native as nat
    torch.cuda.set_device(local)
    n, nf = w["nparticles"], w["nfiles"]
    rng = np.random.default_rng(w["arrival_seed"])
    nreq = w["nrequests"]
    lo, hi = w["size"]
    sizes = np.round(np.exp(rng.uniform(math.log(lo), math.log(hi), nreq))).astype(np.int64)
    nrads = rng.integers(w["nrads"][0], w["nrads"][1] + 1, nreq)
    rmax = rng.uniform(w["rmax"][0], w["rmax"][1], nreq)
    tables = [nat.radius_table(0.001, float(rm), int(k)) for rm, k in zip(rmax, nrads)]
    halos = [np.ascontiguousarray(nat.gen_clustered_halos(w["hseed"] * 1000 + i, int(m))["point"])
             for i, m in enumerate(sizes)]
    ctx = nat.Context(local)
    idx = []
    for f in range(nf):
        if data is not None:
            p = data.parts_d[f]
        else:
            p = torch.from_numpy(nat.gen_clustered_particles(w["pseed"] + f, n)).cuda()
        idx.append(ctx.build_index(p, radius_hint=w["rmax"][1]))
        idx[-1].wait()
        del p
    if data is not None:
        data.release_device()
    torch.cuda.empty_cache()
    ctx.trim()

    import hashlib
    import queue as pyqueue
    import threading as th
    # pinned result buffers, recycled: the counts go straight from the device
    maxcnt = int(max(int(sizes[i]) * int(nrads[i]) for i in range(nreq)))
    pool = pyqueue.Queue()
    pinned = [nat.PinnedBuffer((maxcnt,), np.uint32) for _ in range(24)]
    for b in pinned:
        pool.put(b)

    def digest(a):
        return hashlib.blake2b(a.tobytes(), digest_size=16).hexdigest()

    def run_stream(order, rate, slots):
        """Submit `order` at Poisson times (rate per second); wait in order; latencies."""
        srv = nat.Server(ctx, idx, slots=slots)
        arr = np.cumsum(np.random.default_rng(w["arrival_seed"] + 1).exponential(1.0 / rate, len(order)))
        tickets, lat, done_q = [], [], []
        lock = th.Lock()

        def waiter():
            k = 0
            while k < len(order):
                with lock:
                    t = tickets[k] if k < len(tickets) else None
                if t is None:
                    time.sleep(0.0002)
                    continue
                tk, buf, m = t
                out, info = srv.wait(tk)
                lat.append(info["latency_ms"])
                done_q.append((order[k], digest(out), info["queue_ms"]))
                pool.put(buf)
                k += 1
        wt = th.Thread(target=waiter)
        wt.start()
        t0 = time.perf_counter()
        for k, i in enumerate(order):
            d = t0 + arr[k] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            buf = pool.get()
            m = int(sizes[i]) * int(nrads[i])
            out = buf.array[:m].reshape(int(sizes[i]), int(nrads[i]))
            t = srv.submit(halos[i], tables[i], out=out)
            with lock:
                tickets.append((t, buf, m))
        wt.join()
        makespan = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        return lat, makespan, st, done_q

    halo_files = int(sizes.sum()) * nf
    # capacity: the first 200 requests submitted at once
    cal = list(range(min(200, nreq)))
    lat_c, span_c, _, _ = run_stream(cal, 1e9, 8)
    cap = sum(int(sizes[i]) for i in cal) / span_c  # halos per second
    rate = 0.7 * cap / float(sizes.mean())
    lat, makespan, st, done = run_stream(list(range(nreq)), rate, 8)
    lat_sorted = sorted(lat)
    p50 = lat_sorted[len(lat) // 2]
    p99 = lat_sorted[min(len(lat) - 1, int(math.ceil(0.99 * len(lat))) - 1)]
    # exactness: a sample of requests again, alone (one slot, one at a time)
    sums = {i: s for i, s, _ in done}
    alone_ok = True
    with nat.Server(ctx, idx, slots=1) as srv1:
        for i in list(range(0, nreq, max(1, nreq // 20))):
            out, _ = srv1.wait(srv1.submit(halos[i], tables[i]))
            alone_ok &= digest(out) == sums[i]
    for b in pinned:
        b.free()
    for x in idx:
        x.destroy()
    ctx.close()
    return {
        "metric": "serving: p50/p99 request latency and halos/s (Poisson arrivals, memory admission)",
        "value": round(halo_files / makespan, 1), "unit": "halo-files/s", "n_gpus": world, "steps": 1,
        "warmup": 1, "ms_per_step": round(makespan * 1e3, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic: project generators",
        "config": {"workload": f"serving: {nreq} requests, sizes log-uniform [{lo:.0e},{hi:.0e}] clustered halos, "
                               f"radius 0.001:U[{w['rmax'][0]},{w['rmax'][1]}]:U{{{w['nrads'][0]}..{w['nrads'][1]}}}, "
                               f"Poisson arrivals at 70% of measured capacity (seed {w['arrival_seed']}), "
                               f"{nf} resident indexes x {n:.0e} clustered particles", "slots": 8},
        "latency_ms": {"p50": round(p50, 2), "p99": round(p99, 2), "mean": round(statistics.mean(lat), 2),
                       "max": round(lat_sorted[-1], 2)},
        "arrival_rate_per_s": round(rate, 2), "capacity_halos_per_s": round(cap, 1),
        "server": st, "results_same_alone_and_in_mix": bool(alone_ok),
        "mean_queue_ms": round(statistics.mean(q for _, _, q in done), 2),
    }


def reference_leg(w, particles, halos_sample, r2):
    """cpu_baseline and parity check: astr_rcount (compiled from the reference's
    sources) over every particle file of the workload and a halo sample, on
    this host's cores.  Returns (cpu_baseline, counts of the sampled halos)."""
    from oracle import oracle
    nhs = len(halos_sample)
    if not oracle.ref_available():
        v = port_baseline(w, particles[:w["nparticles"]], halos_sample[:1000], r2)
        return ({"value": round(v, 1), "unit": UNIT, "cores": 1, "kind": "port",
                 "sample": "oracle port, 1 thread, 1 file x 1000 halos, extrapolated"}, None)
    T = ref_threads()
    with tempfile.TemporaryDirectory(prefix="sjcs_ref_") as td:
        files, hf = write_reference_inputs(pathlib.Path(td), particles, w["nfiles"], halos_sample)
        r = run_reference(files, hf, w["radius"], T, result=True)
    b, s = r["build_s"], r["search_s"]
    cpu = {"value": round(reference_extrapolate(w, b, s, nhs), 1), "unit": UNIT, "cores": T, "kind": "reference",
           "sample": f"astr_rcount --thread {T} --next-setup {T} on all {w['nfiles']} files of "
                     f"{w['nparticles']:.0e} particles x the first {nhs} halos: build {b:.3f} s and search "
                     f"{s:.3f} s per file (wall {r['wall_s']:.1f} s); extrapolated to {w['nhalos']:.0e} halos"}
    return cpu, r["counts"]


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------

def run_reference_arm(args, w):
    """The reference program alone, as stock as it ships: its own generators
    write the inputs (MT19937 seeds as our arm's), astr_rcount counts them.
    No library of this package is loaded in this process.  One step is a
    bounded sample of the workload: one whole particle file (built, as
    every file is) and the first nhs halos searched against it; files rotate
    over the workload's files.  ms_per_step is that measured sample; value
    is the whole workload's halo-file passes per second extrapolated from
    the mean sample (build time per file, search time scaled by the halo
    count), under "extrapolation"."""
    from oracle import oracle
    if not oracle.ref_available():
        return {"impl": "reference", "metric": METRIC, "unit": UNIT,
                "unavailable": "reference program not built (oracle/_ref/astr_rcount.exe missing)"}
    nhs = 100_000 if w["nhalos"] >= 1_000_000 else max(1000, w["nhalos"] // 10)
    nf, n = w["nfiles"], w["nparticles"]
    T = ref_threads()

    def gen(exe, paths, count, seed):
        r = subprocess.run([str(exe), "-f", *[str(x) for x in paths], "-n", str(count), "-s", str(seed)],
                           capture_output=True, text=True, timeout=1800)
        if r.returncode != 0:
            raise RuntimeError(f"{exe.name} failed: {r.stderr[-300:]}")

    with tempfile.TemporaryDirectory(prefix="sjcs_refarm_") as td:
        tmp = pathlib.Path(td)
        t0 = time.perf_counter()
        files = [tmp / f"part{f}.dat" for f in range(nf)]
        gen(oracle.REF_PGEN, files, n, w["pseed"])   # one stream over the files, as main.c:42-68
        hf = tmp / "halos.list"
        gen(oracle.REF_HGEN, [hf], nhs, w["hseed"])  # the halo stream's first nhs halos
        gen_s = time.perf_counter() - t0
        # warm-up runs on a small file (untimed): page in the binary and the inputs' cache
        warm = tmp / "warm"
        warm.mkdir()
        wpf, whf = warm / "part.dat", warm / "halos.list"
        gen(oracle.REF_PGEN, [wpf], 1_000_000, w["pseed"])
        gen(oracle.REF_HGEN, [whf], 10_000, w["hseed"])
        for _ in range(args.warmup):
            run_reference([wpf], whf, w["radius"], T, result=False)
        runs = []
        for k in range(args.steps):
            runs.append(run_reference([files[k % nf]], hf, w["radius"], T, result=False))
    b = statistics.mean(r["build_s"] for r in runs)
    s = statistics.mean(r["search_s"] for r in runs)
    step_ms = 1e3 * (b + s)
    v = reference_extrapolate(w, b, s, nhs)
    full_ms = 1e3 * w["nhalos"] * nf / v
    sample = (f"astr_rcount --thread {T} --next-setup {T}: per step 1 file of {n:.0e} particles (build {b:.3f} s) "
              f"and the first {nhs} halos (search {s:.3f} s); files rotate over the {nf} files")
    return {
        "impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": UNIT, "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_ms, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": round(v / PUBLISHED_HALO_FILES_PER_S, 3), "dtype": "f32",
        "data": "synthetic: the reference's own generators (uniform_decoded_particle_generator -s "
                f"{w['pseed']}, uniform_halo_generator -s {w['hseed']})",
        "config": {"workload": workload_name(w), "index": "reference STR tree (CPU)", "parallelism": "cpu threads",
                   "step": f"1 particle file x {nhs} halos (bounded sample of the workload)"},
        "build_s_per_file": round(b, 3),
        "wall_ms_per_step": round(1e3 * statistics.mean(r["wall_s"] for r in runs), 1),
        "extrapolation": {"full_step_ms": round(full_ms, 1),
                          "method": f"{nf} x (build per file + search per file x {w['nhalos']} / {nhs})",
                          "value": round(v, 1)},
        "input_generation_s": round(gen_s, 1),
        "cpu_baseline": {"value": round(v, 1), "unit": UNIT, "cores": T, "kind": "reference", "sample": sample},
        "e2e": {"value": round(v, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--small", action="store_true", help="a 50x smaller workload (smoke runs, CPU tests)")
    ap.add_argument("--files", type=int, default=None, help="override the number of particle files")
    ap.add_argument("--halos", type=int, default=None, help="override the number of halos (same density)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--halo-slab", type=float, default=None,
                    help="keep only halos with z < SLAB (profiling at full halo density on fewer halos)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-check", action="store_true",
                    help="accepted and ignored (parity is checked by the test suite, not by the benchmark)")
    ap.add_argument("--no-forms", action="store_true", help="skip the learned/Morton comparison legs")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline line only: skip the clustered (C3), index-form (C4) and serving (C5) sections")
    ap.add_argument("--extra-steps", type=int, default=3,
                    help="timed steps per leg of the C3/C4 sections of the headline line (at most --steps)")
    ap.add_argument("--overlap", action="store_true",
                    help="let index builds' kernels run beside the counts (default: after them; copies overlap)")
    ap.add_argument("--particles", type=int, default=None, help="override particles per file (profiling cases)")
    ap.add_argument("--no-reserve", action="store_true",
                    help="do not grow the device memory pool up front (profiling cases: keep the footprint small)")
    ap.add_argument("--workload", choices=["uniform", "clustered", "learned", "serving", "io"], default="uniform",
                    help="uniform: the headline line (README scale); clustered: persistent schedule and captured "
                         "steps; learned: index forms on clustered data; serving: the request loop; "
                         "io: the driver's host phases (halo text read, particle read, result write)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    w = dict(SMALL if args.small else FULL)
    if args.files:
        w["nfiles"] = args.files
    if args.halos:
        w["nhalos"] = args.halos
    if args.particles:
        w["nparticles"] = args.particles
    if args.impl == "reference":
        # the reference is a CPU program: rank 0 alone runs it, other ranks exit
        if int(os.environ.get("RANK", "0")) != 0:
            return
        print(json.dumps(run_reference_arm(args, w)), flush=True)
        return
    dist, rank, world, local = dist_setup()
    if args.workload != "uniform":
        base = {"clustered": CLUSTERED, "learned": FORMS, "serving": SERVING, "io": IO}[args.workload]
        w = dict(base)
        if args.small:
            w["nparticles"] //= 50
            if "nhalos" in w:
                w["nhalos"] //= 50
            if "nrequests" in w:
                w["nrequests"] //= 10
                w["size"] = (w["size"][0], w["size"][1] / 50)
        if args.files:
            w["nfiles"] = args.files
        if args.halos and "nhalos" in w:
            w["nhalos"] = args.halos
        if args.particles:
            w["nparticles"] = args.particles
        run = {"clustered": run_clustered, "learned": run_forms, "serving": run_serving,
               "io": run_io}[args.workload]
        line = run(args, w, dist, rank, world, local)
        dist_close(dist)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
        return
    line = run_ours(args, w, dist, rank, world, local)
    # configs 3-5 ride on the headline line at one GPU (replica runs time the headline only)
    if not args.no_extras and world == 1:
        extras, parity = run_extras(args, dist, rank, world, local, K=max(1, min(args.steps, args.extra_steps)),
                                    W=3, small=args.small)
        line.update(extras)
        if parity:
            line["parity_at_scale"] = {**(line.get("parity_at_scale") or {}), **parity}
    dist_close(dist)
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
