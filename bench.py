"""Benchmark of the CSS RK4 hot path on B200: RK4 cell-updates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME]

Default workload: the 256x512x1024 MHD shell (nv = 8: rho, u_theta, u_phi,
u_r, s and the vector potential A; 5 density scale heights, magnetic Prandtl
number 2 through the SLD scaling, FP64, virtual decomposition 8x16x32 =
32^3 blocks), synthetic seeded state with the random, tapered vector
potential of Initialize_Mag.  --workload hydro-128x256x512 runs the hydro
polytrope (3 scale heights, 4x8x16 blocks).  One step = one full RK4 step
(4 RHS evaluations + slope-limited diffusion).  `value` is device-timed
with CUDA events on the stream the library runs on, inputs resident in HBM
(the state, 8.6 GB per buffer for MHD, is larger than L2).  `e2e` is the
same metric through the C ABI with host buffers: each step uploads the
state from pinned host memory, advances it one step and reads it back
(css_step_rk4_host), as a Fortran driver that keeps vars0 on the host would
call it.  N > 1: one process per GPU, each advancing its own replica (the
hot path runs the whole domain on one GPU; no collective), time = max over
ranks.

--impl reference times the reference's CPU implementation of the same path:
the FP64 C restatement in oracle/ (the Fortran itself cannot be built here),
with every host thread, on a bounded sample of the workload (for the MHD
shell: RK4 steps of a 128x256x512 MHD shell with the same physics and the
same 32^3 virtual blocks; cell-updates/s is per cell, and a full step of
the 1.3e8-cell shell would take over a minute of host time).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "css-code_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "RK4 cell-updates/s at stated error vs FP64 oracle; % of HBM roofline"
UNIT = "cell-updates/s"
FALLBACK_HBM_GBS = 6650.0
REF_BUDGET_S = 60  # CPU seconds of the reference arm's timed sample

# compulsory bytes per cell of each kernel (FP64 words read + written once;
# halo re-reads and the LU tables are not counted), hydro nv = 5 / MHD nv = 8
def kernel_alg_bytes(name, nv, stage_mix=None):
    mag = nv == 8
    nb = 3 if mag else 0
    w = {
        "theta_terms": 5 + nb + (8 if mag else 5),
        "phi_terms": 5 + nb + 2 * 5,
        "radial_terms": 5 + nb + 2 * 5,
        "rhot_update": 0,
        "curl_theta": 2 + 2,
        "curl_phi": 2 + 3 + 1,
        "curl_r": 2 + 3 + 3,
        "sld_vcc": 3 + (4 if mag else 0) + 1,
        # MHD runs the SLD as two launches (hydro fields, then A), timed as
        # one, each reading the speed^2: nv + 2 + nv words over the pair
        "sld": nv + (2 if mag else 1) + nv,
        "sld_ohmic": 2 + 3 + 3 + 2,
    }.get(name)
    if name == "thph":
        # the state's five fields [+ B], the tendency of every field and T
        w = 5 + nb + nv + 1
    if name == "rstage":
        # the slab's five fields [+ B_theta, B_phi, B_r], the tendency, T,
        # vars0 and the accumulator read; the next state written, and the
        # accumulator in stages 1-3 (average over the four stages)
        w = 5 + nb + nv + 1 + 2 * nv + (3 * nv) / 4.0 + nv
    if name == "rhot_update":
        # average over the four stages: reads rho,w,s + dv,v0,vs (3 nv), writes
        # vs + next (2 nv) in stages 1-3 and next only (nv) in stage 4
        w = 3 + 3 * nv + (3 * 2 * nv + nv) / 4.0
    return None if w is None else 8.0 * w


# The bounded CPU sample of a workload: (dims, build options, description).
# None: the workload itself (a step takes seconds on the host cores).
CPU_SAMPLES = {
    "mhd-256x512x1024": ((128, 256, 512), dict(magnetic=True, decomp=(4, 8, 16), n_rho=5.0),
                         "a 128x256x512 MHD shell with the workload's physics (n_rho 5, Pm 2) and 32^3 virtual "
                         "blocks (decomposition 4x8x16)"),
}


def cpu_sample(workload):
    """(params, profiles, vars0, dt, description) of the CPU sample."""
    from css_b200 import problem
    spec = CPU_SAMPLES.get(workload)
    if spec is None:
        p, prof, v0, dt, _ = problem.build(workload)
        return p, prof, v0, dt, "the full %dx%dx%d workload" % (p.nr, p.nth, p.nphi)
    dims, kw, desc = spec
    p, prof, v0, dt, _ = problem.build(dims, **kw)
    return p, prof, v0, dt, desc


def step_alg_bytes(nv):
    """Compulsory traffic of a perfectly fused RK4 step: 17 nv words/cell."""
    return 17 * nv * 8


def read_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), smax=float(parts[2]), hw=parts[5], hwt=parts[6], swt=parts[7],
                                 pcap=parts[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        reasons = set()
        for r in rows:
            for key, nm in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"), ("swt", "sw_thermal_slowdown"),
                            ("pcap", "sw_power_cap")):
                if r[key].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(r["sm"] for r in rows), "sm_max_mhz": max(r["smax"] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_setup(n):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(workload, steps):
    """The oracle (FP64 C restatement, every host thread) on the workload's
    bounded CPU sample: one warm-up step, then `steps` timed steps."""
    p, prof, v0, dt, desc = cpu_sample(workload)
    return cpu_baseline_on(p, prof, v0, dt, steps, desc)


def cpu_baseline_on(p, prof, v0, dt, steps, desc):
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    orc = O.Oracle(p, prof)
    orc.step(v0, dt, 1)  # warm-up
    t = time.perf_counter()
    orc.step(v0, dt, steps)
    el = time.perf_counter() - t
    orc.close()
    cells = p.nr * p.nth * p.nphi
    return {"value": cells * steps / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "%d RK4 steps of %s (FP64 C restatement, %d OpenMP threads)" % (steps, desc, threads),
            "seconds": el}


def run_reference(args):
    from css_b200 import problem
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    if args.workload.startswith("ensemble-"):
        return run_reference_ensemble(args, world)
    if args.workload.startswith("closure"):
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned closure: its SLD "
                          "speed is a prescribed radial profile (diffusion.f90:19-63)"}))
        return 0
    p, prof, v0, dt, desc = cpu_sample(args.workload)
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    orc = O.Oracle(p, prof)
    v = v0
    # warm-up: at least one step, which also sizes the sample; the timed
    # sample is bounded to about REF_BUDGET_S of CPU time (a step of the full
    # workload takes seconds on the host cores)
    tw = time.perf_counter()
    for _ in range(max(1, args.warmup)):
        v = orc.step(v, dt, 1)
    per_step = (time.perf_counter() - tw) / max(1, args.warmup)
    timed = max(1, min(args.steps, int(REF_BUDGET_S / max(per_step, 1e-9))))
    t = time.perf_counter()
    for _ in range(timed):
        v = orc.step(v, dt, 1)
    el = time.perf_counter() - t
    cells = p.nr * p.nth * p.nphi
    val = cells * timed / el
    out = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world, "steps": timed,
        "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / timed, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "sample_grid": [p.nr, p.nth, p.nphi],
                   "sample_decomposition": [p.nnr, p.nnt, p.nnp], "fields": 8 if p.magnetic else 5,
                   "l2": "state larger than L2"},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": "%d RK4 steps of %s (bounded to ~%d s of CPU time), FP64 C "
                                   "restatement of the reference (Fortran not buildable here), %d OpenMP threads"
                                   % (timed, desc, REF_BUDGET_S, threads)},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


def run_reference_ensemble(args, world):
    """The oracle over the members of the shell study, one RK4 step each, in
    member order until about REF_BUDGET_S of CPU time has been spent."""
    from css_b200 import ensemble as E
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    count = int(args.workload.split("-")[1])
    specs = E.shell_specs(count, seed=7)
    done_cells, el, k = 0, 0.0, 0
    while k < len(specs) and el < REF_BUDGET_S:
        p, prof, v0, dt = E.build_member(specs[k], seed=1000 + k)
        orc = O.Oracle(p, prof)
        if k == 0:
            orc.step(v0, dt, 1)  # warm-up
        t = time.perf_counter()
        orc.step(v0, dt, 1)
        el += time.perf_counter() - t
        done_cells += E.cells(specs[k])
        orc.close()
        k += 1
    val = done_cells / el
    out = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world, "steps": 1,
           "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el, "higher_is_better": True,
           "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": args.workload, "members_sampled": k, "cells_sampled": done_cells},
           "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": "one RK4 step of each of the first %d members (bounded to ~%d s), FP64 C "
                                      "restatement, %d OpenMP threads" % (k, REF_BUDGET_S, threads)},
           "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def run_ours(args):
    import numpy as np
    import torch
    from css_b200 import problem
    from css_b200.context import Simulation

    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    p, prof, v0, dt, _ = problem.build(args.workload)
    nv = 8 if p.magnetic else 5
    cells = p.nr * p.nth * p.nphi
    if args.precision == "mixed":
        p.precision = 1
    sim = Simulation(p, prof)
    if args.stage == "four":
        sim.set_fused(False)
    stream = torch.cuda.current_stream(dev)
    sim.set_stream(stream.cuda_stream)
    sim.upload(v0)
    # lines per CTA of the four-kernel stage's sweeps (no result changes);
    # the two-pass stage has fixed tiles
    tiles = (0, 0, 0) if sim.fused else sim.autotune(reps=3)
    for _ in range(args.warmup):
        sim.step_rk4(dt, 1)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    if rank == 0:
        clocks.start()
        time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize()
    l0 = sim.launches()
    sim.profile(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        sim.step_rk4(dt, 1)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    launches = sim.launches() - l0
    ms = e0.elapsed_time(e1)
    stats = sim.kernel_stats()
    sim.profile(False)
    clk = clocks.stop() if rank == 0 else None
    ms_max = max_over_ranks(ms, world)
    value = cells * args.steps * world / (ms_max / 1e3)

    # e2e through the C ABI with host buffers (pinned)
    e2e_steps = 0 if args.no_e2e else max(1, min(args.steps, 10))
    host = torch.from_numpy(np.ascontiguousarray(v0)).pin_memory()
    if e2e_steps:
        sim.step_host(host.numpy(), dt, 1)  # warm
    barrier(world)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    import ctypes
    from css_b200 import _lib
    ptr = ctypes.cast(host.data_ptr(), _lib.dp)
    for _ in range(e2e_steps):
        _lib.check(_lib.lib().css_step_rk4_host(sim.h, ptr, float(dt), 1))
    t1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(t0.elapsed_time(t1), world)
    e2e_val = cells * e2e_steps * world / (e2e_ms / 1e3) if e2e_steps else None
    state_bytes = cells * nv * 8

    # roofline of the dominant kernel (largest share of device time)
    peak, peak_src = read_peaks()
    dom = max(stats.items(), key=lambda kv: kv[1][0]) if stats else None
    roof = None
    if dom:
        name, (kms, cnt) = dom
        alg = kernel_alg_bytes(name, nv)
        per_launch_cells = cells
        achieved = alg * per_launch_cells / (kms / cnt / 1e3) / 1e9 if alg else None
        traffic = None
        fp64 = None
        traffic_src = None
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            try:
                tj = json.load(open(tpath))
                key = "%s/%s" % ("mhd" if p.magnetic else "hydro", name)
                if key in tj:
                    traffic = tj[key]["dram_bytes_per_cell"] * per_launch_cells
                    fp64 = tj[key].get("fp64_pipe_pct_of_peak")
                    note = tj[key].get("note") or ""
                    traffic_src = "ncu capture on %s%s" % (tj[key].get("captured_on", "?"),
                                                           "; " + note if note else "")
            except Exception:
                traffic = None
        roof = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "traffic_source": traffic_src,
                "algorithmic_bytes_per_launch": alg * per_launch_cells if alg else None,
                "avg_launch_ms": kms / cnt, "peak_source": peak_src,
                "time_share": kms / sum(v[0] for v in stats.values()),
                # the FP64 bound beside the HBM one: ncu's FP64-pipe activity
                # of this kernel (profiles/traffic.json, captured on the
                # 128x128x256 case of the same kind of run)
                "fp64_pipe_frac": (fp64 / 100.0) if fp64 is not None else None}
    step_ach = step_alg_bytes(nv) * cells * args.steps / (ms / 1e3) / 1e9
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32-storage/f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": [p.nr, p.nth, p.nphi], "decomposition": [p.nnr, p.nnt, p.nnp],
                   "precision": args.precision, "tile_lines_r_theta_phi": list(tiles),
                   "stage": "two-pass (k_thph + k_rstage)" if sim.fused else "four-kernel",
                   "fields": nv, "dt": dt, "l2": "state (%.0f MB per buffer) larger than L2, no flush" % (state_bytes / 1e6),
                   "parallelism": "replicas" if world > 1 else "single-gpu"},
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
                "steps": e2e_steps, "api": "css_step_rk4_host, one step per call, pinned host state"},
        "gpu_launches": launches,
        "roofline": roof,
        "step_roofline": {"algorithmic_bytes_per_cell_step": step_alg_bytes(nv), "achieved": step_ach,
                          "peak": peak, "unit": "GB/s", "frac": step_ach / peak, "peak_source": peak_src},
        "kernels_ms": {k: {"total_ms": v[0], "launches": v[1]} for k, v in sorted(stats.items())},
        "error_vs_oracle": ("FP64: derivatives/RHS <= 1e-12, state after 100 steps <= 1e-10 (tests/test_gpu_parity.py)"
                            if args.precision == "fp64" else
                            "mixed: every field <= 1e-6 of its size after 100 steps of a developed flow (observed "
                            "<= 2.6e-7), rho and s <= 1e-6 and velocities <= 1e-5 from rest (tests/test_mixed.py)"),
    }
    if clk:
        out["clocks"] = clk
    sim.close()
    if rank == 0 and world == 1 and not args.no_cpu:
        del host
        out["cpu_baseline"] = cpu_baseline(args.workload, args.cpu_steps)
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def run_ensemble(args):
    """A study of many small shells (ensemble-<count>): members from the
    seeded shell study, split over ranks by LPT, each rank stepping its
    members through one captured CUDA graph.  Total work is fixed as ranks
    are added (strong scaling)."""
    import numpy as np
    import torch
    from css_b200 import ensemble as E
    from css_b200.context import Simulation

    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    count = int(args.workload.split("-")[1])
    specs = E.shell_specs(count, seed=7)
    mine = E.lpt_partition([E.member_cost(s) for s in specs], world)[rank]
    prec = 1 if args.precision == "mixed" else 0
    members = [E.build_member(specs[i], seed=1000 + i, precision=prec) for i in mine]
    sims = []
    for p, prof, v0, dt in members:
        sim = Simulation(p, prof)
        sim.upload(v0)
        sim.autotune(reps=2)
        sims.append(sim)
    ens = E.Ensemble(sims)
    dts = [m[3] for m in members]
    ens.step(dts, args.warmup)  # the first call captures the graph
    clocks = ClockSampler(local)
    if rank == 0:
        clocks.start()
        time.sleep(0.3)
    barrier(world)
    l0 = ens.launches()
    ens.step(dts, args.steps)
    ms = ens.last_ms()
    barrier(world)
    clk = clocks.stop() if rank == 0 else None
    launches = ens.launches() - l0
    ms_max = max_over_ranks(ms, world)
    total_cells = sum(E.cells(s) for s in specs)
    value = total_cells * args.steps / (ms_max / 1e3)
    mine_bytes = sum(E.cells(specs[i]) * 17 * (8 if specs[i]["magnetic"] else 5) * 8 for i in mine)
    step_ach = mine_bytes * args.steps / (ms / 1e3) / 1e9
    peak, peak_src = read_peaks()

    # e2e: every step uploads every member's state from pinned host memory,
    # steps the ensemble once and downloads every state
    e2e_steps = 0 if args.no_e2e else max(1, min(args.steps, 3))
    hosts = [torch.from_numpy(np.ascontiguousarray(m[2])).pin_memory() for m in members]
    stream = torch.cuda.current_stream(dev)
    barrier(world)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    import ctypes
    from css_b200 import _lib
    for _ in range(e2e_steps):
        for sim, h in zip(sims, hosts):
            _lib.check(_lib.lib().css_upload_state(sim.h, ctypes.cast(h.data_ptr(), _lib.dp)))
        ens.step(dts, 1)
        for sim, h in zip(sims, hosts):
            _lib.check(_lib.lib().css_download_state(sim.h, ctypes.cast(h.data_ptr(), _lib.dp)))
    t1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(t0.elapsed_time(t1), world) if e2e_steps else None
    state_bytes = sum(E.cells(s) * (8 if s["magnetic"] else 5) * 8 for s in specs)
    summ = E.summary(specs)
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64" if not prec else "f32-storage/f64", "data": "synthetic",
        "config": {"workload": args.workload, "members": summ["members"], "mhd_members": summ["mhd"],
                   "precision": args.precision, "ro_range": list(E.RO_RANGE), "pm_range": list(E.PM_RANGE),
                   "cells": total_cells, "members_on_rank0": len(mine),
                   "l2": "states (%.1f GB) larger than L2, no flush" % (state_bytes / 1e9),
                   "parallelism": "lpt over %d ranks, one CUDA graph per rank" % world},
        "e2e": {"value": total_cells * e2e_steps / (e2e_ms / 1e3) if e2e_steps else None, "unit": UNIT,
                "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes, "steps": e2e_steps,
                "api": "css_upload_state + css_ensemble_step + css_download_state per member, pinned host state"},
        "gpu_launches": launches,
        "step_roofline": {"algorithmic_bytes_per_cell_step": "17 nv words", "achieved": step_ach, "peak": peak,
                          "unit": "GB/s", "frac": step_ach / peak, "peak_source": peak_src},
        "error_vs_oracle": ("bit-identical to the members stepped alone, 200 steps (tests/test_ensemble.py)"
                            if not prec else
                            "every member within the mixed form's bounds of its own unbatched FP64 run after "
                            "200 steps (tests/test_ensemble.py)"),
    }
    if clk:
        out["clocks"] = clk
    if rank == 0 and world == 1 and not args.no_cpu:
        p, prof, v0, dt = members[0]
        out["cpu_baseline"] = cpu_baseline_on(p, prof, v0, dt, 1, "ensemble member %d (%dx%dx%d)" % (
            mine[0], p.nr, p.nth, p.nphi))
    ens.close()
    for sim in sims:
        sim.close()
    if rank == 0:
        print(json.dumps(out))
    return 0


CLOSURE_STUDIES = {
    # workload: fine grid, coarse grid, magnetic, n_rho, decompositions, study steps
    "closure-study": ((96, 128, 256), (24, 32, 64), False, 3.0, (3, 4, 8), (2, 2, 4),
                      dict(n_pre=5000, n_adjust=500, n_train=400, nsnap=8, n_win=1000, nstat=10, train_steps=400)),
    "closure-study-mhd": ((256, 512, 1024), (64, 128, 256), True, 5.0, (8, 16, 32), (2, 4, 8),
                          dict(n_pre=20000, n_adjust=500, n_train=500, nsnap=10, n_win=2000, nstat=20,
                               train_steps=600)),
}


PRECISION_STUDIES = {
    # workload: grid, magnetic, mixed steps, FP64 steps, checkpoints, statistics every
    "precision-study": ("hydro-128x256x512", 1000, 1000, (100, 1000), 20),
    "precision-study-mhd": ("mhd-256x512x1024", 500, 100, (100,), 20),
}


def run_precision_study(args):
    """The mixed-precision form beside FP64 from the same seeded state, the
    two runs stepped side by side.  ``precision-study``: hydro 128x256x512,
    1000 steps of each; per-field relative error (max |mixed - fp64| / max
    |fp64|, plane by plane) at steps 100 and 1000, and the time-averaged
    kinetic energy (Scalar_Output's kinener) and enthalpy-flux profile
    (Shell_Average code 16) of each run.  ``precision-study-mhd``: MHD
    256x512x1024, 500 mixed steps with the FP64 run over the first 100 as
    the reference; the error at step 100 and each run's statistics over its
    own steps.  Prints one JSON line."""
    import numpy as np
    import torch
    from css_b200 import problem
    from css_b200.context import Simulation
    torch.cuda.set_device(0)
    name, n_mixed, n_fp64, checks, every = PRECISION_STUDIES[args.workload]
    p, prof, v0, dt, _ = problem.build(name)
    steps = {"fp64": n_fp64, "mixed": n_mixed}
    sims, acc = {}, {}
    for label, prec in (("fp64", 0), ("mixed", 1)):
        q = p.copy()
        q.precision = prec
        sims[label] = Simulation(q, prof)
        sims[label].upload(v0)
        acc[label] = {"ke": [], "fen": [], "ms": 0.0}
    del v0
    names = ["rho", "u_theta", "u_phi", "u_r", "s", "A_theta", "A_phi", "A_r"]
    nv = 8 if p.magnetic else 5
    errors, done = {}, 0
    while done < max(steps.values()):
        k = every
        for label, sim in sims.items():
            if done >= steps[label]:
                continue
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sim.step_rk4(dt, k)
            torch.cuda.synchronize()
            acc[label]["ms"] += 1e3 * (time.perf_counter() - t0)
            acc[label]["ke"].append(sim.scalars()["kinener"])
            acc[label]["fen"].append(sim.shell_averages([16])[0])
        done += k
        if done in checks and done <= min(steps.values()):
            err = {}
            for iv in range(nv):
                dmax = amax = 0.0
                for ir in range(p.nr):
                    a, b = sims["mixed"].plane(iv, ir), sims["fp64"].plane(iv, ir)
                    dmax = max(dmax, float(np.abs(a - b).max()))
                    amax = max(amax, float(np.abs(b).max()))
                err[names[iv]] = dmax / max(amax, 1e-300)
            errors[str(done)] = err
        for label in list(sims):
            if done >= steps[label] and label == "fp64" and steps["mixed"] > steps["fp64"]:
                sims.pop(label).close()  # the reference run ends here; its memory goes back
    for sim in sims.values():
        sim.close()
    res = {k: {"ke": float(np.mean(a["ke"])), "fen": np.mean(a["fen"], axis=0), "ms": a["ms"] / steps[k]}
           for k, a in acc.items()}
    out = {"metric": "mixed-precision state error against FP64 and time-averaged statistics",
           "value": max(max(e.values()) for e in errors.values()), "unit": "max per-field relative error",
           "higher_is_better": False, "n_gpus": 1, "data": "synthetic",
           "config": {"workload": args.workload, "grid": name, "dt": dt, "mixed_steps": n_mixed,
                      "fp64_steps": n_fp64, "statistics_every": every},
           "errors_at_step": errors,
           "kinetic_energy_time_avg": {k: r["ke"] for k, r in res.items()},
           "ms_per_step": {k: r["ms"] for k, r in res.items()},
           "enthalpy_flux_time_avg": {k: [float(x) for x in r["fen"]] for k, r in res.items()}}
    if steps["fp64"] == steps["mixed"]:
        f, m = res["fp64"]["fen"], res["mixed"]["fen"]
        out["enthalpy_flux_rel_diff"] = float(np.linalg.norm(m - f) / max(np.linalg.norm(f), 1e-300))
        out["kinetic_energy_rel_diff"] = abs(res["mixed"]["ke"] - res["fp64"]["ke"]) / max(abs(res["fp64"]["ke"]),
                                                                                            1e-300)
    print(json.dumps(out))
    return 0


def run_closure_study(args):
    """The closure measured against a resolved run (closure.study): a fine run
    box-filtered 4x in every direction trains the network; coarse runs from
    the filtered fine state (prescribed profile, and the closure's two
    couplings) cover the window of the fine run and are compared with its
    filtered statistics.  ``closure-study``: hydro 96x128x256 onto 24x32x64.
    ``closure-study-mhd``: MHD 256x512x1024 onto 64x128x256, a 2000-step
    window (the learned-closure configuration).  Prints one JSON line: the
    relative errors of the time-averaged KE (and ME) spectra (m >= 1),
    enthalpy and kinetic-energy flux profiles of every coarse run, and the
    wall-time ratio of the fine to the coarse window."""
    import torch
    from css_b200 import closure as C
    from css_b200 import problem
    torch.cuda.set_device(0)
    fdims, cdims, mag, nrho, fdec, cdec, kw = CLOSURE_STUDIES[args.workload]
    fp, fprof, fv0, fdt, fi = problem.build(fdims, magnetic=mag, decomp=fdec, n_rho=nrho)
    cp, cprof, cv0, cdt, ci = problem.build(cdims, magnetic=mag, decomp=cdec, n_rho=nrho)
    r = C.study((fp, fprof, fv0, fdt, problem.background(fp, fprof, fi)),
                (cp, cprof, cv0, cdt, problem.background(cp, cprof, ci)), factor=4, **kw)
    out = {"metric": "closure study: relative error of time-averaged spectra (m >= 1) and radial flux profiles "
                     "of coarse runs against the filtered fine run",
           "value": r["errors"]["variance"]["E_K"], "unit": "relative L2 error (KE spectrum, learned closure)",
           "higher_is_better": False, "n_gpus": 1, "data": "synthetic",
           "config": {"workload": args.workload, "fine": list(fdims), "coarse": list(cdims), "filter": 4,
                      "magnetic": mag, "n_rho": nrho, **kw},
           "result": {k: r[k] for k in ("errors", "end_state_error", "fine_window_s", "coarse_window_s",
                                        "pre_spin_s", "wall_ratio", "loss_first", "loss_last", "fine_steps",
                                        "coarse_steps", "fine_dt", "coarse_dt", "t_window")},
           "spectra": {name: {k: [float(x) for x in v[:33]] for k, v in st.items()}
                       for name, st in r["stats"].items()}}
    print(json.dumps(out))
    return 0


def run_closure(args):
    """The closure network (closure-<nr>x<nth>x<nphi>: one row per coarse
    cell): inference over the whole coarse grid and Adam steps of 65536
    rows, both timed with CUDA events on the network's stream.  The bound
    is the tensor cores: achieved FLOP/s of the products against the
    measured BF16 GEMM peak."""
    import numpy as np
    import torch
    from css_b200 import closure as C
    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    nr, nth, nphi = (int(x) for x in args.workload.split("-")[1].split("x"))
    nc = nr * nth * nphi
    batch = 65536
    g = torch.Generator(device="cpu").manual_seed(11)
    xh = torch.zeros(nc, C.XPAD, dtype=torch.bfloat16)
    xh[:, :135] = torch.randn(nc, 135, generator=g).to(torch.bfloat16)
    x = xh.to(dev)
    t = torch.zeros(batch, C.YPAD, dtype=torch.float32)
    t[:, :12] = torch.randn(batch, 12, generator=g)
    t = t.to(dev)
    net = C.Mlp(135, 128, 12, max_rows=batch, seed=1)
    stream = torch.cuda.current_stream(dev)
    net.set_stream(stream.cuda_stream)
    d = net.dims
    fwd_flop_row = 2.0 * sum(d[l] * d[l + 1] for l in range(4))
    # backward: weight gradients of every layer, input gradients of layers 1-3
    bwd_flop_row = 2.0 * sum(d[l] * d[l + 1] for l in range(4)) + 2.0 * sum(d[l] * d[l + 1] for l in range(1, 4))
    for _ in range(args.warmup):
        net.forward(x, nc)
        net.train_step(x[:batch], t, batch, 1e-4)
    clocks = ClockSampler(local)
    if rank == 0:
        clocks.start()
        time.sleep(0.3)
    barrier(world)
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    for _ in range(args.steps):
        net.forward(x, nc)
    e1.record(stream)
    for _ in range(args.steps):
        net.train_step(x[:batch], t, batch, 1e-4)
    e2.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop() if rank == 0 else None
    inf_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
    # the other forward paths, for comparison: the fused mma.sync kernel and
    # the per-layer GEMMs
    other_ms = {}
    for mode in ("mma", "gemm"):
        net.set_forward(mode)
        net.forward(x, nc)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            net.forward(x, nc)
        f1.record(stream)
        torch.cuda.synchronize()
        other_ms[mode] = max_over_ranks(f0.elapsed_time(f1) / args.steps, world)
    net.set_forward("tcgen05")
    gemm_ms = other_ms["gemm"]
    tr_ms = max_over_ranks(e1.elapsed_time(e2) / args.steps, world)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("bf16_tflops", 1590.0)
    inf_tf = fwd_flop_row * nc / (inf_ms / 1e3) / 1e12
    tr_tf = (fwd_flop_row + bwd_flop_row) * batch / (tr_ms / 1e3) / 1e12
    # e2e: features from pinned host memory, inference, predictions back
    xp = xh.pin_memory()
    yp = torch.empty(nc * C.YPAD, dtype=torch.float32).pin_memory()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    xd = xp.to(dev, non_blocking=True)
    y = net.forward(xd, nc)
    yp.copy_(y, non_blocking=True)
    h1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(h0.elapsed_time(h1), world)
    out = {"metric": "closure inference rows/s (one row per coarse cell)", "value": nc * world / (inf_ms / 1e3),
           "unit": "rows/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": inf_ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16 (fp32 accumulate)",
           "data": "synthetic",
           "config": {"workload": args.workload, "rows": nc, "layers": list(d), "train_batch": batch,
                      "l2": "features (%.0f MB) larger than L2" % (nc * C.XPAD * 2 / 1e6)},
           # a training step: 4 weight transposes, 4 GEMMs forward and 7 backward (k_gemm_bf16; the
           # weight gradients add a split-K partial sum each), 4 bias/GELU, loss, 4 column sums,
           # 3 GELU backward, 8 Adam
           "training": {"rows_per_s": batch * world / (tr_ms / 1e3), "ms_per_step": tr_ms, "tflops": tr_tf,
                        "own_kernels_per_step": 39},
           "inference_per_layer_gemms": {"ms": gemm_ms, "rows_per_s": nc * world / (gemm_ms / 1e3)},
           "inference_fused_mma_sync": {"ms": other_ms["mma"], "rows_per_s": nc * world / (other_ms["mma"] / 1e3)},
           "kernel": "k_mlp_tc (one launch: weights in shared memory, 128-row tiles, tcgen05.mma kind::f16 with "
                     "FP32 accumulators in tensor memory)",
           "roofline": {"bound": "tensor", "achieved": inf_tf, "peak": peak, "unit": "TFLOP/s",
                        "frac": inf_tf / peak, "traffic": None, "peak_source": "measured" if peaks else "fallback",
                        "flop_per_row": fwd_flop_row},
           "e2e": {"value": nc * world / (e2e_ms / 1e3), "unit": "rows/s", "h2d_bytes_per_step": nc * C.XPAD * 2,
                   "d2h_bytes_per_step": nc * C.YPAD * 4},
           # the timed inference region launches k_mlp_fused once per pass
           "gpu_launches": args.steps}
    if clk:
        out["clocks"] = clk
    net.close()
    if rank == 0:
        print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mhd-256x512x1024")
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--stage", default="auto", choices=["auto", "four"],
                    help="four: the four-kernel RK4 stage even where the two-pass stage applies")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="mixed: FP32 stage states (rho, s as perturbations), FP64 arithmetic and accumulator")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload.startswith("ensemble-"):
        return run_ensemble(args)
    if args.workload in CLOSURE_STUDIES:
        return run_closure_study(args)
    if args.workload in PRECISION_STUDIES:
        return run_precision_study(args)
    if args.workload.startswith("closure-"):
        return run_closure(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
