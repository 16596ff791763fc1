#!/usr/bin/env python
"""DOF x RK-stage throughput of the Wasl SSP-RK3 step on one B200.

Workload (the metric's quoted configuration): 2D Euler (gamma 1.4) isentropic
vortex of strength 5 centred at (5,5), advected with (1,1) on the periodic
square [0,10]^2; 256x256 quads split along seeded random diagonals with
interior vertices jittered +-0.15h (131,072 triangles); P2 (6 modes x 4
variables, 3,145,728 DOF); CFL 0.15; limiter off.  A step is one SSP-RK3 step
(three stages plus the device CFL reduction).  L2 is flushed (256 MiB write)
between timed steps, outside the timed events.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  Under torchrun each rank advances its own replica
(the path shards by element but this benchmark runs replicas: weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("DOF·RK-stage/s on 1 B200: chosen form vs plain FP64 path at matched L1 error")
UNIT = "DOF*stage/s"
CFL = 0.15
# Algorithmic bytes per stage launch (per DOF and per element): each stage
# reads its input state (8 B/DOF), stages 2-3 also read u^n, and every stage
# writes its output -> (16+24+24)/3 B/DOF on average; per element 40 B of
# geometry, 16 B of face indices/codes and 1.5 faces x 24 B of normals and
# edge scales = 92 B.
BYTES_PER_DOF = 64.0 / 3.0
BYTES_PER_ELEMENT = 92.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--form", choices=["chosen", "plain", "mixed"], default="chosen")
    ap.add_argument("--n", type=int, default=256, help="quads per side")
    ap.add_argument("--p", type=int, default=2)
    ap.add_argument("--rule", type=int, default=None,
                    help="mixed form's volume rule: -1 the symmetric degree-2p rule (default),"
                         " p..p+2 the collapsed rule of that order (the reference uses p+2)")
    ap.add_argument("--kernel", type=int, default=0,
                    help="mixed form's kernel: 0 autotuned, 1 face-centric, 2+s tile shape s")
    ap.add_argument("--workload", choices=["vortex", "advection-line", "batched", "quadrant",
                                           "shock-vortex", "line-euler", "line-scalar",
                                           "tri-scalar"],
                    default="vortex",
                    help="vortex: the 256x256 isentropic vortex (default); advection-line: the"
                         " 400-cell P2 advection run to t = 1 in one launch; batched: independent"
                         " two-state Riemann cases of uneven size and order in one batch;"
                         " quadrant: four-quadrant Riemann, 1024x1024 quads, P3, limiter;"
                         " shock-vortex: 2048x1024 quads, P3, learned indicator;"
                         " line-euler / line-scalar / tri-scalar: the plain FP64 1D Euler"
                         " (4M cells), 1D scalar (16M cells) and 2D scalar (1024x1024 quads)"
                         " paths at P2")
    ap.add_argument("--cases", type=int, default=512, help="batched workload: number of cases")
    ap.add_argument("--quads", type=int, default=1024,
                    help="quadrant / shock-vortex workloads: quads per unit side")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the other workloads the default run reports under other_workloads")
    ap.add_argument("--extra-budget", type=float, default=480.0,
                    help="seconds allowed for the other workloads in total")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons of this process's GPU during the timed
    region, polled through NVML every millisecond from a thread (the timed
    regions are milliseconds long), with one sample when polling starts and
    one when it stops; nvidia-smi polling where NVML is unavailable."""

    # NVML clocks-event reason bits (nvmlClocksEventReason*).
    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, index):
        self.index, self.samples, self.nvml, self.handle = index, [], None, None
        self.smax, self.stop_flag, self.thread = None, threading.Event(), None

    def _open(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(self.index).uuid)
        try:
            handle = pynvml.nvmlDeviceGetHandleByUUID(
                uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except pynvml.NVMLError:
            handle = pynvml.nvmlDeviceGetHandleByIndex(self.index)
        self.nvml, self.handle = pynvml, handle
        self.smax = pynvml.nvmlDeviceGetMaxClockInfo(handle, pynvml.NVML_CLOCK_SM)

    def _sample(self):
        nv, h = self.nvml, self.handle
        self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                             nv.nvmlDeviceGetCurrentClocksEventReasons(h)))

    def _poll(self):
        while not self.stop_flag.wait(0.001):
            try:
                self._sample()
            except Exception:
                return

    def start(self):
        try:
            self._open()
            self._sample()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
        except Exception:
            self.nvml = None

    def stop(self):
        if self.nvml is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["NVML unavailable"],
                    "samples": 0}
        self.stop_flag.set()
        self.thread.join(timeout=2)
        try:
            self._sample()
        except Exception:
            pass
        reasons = sorted(name for name, bit in self.REASONS.items()
                         if any(r & bit for _, r in self.samples))
        sm = [c for c, _ in self.samples]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax,
                "reasons": reasons, "samples": len(sm), "source": "NVML, 1 ms polling"}


# ---------------------------------------------------------------------------------
# ranks (one process per GPU under torchrun; replicas, weak scaling)
# ---------------------------------------------------------------------------------

def init_ranks(world, local_rank, backend="nccl", timeout_s=120):
    """The process group for world > 1 (None for one rank)."""
    if world <= 1:
        return None
    import datetime
    import torch
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl":
        kw["device_id"] = torch.device("cuda", local_rank)
    dist.init_process_group(backend, **kw)
    return dist


def reduce_over_ranks(dist, value, op="max", device="cuda"):
    """value reduced over all ranks (max, min or sum); value itself for one rank."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op={"max": dist.ReduceOp.MAX, "min": dist.ReduceOp.MIN,
                           "sum": dist.ReduceOp.SUM}[op])
    return float(t.item())


# ---------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------

def rule_order(args, form):
    """The plain path: the reference's order-(p+2) rule; the mixed form: the
    symmetric degree-2p rule unless --rule names another."""
    if form == "plain":
        return 0
    return -1 if args.rule is None else args.rule


def rule_description(rule, p):
    if rule == -1:
        return f"symmetric, degree {2 * p} ({ {1: 3, 2: 6, 3: 12}[p]} points)"
    order = rule or p + 2
    return f"collapsed order {order} ({(order + 1) ** 2} points)"


def build_solver(args, form, device):
    import wasl_b200
    from wasl_b200 import cases
    arrays = cases.vortex_mesh(args.n)
    vortex = cases.IsentropicVortex()
    g = wasl_b200.Solver(*arrays, polynomial_order=args.p, precision=form, device=device,
                         volume_rule_order=rule_order(args, form),
                         mixed_kernel=args.kernel if form == "mixed" else 0)
    cases.project_initial(g, vortex.conserved)
    return g, vortex


def time_device_steps(g, args, torch, flush, stream):
    """W untimed steps, then K timed steps, each bracketed by an event pair on
    the handle's stream with L2 flushed between: the headline pass, with no
    event inside a step (timing events between kernels serialise their
    launches: about 15 us per step of three stage kernels).  Then the same K
    steps once more with an event pair around every stage kernel, for the
    stage-kernel times of the roofline and the launch count."""
    g.advance(CFL, args.warmup)
    torch.cuda.synchronize()

    def timed(per_stage_events):
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        if per_stage_events:
            g.profile_begin()
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.zero_()
                starts[k].record(stream)
                g.advance(CFL, 1, sync=False)  # enqueue only: no host round trip inside the events
                ends[k].record(stream)
        torch.cuda.synchronize()
        g.sync()  # device errors of the timed steps
        return sum(s.elapsed_time(e) for s, e in zip(starts, ends))

    total_ms = timed(False)
    timed(True)
    stage_ms, stage_kernels, launches = g.profile_end()
    # Mean stage-kernel ms of RK stages 0, 1, 2 (stage 0 reads u^n after the
    # L2 flush; stages 1 and 2 also read u^n for the Shu-Osher combination).
    by_stage = [round(ms / args.steps, 5) for ms in g.profile_stages()]
    return total_ms, stage_ms, stage_kernels, launches, by_stage


def time_e2e(g, args, torch, stream):
    """Through the C-ABI with host buffers: each step copies the state in from
    pinned host memory, computes the CFL step, advances, and copies it out."""
    n = g.state_size
    host_in = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    host_out = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    g.get_state_into(host_in)
    steps = max(5, min(args.steps, 50))
    for _ in range(2):
        g.set_state(host_in)
        g.step(g.stable_dt(CFL))
        g.get_state_into(host_out)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        g.set_state(host_in)
        g.step(g.stable_dt(CFL))
        g.get_state_into(host_out)
        host_in, host_out = host_out, host_in
    end.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    return 3.0 * n * steps / (ms * 1e-3), steps, 8 * n, 8 * n


def accuracy(args, form, device):
    """Run the vortex to t=1 with the plain and the chosen form; L1 density error."""
    from wasl_b200 import cases
    out = {}
    for name in sorted({"plain", form}):
        g, vortex = build_solver(args, name, device)
        steps, t = g.run(CFL, 0.0, 1.0)
        out[name] = (cases.l1_density_error(g, lambda x, y: vortex.conserved(x, y, t)), steps)
        g.close()
    res = {"t_end": 1.0, "l1_plain_fp64": out["plain"][0], "steps": out["plain"][1]}
    if form != "plain":
        res[f"l1_{form}"] = out[form][0]
        res["ratio"] = out[form][0] / out["plain"][0]
    return res


def cpu_baseline(args):
    """The reference CPU solver (oracle/_ref, else the oracle port) on one core:
    two SSP-RK3 steps of the same workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from wasl_b200 import cases
    arrays = cases.vortex_mesh(args.n)
    vortex = cases.IsentropicVortex()
    oracle = pyoracle.Oracle()
    om = oracle.tri_mesh(*arrays)
    rule = max(args.p, 5)
    xs, ys = om.rule_points(rule)
    c = om.project(args.p, rule, vortex.conserved(xs, ys))
    steps = 2
    if pyoracle.Reference.available():
        ref = pyoracle.Reference()
        mesh = ref.tri_mesh(*arrays)
        donors, basis = mesh.periodic_trace(args.p)
        dt = mesh.cfl(1.4, c, args.p, CFL)
        t0 = time.perf_counter()
        for _ in range(steps):
            mesh.euler_step(1.4, args.p, dt, c, donors, basis)
        elapsed = time.perf_counter() - t0
        kind = "reference"
    else:
        donors, basis = om.periodic_trace(args.p)
        dt = om.cfl(1.4, c, args.p, CFL)
        t0 = time.perf_counter()
        for _ in range(steps):
            om.euler_step(1.4, args.p, dt, c, donors=donors, basis=basis)
        elapsed = time.perf_counter() - t0
        kind = "port"
    dofs = c.size
    return {"value": 3.0 * dofs * steps / elapsed, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{steps} SSP-RK3 steps of the full workload ({om.ne} triangles, P{args.p}),"
                      f" single-threaded, {elapsed:.1f} s"}


# The other workloads of the benchmark suite, run after the headline one in
# the default invocation (one GPU), each in its own process with its own clock
# record: (workload, extra arguments, seconds allowed).
EXTRA_WORKLOADS = [
    ("advection-line", [], 120),
    ("quadrant", ["--steps", "20", "--warmup", "3"], 420),
    ("batched", ["--steps", "200", "--warmup", "3"], 600),
    ("shock-vortex", ["--steps", "20", "--warmup", "3"], 600),
]
EXTRA_KEYS = ("value", "unit", "steps", "ms_per_step", "ms_per_run", "chosen_vs_plain", "roofline",
              "e2e", "gpu_launches", "clocks", "cpu_baseline", "failed_cases", "simulated_time")


def extra_workloads(args):
    """Each other workload's JSON line (its key fields), or why it is absent."""
    out = {}
    budget = time.perf_counter() + args.extra_budget
    for name, extra, limit in EXTRA_WORKLOADS:
        left = budget - time.perf_counter()
        if left < 30:
            out[name] = {"skipped": f"time budget of {args.extra_budget} s used up"}
            continue
        cmd = [sys.executable, os.path.abspath(__file__), "--workload", name, *extra]
        if args.no_cpu:
            cmd.append("--no-cpu")
        t0 = time.perf_counter()
        try:
            run = subprocess.run(cmd, capture_output=True, text=True, timeout=min(limit, left),
                                 cwd=ROOT)
        except subprocess.TimeoutExpired:
            out[name] = {"skipped": f"timed out after {min(limit, left):.0f} s"}
            continue
        lines = [x for x in run.stdout.splitlines() if x.startswith("{")]
        if run.returncode != 0 or not lines:
            out[name] = {"failed": (run.stderr or run.stdout).strip().splitlines()[-1:]}
            continue
        line = json.loads(lines[-1])
        entry = {k: line[k] for k in EXTRA_KEYS if k in line}
        entry["workload"] = line["config"]["workload"]
        entry["wall_s"] = round(time.perf_counter() - t0, 1)
        out[name] = entry
    return out


def ours(args, rank, world, local_rank):
    import torch
    import wasl_b200
    torch.cuda.set_device(local_rank)
    dist = init_ranks(world, local_rank)
    form = args.form
    if form == "chosen":
        form = "mixed" if wasl_b200.form_available("mixed") else "plain"
    g, _ = build_solver(args, form, local_rank)
    stream = torch.cuda.ExternalStream(g.stream_handle())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    sampler = ClockSampler(local_rank)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    total_ms, stage_ms, stage_kernels, launches, by_stage = time_device_steps(g, args, torch, flush,
                                                                              stream)
    clocks = sampler.stop()
    total_ms = reduce_over_ranks(dist, total_ms, "max")
    dofs = g.state_size
    value = world * 3.0 * dofs * args.steps / (total_ms * 1e-3)
    e2e_value, e2e_steps, h2d, d2h = time_e2e(g, args, torch, stream)
    if dist:
        e2e_value = reduce_over_ranks(dist, e2e_value, "min") * world
    peaks, peak_kind = measured_peaks()
    per_launch_bytes = BYTES_PER_DOF * dofs + BYTES_PER_ELEMENT * g.elements
    kernel_s = stage_ms * 1e-3 / max(stage_kernels, 1)
    achieved = per_launch_bytes / kernel_s / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "stage_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(f"{form}_p{args.p}_n{args.n}")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if form == "plain" else "f32+f64",
        "data": "synthetic (seeded jittered mesh, projected isentropic vortex)",
        "config": {"workload": f"isentropic vortex, {args.n}x{args.n} quads -> {g.elements}"
                               f" jittered triangles, P{args.p} Euler, periodic, CFL {CFL},"
                               " limiter off",
                   "form": "plain-fp64" if form == "plain" else "mixed-precision",
                   "volume_rule": rule_description(rule_order(args, form), args.p),
                   "kernel": kernel_description(g.tuning()),
                   "elements": g.elements, "dof": dofs, "parallelism": f"replicas x{world}",
                   "l2": "flushed between timed steps (256 MiB write)",
                   "timing": "K steps with an event pair per step (value); the stage-kernel"
                             " times of the roofline from a second pass of the same K steps"
                             " with an event pair around each stage kernel"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                "path": "C-ABI set_state/stable_dt/step/get_state with pinned host buffers"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "kernel": "euler_tri_stage", "kernel_ms": kernel_s * 1e3,
                     "kernel_ms_by_rk_stage": by_stage,
                     "bytes_per_launch": per_launch_bytes},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_accuracy:
        line["accuracy"] = accuracy(args, form, local_rank)
    if rank == 0 and form != "plain":
        gp, _ = build_solver(args, "plain", local_rank)
        p_ms, _, _, _, _ = time_device_steps(gp, args, torch, flush, stream_of(gp, torch))
        line["plain_fp64"] = {"value": 3.0 * gp.state_size * args.steps / (p_ms * 1e-3),
                              "ms_per_step": p_ms / args.steps}
        line["chosen_vs_plain"] = value / world / line["plain_fp64"]["value"]
        gp.close()
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(args)
    g.close()
    if rank == 0 and world == 1 and not args.no_extra:
        line["other_workloads"] = extra_workloads(args)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def kernel_description(tuning):
    choice, ms = tuning
    names = ["face-centric (face + element kernels)", "tile 128 el/CTA, <=128 regs",
             "tile 128 el/CTA, uncapped regs", "tile 256 el/CTA, <=128 regs",
             "tile 64 el/CTA, <=128 regs", "shared-face tile 64 el/CTA, 7 CTAs/SM",
             "shared-face tile 96 el/CTA, 5 CTAs/SM", "shared-face tile 128 el/CTA, 4 CTAs/SM",
             "shared-face tile 128 el/CTA, 3 CTAs/SM", "patch 128 el/CTA, <=128 regs",
             "patch 128 el/CTA, 5 CTAs/SM", "patch 64 el/CTA, 8 CTAs/SM",
             "patch 64 el/CTA, 10 CTAs/SM", "patch + tensor-core volume 128 el/CTA, <=128 regs",
             "patch + tensor-core volume 128 el/CTA, 5 CTAs/SM",
             "persistent tile 128 el/CTA, <=128 regs", "persistent tile 256 el/CTA, <=128 regs"]
    if choice < 0:
        return {"name": "single stage kernel"}
    out = {"name": names[choice] if choice < len(names) else str(choice)}
    if ms:
        out["autotuned_stage_ms"] = {names[i]: round(t, 5) for i, t in enumerate(ms) if t > 0}
    return out


def stream_of(g, torch):
    return torch.cuda.ExternalStream(g.stream_handle())


# ---------------------------------------------------------------------------------
# reference arm: the reference CPU solver on the host cores
# ---------------------------------------------------------------------------------

# The reference arm's bounded sample: each host process runs the full
# workload mesh for at most REF_STEPS timed steps after at most REF_WARMUP
# untimed ones (a reference step on the 256x256 mesh takes ~10 s on one core).
REF_STEPS, REF_WARMUP = 3, 1


def _ref_worker(n, p, steps, warmup, queue, barrier):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from wasl_b200 import cases
    arrays = cases.vortex_mesh(n)
    vortex = cases.IsentropicVortex()
    oracle = pyoracle.Oracle()
    om = oracle.tri_mesh(*arrays)
    rule = max(p, 5)
    xs, ys = om.rule_points(rule)
    c = om.project(p, rule, vortex.conserved(xs, ys))
    if pyoracle.Reference.available():
        mesh = pyoracle.Reference().tri_mesh(*arrays)
        donors, basis = mesh.periodic_trace(p)
        advance = lambda dt: mesh.euler_step(1.4, p, dt, c, donors, basis)  # noqa: E731
        cfl = lambda: mesh.cfl(1.4, c, p, CFL)  # noqa: E731
        kind = "reference"
    else:
        donors, basis = om.periodic_trace(p)
        advance = lambda dt: om.euler_step(1.4, p, dt, c, donors=donors, basis=basis)  # noqa
        cfl = lambda: om.cfl(1.4, c, p, CFL)  # noqa: E731
        kind = "port"
    for _ in range(warmup):
        advance(cfl())
    barrier.wait()
    t0 = time.perf_counter()
    for _ in range(steps):
        advance(cfl())
    queue.put((time.perf_counter() - t0, c.size, kind))


def reference(args, rank):
    if rank != 0:
        return
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    steps, warmup = max(1, min(args.steps, REF_STEPS)), min(args.warmup, REF_WARMUP)
    queue, barrier = ctx.Queue(), ctx.Barrier(cores)
    procs = [ctx.Process(target=_ref_worker,
                         args=(args.n, args.p, steps, warmup, queue, barrier))
             for _ in range(cores)]
    for pr in procs:
        pr.start()
    results = [queue.get() for _ in procs]
    for pr in procs:
        pr.join()
    elapsed = max(r[0] for r in results)
    dofs = results[0][1]
    kind = results[0][2]
    value = cores * 3.0 * dofs * steps / elapsed
    sample = (f"{cores} independent processes (one per host core), each {steps} timed SSP-RK3"
              f" steps (after {warmup} untimed) of the full workload mesh ({args.n}x{args.n}"
              f" quads, {2 * args.n * args.n} triangles, P{args.p}); the reference solver is"
              " single-threaded")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": steps, "warmup": warmup,
        "ms_per_step": elapsed * 1e3 / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded jittered mesh, projected isentropic vortex)",
        "config": {"workload": f"isentropic vortex, {args.n}x{args.n} quads ->"
                               f" {2 * args.n * args.n} jittered triangles, P{args.p} Euler,"
                               f" periodic, CFL {CFL}, limiter off",
                   "form": "reference CPU (oracle/_ref)" if kind == "reference" else "oracle port",
                   "parallelism": f"{cores} host processes, each the full mesh",
                   "sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------
# 1D advection: the whole 400-cell run in one launch
# ---------------------------------------------------------------------------------

ADVECTION_CELLS, ADVECTION_CFL = 400, 0.1


def advection_cpu(arrays, c0):
    """The reference's own CPU run of the same case (oracle/_ref: its
    SSP-RK3 and run-loop arithmetic in C++, one core), else the oracle port."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    ne, M = ADVECTION_CELLS, 3
    c = np.ascontiguousarray(c0.reshape(M, ne).T).ravel()  # solver layout [element][mode]
    if pyoracle.Reference.available():
        mesh = pyoracle.Reference().line_mesh(*arrays)
        t0 = time.perf_counter()
        steps, _ = mesh.scalar_run(1.0, 2, ADVECTION_CFL, 0.0, 1.0, c)
        return time.perf_counter() - t0, steps, "reference"
    om = pyoracle.Oracle().line_mesh(*arrays)
    dt = om.advection_cfl(1.0, 2, ADVECTION_CFL)
    t, steps = 0.0, 0
    t0 = time.perf_counter()
    while t < 1.0:
        d = min(dt, 1.0 - t)
        om.scalar_step(1.0, 2, d, c)
        t += d
        steps += 1
    return time.perf_counter() - t0, steps, "port"


def advection_line(args, local_rank, cpu=True):
    """1D linear advection u_t + u_x = 0 on 400 jittered periodic cells, P2,
    u0 = sin(2 pi x) + exp(-300 (x - 0.5)^2), CFL 0.1, to t = 1 (~33,000
    steps): each timed repetition is the whole run, on the device in one
    kernel launch (wasl_gpu_run_resident), plain FP64 and bit-identical to the
    reference's run.  e2e adds the state's copies in and out through the
    C-ABI; the reference's CPU run of the same case is timed beside it."""
    import torch
    import wasl_b200
    from wasl_b200 import cases
    torch.cuda.set_device(local_rank)
    arrays = cases.advection_line_mesh(ADVECTION_CELLS)
    pulse = cases.AdvectedPulse(1.0)
    g = wasl_b200.Solver(*arrays, dimensions=1, equation="scalar", polynomial_order=2,
                         velocity=(1.0, 0.0), device=local_rank)
    cases.project_line(g, pulse.value)
    c0 = g.get_state()
    stream = torch.cuda.ExternalStream(g.stream_handle())
    reps = max(1, min(args.steps, 5))
    for _ in range(max(1, min(args.warmup, 2))):
        g.set_state(c0)
        steps, t = g.run_resident(ADVECTION_CFL, 0.0, 1.0)
    sampler = ClockSampler(local_rank)
    sampler.start()
    ms = 0.0
    launches = 0
    for _ in range(reps):
        g.set_state(c0)
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g.profile_begin()
        start.record(stream)
        steps, t = g.run_resident(ADVECTION_CFL, 0.0, 1.0)
        end.record(stream)
        torch.cuda.synchronize()
        launches += g.profile_end()[2]
        ms += start.elapsed_time(end)
    # end to end: host state in, the whole run, state out
    host = torch.empty(g.state_size, dtype=torch.float64, pin_memory=True).numpy()
    host[:] = c0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        g.set_state(host)
        g.run_resident(ADVECTION_CFL, 0.0, 1.0)
        g.get_state_into(host)
        host[:] = c0
    e2e_s = time.perf_counter() - t0
    clocks = sampler.stop()
    error = cases.l1_line_error(g, lambda x: pulse.value(x, t))
    dof_stages = 3.0 * g.state_size * steps
    line = {"metric": METRIC, "value": dof_stages * reps / (ms * 1e-3), "unit": UNIT,
            "n_gpus": 1, "steps": steps, "repetitions": reps, "ms_per_run": ms / reps,
            "ms_per_step": ms / reps / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded jittered line, projected sine + Gaussian)",
            "config": {"workload": f"1D scalar advection, {ADVECTION_CELLS} jittered periodic"
                                   f" cells, P2, a = 1, CFL {ADVECTION_CFL}, t = 1 ({steps}"
                                   " steps), limiter off, whole run in one kernel launch",
                       "form": "plain-fp64", "dof": g.state_size,
                       "l1_error_at_t1": error},
            "e2e": {"value": dof_stages * reps / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": 8 * g.state_size / steps,
                    "d2h_bytes_per_step": 8 * g.state_size / steps,
                    "path": "C-ABI set_state / run_resident / get_state, host wall clock"},
            "roofline": {"bound": "latency",
                         "note": "the state (9.6 KB) lives in one SM's shared memory for the"
                                 " whole run; the run is a chain of 3 x steps dependent stages"},
            "gpu_launches": launches, "clocks": clocks}
    if cpu:
        cpu_s, cpu_steps, kind = advection_cpu(arrays, c0)
        line["cpu_baseline"] = {"value": 3.0 * g.state_size * cpu_steps / cpu_s, "unit": UNIT,
                                "cores": 1, "kind": kind,
                                "sample": f"the whole run to t = 1 ({cpu_steps} steps),"
                                          f" single-threaded, {cpu_s:.2f} s"}
    g.close()
    return line


# ---------------------------------------------------------------------------------
# batched workload
# ---------------------------------------------------------------------------------

def batched(args, rank, world, local_rank):
    """Independent planar two-state Riemann cases on [0,1]^2 (triangle counts
    log-uniform in [2k, 128k], orders drawn from {1,2,3}, transmissive
    boundaries, limiter on with positivity on every element, mixed form with
    the order-p volume rule), advanced
    together by one Batch: per-case CFL dt (CFL 0.1), tile shape autotuned per
    order, each step replayed from a CUDA graph.  Every rank runs its own batch
    (replicas, weak scaling)."""
    import torch
    import wasl_b200
    from wasl_b200 import cases
    torch.cuda.set_device(local_rank)
    dist = init_ranks(world, local_rank, timeout_s=600)
    cfl = 0.1
    t0 = time.perf_counter()
    specs = cases.batched_riemann_cases(args.cases, seed=4 + rank)
    b = wasl_b200.Batch([s[:4] for s in specs], limiting=True, positivity_all=True,
                        boundary="transmissive", device=local_rank)
    setup_s = time.perf_counter() - t0
    for c, s in enumerate(specs):
        cases.project_batch_case(b, c, s[4].conserved, s[3])
    b.limit()
    stream = torch.cuda.ExternalStream(b.stream_handle())
    b.advance(cfl, args.warmup)  # autotune, graph capture
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    b.advance(cfl, args.steps)
    end.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = reduce_over_ranks(dist, start.elapsed_time(end), "max")
    value = world * 3.0 * b.dof * args.steps / (ms * 1e-3)
    per_step, graph, _ = b.launches()
    # e2e through the C-ABI with host buffers: every case's state in from
    # pinned host memory, one step, every state out.
    sizes = [b.case_size(c) for c in range(b.cases)]
    host = [torch.empty(4 * nm * ne, dtype=torch.float64, pin_memory=True).numpy()
            for ne, nm in sizes]
    for c in range(b.cases):
        host[c][:] = b.get_state(c)
    e2e_steps = 3
    start.record(stream)
    for _ in range(e2e_steps):
        for c in range(b.cases):
            b.set_state(c, host[c])
        b.advance(cfl, 1)
        for c in range(b.cases):
            b._check(b._lib.wasl_batch_get_state(b._h, c, wasl_b200._ptr(host[c]), host[c].size))
    end.record(stream)
    torch.cuda.synchronize()
    e2e_ms = start.elapsed_time(end) / e2e_steps
    times, dts = b.times()
    status = b.status()
    peaks, peak_kind = measured_peaks()
    per_step_bytes = 3.0 * (BYTES_PER_DOF * b.dof + BYTES_PER_ELEMENT * b.elements)
    achieved = per_step_bytes / (ms * 1e-3 / args.steps) / 1e9
    orders = sorted(set(b.orders))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded jittered meshes, projected two-state Riemann data)",
        "config": {"workload": f"batched: {b.cases} independent two-state Riemann cases,"
                               f" {b.elements} triangles in total (log-uniform 2k-128k per case),"
                               " orders {1,2,3}, transmissive, limiter on (positivity on every"
                               " element), CFL 0.1 per case",
                   "form": "mixed-precision batched (tile work list, CUDA graph)",
                   "elements": b.elements, "dof": b.dof,
                   "cases_per_order": {p: b.orders.count(p) for p in orders},
                   "tile_shape_per_order": {p: b.tuning(p)[0] for p in orders},
                   "autotuned_stage_ms": {p: [round(t, 4) for t in b.tuning(p)[1]]
                                          for p in orders},
                   "setup_s": round(setup_s, 1), "graph": graph,
                   "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (state " f"{8 * b.dof / 1e9:.2f} GB)"},
        "e2e": {"value": 3.0 * b.dof / (e2e_ms * 1e-3), "unit": UNIT,
                "h2d_bytes_per_step": 8 * b.dof, "d2h_bytes_per_step": 8 * b.dof,
                "path": "wasl_batch_set_state / advance / get_state per case, pinned host buffers"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": None,
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "note": "whole step (CFL, three stages, limiter) over algorithmic bytes"},
        "gpu_launches": per_step * args.steps,
        "clocks": clocks,
        "simulated_time": {"min": float(times.min()), "max": float(times.max())},
        "failed_cases": {"count": int((status != 0).sum()),
                         "cases": [int(c) for c in np.nonzero(status)[0][:20]],
                         "note": "a failed case is frozen (dt 0) and still swept by every launch"},
    }
    b.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------
# limited P3 workloads (four-quadrant Riemann; shock-vortex with the learned indicator)
# ---------------------------------------------------------------------------------

def timed_steps(g, torch, steps, cfl):
    """Device-resident steps (CFL on the device every step), enqueued without
    host round trips and timed with events on the handle's stream; device
    errors are checked after the timed region."""
    stream = torch.cuda.ExternalStream(g.stream_handle())
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g.profile_begin()
    start.record(stream)
    g.advance(cfl, steps, sync=False)
    end.record(stream)
    torch.cuda.synchronize()
    g.sync()
    _, _, launches = g.profile_end()
    return start.elapsed_time(end), launches


LIMITED_STEPS, LIMITED_WARMUP = 20, 3


def limited(args, rank, world, local_rank):
    """Four-quadrant Riemann (seeded states in the config's ranges, redrawn
    where an interface would open a vacuum) on [0,1]^2, 1024x1024 quads,
    transmissive, P3, characteristic WENO + positivity, CFL 0.1; or the Mach
    1.1 shock-vortex on [0,2]x[0,1] with 2048x1024 quads, P3, with the learned
    indicator (trained first on seeded two-state Riemann runs of the method
    with the reference sensor) and positivity on every element.  A bounded
    number of timed steps (a full run to t = 0.25 / 0.6 is ~10^5 steps): at
    most LIMITED_STEPS after at most LIMITED_WARMUP, because on the seeded
    four-quadrant data the plain path (positivity only in troubled cells, as
    the reference limits) produces a non-physical cell average after about
    60 steps, and the mixed form (positivity on every element) after about
    300; the reference's algorithm on the CPU breaks down on the same data
    too."""
    import torch
    import wasl_b200
    args.steps = min(args.steps, LIMITED_STEPS)
    args.warmup = min(args.warmup, LIMITED_WARMUP)
    from wasl_b200 import cases, indicator, meshgen
    torch.cuda.set_device(local_rank)
    cfl = 0.1
    p = 3
    t0 = time.perf_counter()
    if args.workload == "quadrant":
        arrays = meshgen.jittered_box(args.quads, jitter=0.15, seed=3)
        problem = cases.QuadrantRiemann(seed=3)
        forms = ("plain", "mixed")
        weights = None
    else:
        arrays = indicator.shock_vortex_mesh(args.quads, seed=5)
        problem = cases.ShockVortex(seed=5)
        forms = ("mixed",)
        xs, ys = [], []
        for seed in range(12):
            a = meshgen.jittered_box(24, jitter=0.15, seed=seed)
            x, y = indicator.collect_run(a, cases.PlanarRiemann(seed=seed), p, 100, 4,
                                         boundary="transmissive", positivity_all=True)
            xs.append(x)
            ys.append(y)
        xb, yb = indicator.balance(np.concatenate(xs), np.concatenate(ys), 3, seed=0)
        weights, train_loss = indicator.train(xb, yb)
    out = {}
    for form in forms:
        g = wasl_b200.Solver(*arrays, polynomial_order=p, precision=form, limiting=True,
                             boundary="transmissive", device=local_rank,
                             volume_rule_order=-1 if form == "mixed" else 0,
                             positivity_all=form == "mixed")
        setup_s = time.perf_counter() - t0
        setup_ms = {k: round(v, 1) for k, v in g.setup_times().items()}
        cases.project_initial(g, problem.conserved)
        g.limit()
        if weights is not None:
            g.set_indicator(weights, 0.005, 0.999)
        for _ in range(args.warmup):
            g.step(g.stable_dt(cfl))
        if weights is not None:
            g.indicator_stats(reset=True)
        sampler = ClockSampler(local_rank)
        sampler.start()
        ms, launches = timed_steps(g, torch, args.steps, cfl)
        clocks = sampler.stop()
        flags = g.flags()
        entry = {"value": 3.0 * g.state_size * args.steps / (ms * 1e-3),
                 "ms_per_step": ms / args.steps, "gpu_launches": launches,
                 "troubled_fraction_last_step": float(flags.mean()),
                 "setup_s": round(setup_s, 1), "setup_ms_by_phase": setup_ms,
                 "kernel": kernel_description(g.tuning()), "clocks": clocks}
        if weights is not None:
            entry["indicator"] = g.indicator_stats()
            entry["indicator_training_loss"] = train_loss
        out[form] = entry
        elements, dof = g.elements, g.state_size
        g.close()
        t0 = time.perf_counter()
    chosen = out["mixed"]
    peaks, peak_kind = measured_peaks()
    bytes_per_step = 3.0 * (BYTES_PER_DOF * dof + BYTES_PER_ELEMENT * elements)
    achieved = bytes_per_step / (chosen["ms_per_step"] * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": chosen["value"], "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": chosen["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded jittered mesh, projected initial data)",
        "config": {"workload": (f"four-quadrant Riemann, {args.quads}x{args.quads} quads ->"
                                f" {elements}"
                                " jittered triangles, P3, transmissive, WENO + positivity,"
                                " CFL 0.1" if args.workload == "quadrant" else
                                f"shock-vortex, {2 * args.quads}x{args.quads} quads ->"
                                f" {elements} jittered"
                                " triangles, P3, transmissive, learned indicator + WENO +"
                                " positivity on every element, CFL 0.1"),
                   "elements": elements, "dof": dof, "forms": out,
                   "l2": f"inputs larger than L2 (state {8 * dof / 1e9:.2f} GB)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "note": "whole step (CFL, stages, indicator, limiter) over algorithmic"
                             " bytes"},
        "gpu_launches": chosen["gpu_launches"],
        "clocks": chosen["clocks"],
    }
    if "plain" in out:
        line["chosen_vs_plain"] = chosen["value"] / out["plain"]["value"]
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------
# plain FP64 1D Euler, 1D scalar and 2D scalar paths (meshes larger than L2)
# ---------------------------------------------------------------------------------

OTHER_PATHS = {
    # workload: (dimensions, equation, cells or quads per side, cell means)
    "line-euler": (1, "euler", 1 << 22, (1.0, 0.2, 0.0, 2.5)),
    "line-scalar": (1, "scalar", 1 << 24, (1.0,)),
    "tri-scalar": (2, "scalar", 1024, (1.0,)),
}


def other_path(args, rank, world, local_rank):
    """A smooth random P2 state (mode 0 from the cell means, higher modes
    1e-3 N(0,1), seed 1) on a periodic jittered mesh; device-resident steps
    at CFL 0.1 timed with events on the handle's stream."""
    import torch
    import wasl_b200
    from wasl_b200 import meshgen
    torch.cuda.set_device(local_rank)
    dims, equation, n, means = OTHER_PATHS[args.workload]
    arrays = (meshgen.jittered_line(n, jitter=0.2, seed=1) if dims == 1
              else meshgen.jittered_box(n, jitter=0.15, seed=1))
    g = wasl_b200.Solver(*arrays, dimensions=dims, equation=equation, polynomial_order=2,
                         velocity=(1.0, 0.5) if equation == "scalar" else (0.0, 0.0),
                         device=local_rank)
    rng = np.random.Generator(np.random.PCG64(1))
    c = 1e-3 * rng.standard_normal((g.variables, g.modes, g.elements))
    for v, mean in enumerate(means[:g.variables]):
        c[v, 0] = np.sqrt(2.0) * mean
    g.set_state(c.ravel())
    for _ in range(args.warmup):
        g.step(g.stable_dt(0.1))
    steps = max(1, min(args.steps, 50))
    ms, launches = timed_steps(g, torch, steps, 0.1)
    line = {"metric": METRIC, "value": 3.0 * g.state_size * steps / (ms * 1e-3), "unit": UNIT,
            "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": ms / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded jittered mesh, smooth random state)",
            "config": {"workload": f"{args.workload}: {g.elements} elements, P2, periodic,"
                                   " CFL 0.1, plain FP64",
                       "elements": g.elements, "dof": g.state_size,
                       "l2": f"inputs larger than L2 (state {8 * g.state_size / 1e6:.0f} MB)"},
            "gpu_launches": launches}
    g.close()
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference(args, rank)
    elif args.workload == "advection-line":
        if rank == 0:
            print(json.dumps(advection_line(args, local_rank, cpu=not args.no_cpu)), flush=True)
    elif args.workload == "batched":
        batched(args, rank, world, local_rank)
    elif args.workload in ("quadrant", "shock-vortex"):
        if rank == 0:
            limited(args, rank, world, local_rank)
    elif args.workload in OTHER_PATHS:
        if rank == 0:
            other_path(args, rank, world, local_rank)
    else:
        ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
