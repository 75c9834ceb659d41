"""Benchmark of the InteraxFF short-range path on B200: the plain drop-in at size (24,000-atom water box).

One step = one velocity-Verlet MD step of 1 fs on the device: the fused pair pass (dispersion + exchange + short
range over one neighbor list, with the list maintenance it needs) and the three-body (ATM) pass over 8,000 molecular
sites, plus the integration.  Metric: interactions/s, the interacting pairs plus interacting triples evaluated per
second (the pair and triple counts come from the kernels, per step); ns/day follows from the step time.

  value      device-resident: per-step CUDA-event time on the context's stream, L2 flushed between steps
  e2e        through the C ABI with host buffers: positions host->device, evaluation, forces device->host, per step
  roofline   the pair kernel (the dominant kernel): algorithmic operations per launch (pairs x F_PAIR) over its
             event-timed duration, against the device's FP32 issue peak measured live by ix_measure_fp32_peak
  cpu_baseline  the reference's CPU platform algorithm (restated in oracle/cpu_platform.cpp) on every host thread

--impl reference times the reference's own CPU implementation of the path (its CPU platform, restated, since the
plugin cannot be built without OpenMM) on every host thread, one full evaluation of the same workload per step.
"""
import os

# Kernels of many CUDA streams run concurrently only as far as the device's hardware work queues keep them apart;
# the default 8 queues make the served stream's requests wait behind one another's work.  Read when CUDA starts.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import argparse  # noqa: E402
import ctypes  # noqa: E402
import json  # noqa: E402
import math  # noqa: E402
import subprocess  # noqa: E402
import sys  # noqa: E402
import threading  # noqa: E402
import time  # noqa: E402
from pathlib import Path  # noqa: E402

ROOT = Path(__file__).resolve().parent
sys.path[:0] = [str(ROOT / "openmm-interax-plugin_b200"), str(ROOT / "oracle")]

import numpy as np  # noqa: E402

# Algorithmic operations per interacting pair and per interacting triple of the reference algorithm, counted once by
# running the FP64 oracle on counting values over the 24,000-atom box (oracle/count_ops.py): the three pair terms'
# functions (order-6 Taylor overlap for equal widths, closed form otherwise, full Tang-Toennies series) plus the pair
# driver, and the ATM triple with C9.
F_PAIR = 612.4
F_TRIPLE = 151.0
# DRAM bytes (read + write) of one pair-kernel launch on this workload, from one ncu capture of an MD-step launch
# (dram__bytes.sum.per_second x gpu__time_duration.sum); the kernel is FP32-issue bound, the traffic is reported beside it
PAIR_TRAFFIC_BYTES = 10162432
# The same capture's hardware view: FMA-pipe busy fraction (sm__pipe_fma_cycles_active, pct of peak over active
# cycles) and issue-slot use (sm__inst_issued), beside the algorithmic fraction
PAIR_FMA_PIPE_ACTIVE = 0.355
PAIR_ISSUE_ACTIVE = 0.747
METRIC = "interactions/s"
WORKLOAD = "water box 24,000 atoms (8,000 rigid 3-site waters, constrained, 6.208 nm periodic, cutoff 1.0 nm) + ATM " \
           "on 8,000 molecular sites (cutoff 0.6 nm); velocity-Verlet 1 fs with SHAKE/RATTLE"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default="24k")
    p.add_argument("--seed", type=int, default=1)
    # graph: each step replays one CUDA graph (conditional nodes skip the list rebuild); direct: kernel by kernel,
    # the same kernels and results (profilers cannot see into graphs with conditional nodes)
    p.add_argument("--launch", default="graph", choices=["graph", "direct"])
    # served stream: Poisson arrival rate (requests/s) of its latency phase and the server's running-request limit
    p.add_argument("--rate", type=float, default=100.0)
    p.add_argument("--latency-requests", type=int, default=4000)
    p.add_argument("--max-running", type=int, default=512)
    p.add_argument("--requests", type=int, default=20000)
    p.add_argument("--server-threads", type=int, default=3)
    p.add_argument("--cohort-window", type=float, default=200e-6)
    return p.parse_args()


_T0 = time.time()


def progress(msg):
    """A stage of the run on stderr (the JSON line alone goes to stdout)."""
    print(f"[bench {time.time() - _T0:7.1f} s] {msg}", file=sys.stderr, flush=True)


def dist_init(args):
    """One process per GPU under torchrun (NCCL); on a host without GPUs (the CPU tests of the rank logic) the ranks
    use gloo.  Returns (rank, world)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
            backend = "nccl"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world


def _rank_reduce(x, world, op):
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=op)
    return float(t.item())


def rank_max(x, world):
    """x's maximum over the ranks: a timed region lasts as long as its slowest rank."""
    import torch.distributed as dist
    return _rank_reduce(x, world, dist.ReduceOp.MAX)


def rank_sum(x, world):
    """x summed over the ranks (work done by the whole job)."""
    import torch.distributed as dist
    return _rank_reduce(x, world, dist.ReduceOp.SUM)


def build_system(args, rank, rigid=True):
    from interaxplugin import workloads as W
    cfg = W.CONFIGS[args.config]
    # every rank runs an independent replica (a single box does not shard)
    return W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=args.seed + rank,
                       three_body_cutoff=cfg["three_body_cutoff"], rigid=rigid)


def relax(ctx, system, positions, iterations=60, max_step=0.01):
    """Steepest descent with a capped step, so that 1 fs velocity Verlet starts without the lattice's hot contacts.
    A System with constraints (rigid waters, three consecutive particles) moves each molecule as a whole along its
    total force, so that its geometry is kept."""
    pos = positions.copy()
    rigid = system.getNumConstraints() > 0
    for _ in range(iterations):
        ctx.setPositions(pos)
        f = ctx.getState(getEnergy=False).getForces()
        if rigid:
            f = np.repeat(f.reshape(-1, 3, 3).sum(1), 3, axis=0)
        fmax = np.sqrt((f ** 2).sum(1)).max()
        pos = pos + f * (max_step / max(fmax, 1e-12))
    ctx.setPositions(pos)
    return pos


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled through NVML every ~1 ms during the timed region (the
    region lasts milliseconds, too short for nvidia-smi's sampling period).  Read-only: no setting is changed."""
    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
        except Exception:
            self.nvml = None
        return self

    def _run(self):
        nv = self.nvml
        while not self._stop.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM)))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                for name, bit in self.REASONS.items():
                    if mask & bit:
                        self.reasons.add(name)
            except Exception:
                break
            time.sleep(0.001)

    def __exit__(self, *exc):
        self._stop.set()
        if self.nvml:
            self.thread.join(timeout=5)

    def summary(self):
        return {"sm_mhz": float(np.median(self.samples)) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def cpu_baseline(system, pos, box, min_seconds=10.0, max_evaluations=50):
    """The reference's CPU platform algorithm (its restatement in oracle/cpu_platform.cpp: FP32 pair forces one pass
    each with a per-evaluation neighbor list, FP64 three-body by marking, on every host thread) timed on full
    energy+force evaluations of the workload: at least `min_seconds` of evaluations (after one untimed warm-up)."""
    import pyoracle
    cpu = pyoracle.CpuPlatform(system)
    cpu.evaluate(pos, box)
    interactions, elapsed, evaluations = 0, 0.0, 0
    while elapsed < min_seconds and evaluations < max_evaluations:
        counts = []
        t0 = time.perf_counter()
        cpu.evaluate(pos, box, counts=counts)
        elapsed += time.perf_counter() - t0
        interactions += sum(counts)
        evaluations += 1
    return {"value": interactions / elapsed, "unit": METRIC, "cores": cpu.threads, "kind": "port",
            "sample": f"{evaluations} full energy+force evaluations of the 24,000-atom box (pairs of the three forces "
                      f"in FP32, triples in FP64) by the restatement of the reference's CPU platform on "
                      f"{cpu.threads} threads, {elapsed:.1f} s",
            "seconds_per_evaluation": elapsed / evaluations}


def run_reference(args, rank, world):
    """The reference's CPU implementation of the path (its CPU platform, restated: the plugin needs OpenMM to build),
    on every host thread: one full energy+force evaluation of the 24,000-atom box per step."""
    if rank != 0:
        return
    import pyoracle
    system, pos, box = build_system(args, 0)
    cpu = pyoracle.CpuPlatform(system)
    times, interactions = [], 0
    for step in range(args.warmup + args.steps):
        counts = []
        t0 = time.perf_counter()
        cpu.evaluate(pos, box, counts=counts)
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt)
            interactions += sum(counts)
    value = interactions / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * float(np.mean(times)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD + " (one energy+force evaluation per step)"},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cpu.threads, "kind": "port",
                             "sample": "one full energy+force evaluation of the 24,000-atom box per step by the "
                                       "restatement of the reference's CPU platform (FP32 pairs, FP64 triples) on "
                                       f"{cpu.threads} threads"},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def md_ns_per_day(args, built, device, dt_ps):
    """ns/day of velocity-Verlet on a (system, positions, box) from build_system (relaxed first), over the bench's
    step count: mean step time by CUDA events on the context's stream, L2 flushed between steps."""
    import torch
    from interaxplugin import Context, _capi
    from interaxplugin import workloads as W
    system, pos0, _ = built
    ctx = Context(system, properties={"DeviceIndex": device})
    L = _capi.lib()
    pos = relax(ctx, system, pos0)
    vel = np.ascontiguousarray(W.initial_velocities(system, 300.0, seed=0))
    masses = np.array([system.getParticleMass(i) for i in range(system.getNumParticles())])
    ctx._check(L.ix_md_set_masses(ctx._ctx, _capi.ptr(masses)))
    ctx._check(L.ix_md_run(ctx._ctx, 1, dt_ps, None, _capi.ptr(vel), None))
    stream = torch.cuda.ExternalStream(L.ix_get_stream(ctx._ctx))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    ms = []
    for step in range(args.warmup + args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx._check(L.ix_md_steps_async(ctx._ctx, 1, dt_ps))
        b.record(stream)
        ctx._check(L.ix_md_finish(ctx._ctx, None, None, None))
        if step >= args.warmup:
            ms.append(a.elapsed_time(b))
    return 86400 * dt_ps * 1e-3 / (float(np.mean(ms)) * 1e-3)


def general_pair_kernel(args, device, peak_tflops, evaluations=20):
    """The pair kernel's per-particle instance (no class-pair table: more than 16 parameter classes, as in an
    InteraxFF system of many atom types) on the 24,000-atom box with 32 variants of each atom type (64 classes):
    its CUDA-event duration per launch and achieved fraction of the FP32 peak, and the oracle error of one
    evaluation."""
    import pyoracle
    from interaxplugin import Context, _capi
    from interaxplugin import workloads as W
    cfg = W.CONFIGS[args.config]
    system, pos, box = W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=args.seed,
                                   three_body_cutoff=cfg["three_body_cutoff"], rigid=True, distinct=32)
    ctx = Context(system, properties={"DeviceIndex": device})
    L = _capi.lib()
    pos = relax(ctx, system, pos, iterations=20)
    ctx._check(L.ix_set_profiling(ctx._ctx, 2))
    times, pairs = [], 0
    for k in range(evaluations + 3):
        st = ctx.getState()
        pms, tms = ctypes.c_double(), ctypes.c_double()
        ctx._check(L.ix_get_kernel_times(ctx._ctx, ctypes.byref(pms), ctypes.byref(tms)))
        if k >= 3:
            times.append(pms.value)
        pairs = ctx.getCounts()[0]
    pair_ms = float(np.median(times))
    achieved = pairs * F_PAIR / (pair_ms * 1e-3) / 1e12
    e_or, f_or = pyoracle.evaluate(system, pos, box)
    f = st.getForces()
    return {"kernel_ms": pair_ms, "achieved": achieved, "frac": achieved / peak_tflops, "unit": "TFLOP/s",
            "pairs": int(pairs), "parameter_classes": 64,
            "oracle_error": {"energy_rel": abs(st.getPotentialEnergy() - e_or) / abs(e_or),
                             "force_rms_rel": float(np.sqrt(((f - f_or) ** 2).mean() / (f_or ** 2).mean()))}}


def run_ours(args, rank, world):
    import torch
    from interaxplugin import Context, _capi
    from interaxplugin import workloads as W

    device = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(device)
    progress("building the 24k box")
    system, pos0, box = build_system(args, rank)
    ctx = Context(system, properties={"DeviceIndex": device})
    L = _capi.lib()
    if args.launch == "direct":
        ctx._check(L.ix_set_graphs(ctx._ctx, 0))
    pos = relax(ctx, system, pos0)
    vel = W.initial_velocities(system, 300.0, seed=rank)
    dt_ps = 0.001
    # masses, velocities and the first forces
    masses = np.array([system.getParticleMass(i) for i in range(system.getNumParticles())])
    ctx._check(L.ix_md_set_masses(ctx._ctx, _capi.ptr(masses)))
    vel = np.ascontiguousarray(vel)
    ctx._check(L.ix_md_run(ctx._ctx, 1, dt_ps, None, _capi.ptr(vel), None))
    stream = torch.cuda.ExternalStream(L.ix_get_stream(ctx._ctx))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")   # 256 MB > 126 MB L2
    peak = ctypes.c_double()
    ctx._check(L.ix_measure_fp32_peak(device, ctypes.byref(peak)))

    def md_step():
        with torch.cuda.stream(stream):
            flush.zero_()
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        ctx._check(L.ix_md_steps_async(ctx._ctx, 1, dt_ps))
        end.record(stream)
        rc = L.ix_md_finish(ctx._ctx, None, None, None)
        if rc != 0:
            raise RuntimeError(L.ix_last_error(ctx._ctx).decode())
        pair_ms, atm_ms = ctypes.c_double(), ctypes.c_double()
        ctx._check(L.ix_get_kernel_times(ctx._ctx, ctypes.byref(pair_ms), ctypes.byref(atm_ms)))
        pairs, triples = ctx.getCounts()
        return start.elapsed_time(end), pair_ms.value, atm_ms.value, pairs, triples

    progress("relaxed; MD warm-up")
    for _ in range(args.warmup):
        md_step()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    progress("timed MD steps")
    rows = []
    launches0 = ctypes.c_longlong()
    ctx._check(L.ix_get_launch_count(ctx._ctx, ctypes.byref(launches0)))
    with ClockSampler(device) as clocks:
        for _ in range(args.steps):
            rows.append(md_step())
    torch.cuda.synchronize()
    launches1 = ctypes.c_longlong()
    ctx._check(L.ix_get_launch_count(ctx._ctx, ctypes.byref(launches1)))
    rows = np.array(rows)
    step_ms = rows[:, 0].sum()
    interactions = rows[:, 3].sum() + rows[:, 4].sum()
    # kernel durations for the roofline, in a separate pass of the same steps with events around the pair and triple
    # kernels and the three-body chain serialised after the pair chain, so that each bracket holds one kernel alone
    ctx._check(L.ix_set_profiling(ctx._ctx, 2))
    kernel_rows = np.array([md_step() for _ in range(args.warmup + args.steps)][args.warmup:])
    ctx._check(L.ix_set_profiling(ctx._ctx, 0))
    step_ms = rank_max(step_ms, world)
    interactions = rank_sum(interactions, world)
    value = interactions / (step_ms * 1e-3)
    ms_per_step = step_ms / args.steps

    # e2e: through the host API (positions in, forces out, pinned host buffers) over configurations of the same
    # trajectory, one per step, recorded first by continuing the MD run (untimed)
    n = system.getNumParticles()
    hfor = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    cur = np.empty((n, 3))
    ctx._check(L.ix_md_finish(ctx._ctx, _capi.ptr(cur), None, None))
    frames = []
    for _ in range(args.warmup + args.steps):
        ctx._check(L.ix_md_steps_async(ctx._ctx, 1, dt_ps))
        ctx._check(L.ix_md_finish(ctx._ctx, _capi.ptr(cur), None, None))
        frames.append(torch.from_numpy(cur.copy()).pin_memory())
    terms = np.zeros(4)
    energy = ctypes.c_double()
    e2e_t, e2e_inter = 0.0, 0
    for step in range(args.warmup + args.steps):
        hpos = frames[step]
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx._check(L.ix_set_positions(ctx._ctx, ctypes.c_void_p(hpos.data_ptr()), None))
        ctx._check(L.ix_compute(ctx._ctx, -1, 1, 1, _capi.ptr(terms), ctypes.byref(energy),
                                ctypes.c_void_p(hfor.data_ptr())))
        t1 = time.perf_counter()
        if step >= args.warmup:
            e2e_t += t1 - t0
            p, tr = ctx.getCounts()
            e2e_inter += p + tr
    e2e_value = e2e_inter / e2e_t

    if rank != 0:
        return
    progress("timed steps and e2e done; oracle error")
    # the error of this run against the FP64 oracle: the last e2e frame, evaluated by both (outside the timed region)
    import pyoracle
    last = frames[-1].numpy()
    e_or, f_or = pyoracle.evaluate(system, last, box)
    f_gpu = hfor.numpy()
    oracle_error = {"energy_rel": abs(energy.value - e_or) / abs(e_or),
                    "force_rms_rel": float(np.sqrt(((f_gpu - f_or) ** 2).mean() / (f_or ** 2).mean())),
                    "frame": "the last configuration of the e2e pass (rigid-water MD trajectory)"}
    # the same box without constraints (flexible waters whose intramolecular pairs are excluded), for comparison
    progress("unconstrained ns/day")
    flex = md_ns_per_day(args, build_system(args, rank, rigid=False), device, dt_ps)
    progress("general pair-kernel instance")
    # the pair kernel's general instance: the same box with every atom its own parameter class
    general = general_pair_kernel(args, device, peak.value)
    # the batched workload's evaluations/s beside the plain per-system path (one GPU)
    batched = None
    progress("batched workload")
    if world == 1:
        cl = clusters_measure(argparse.Namespace(**{**vars(args), "steps": 10, "warmup": 3}), 0, 1)
        batched = {"value": cl["value"], "unit": "evaluations/s", "e2e": cl["e2e"]["value"],
                   "plain_per_system": cl["plain_per_system"]["value"], "batched_over_plain": cl["batched_over_plain"],
                   "workload": cl["config"]["workload"]}
    pair_ms = float(np.mean(kernel_rows[:, 1]))
    atm_ms = float(np.mean(kernel_rows[:, 2]))
    pairs_per_launch = float(np.mean(kernel_rows[:, 3]))
    triples_per_launch = float(np.mean(kernel_rows[:, 4]))
    achieved = pairs_per_launch * F_PAIR / (pair_ms * 1e-3) / 1e12
    progress("CPU baseline")
    base = cpu_baseline(system, cur, box)
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "atoms": n, "sites": system.getForce(3).getNumSites(),
                   "pairs_per_step": float(np.mean(rows[:, 3])), "triples_per_step": float(np.mean(rows[:, 4])),
                   "ns_per_day": 86400 * dt_ps * 1e-3 / (ms_per_step * 1e-3),
                   "ns_per_day_unconstrained": flex,
                   "l2": "flushed between steps (256 MB write)", "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                     "frac": achieved / peak.value, "traffic": PAIR_TRAFFIC_BYTES,
                     "kernel": "kPairTiles", "kernel_ms": pair_ms, "ops_per_pair": F_PAIR,
                     "peak_source": "measured live: FMA-chain kernel on every SM (ix_measure_fp32_peak)",
                     "timing": "CUDA events around the kernel in a pass of the same steps with the three-body "
                               "chain serialised after the pair chain",
                     "traffic_gbs": PAIR_TRAFFIC_BYTES / (pair_ms * 1e-3) / 1e9,
                     "hardware_ncu": {"fma_pipe_active": PAIR_FMA_PIPE_ACTIVE, "issue_active": PAIR_ISSUE_ACTIVE,
                                      "source": "ncu capture of one MD-step launch (profiles/kPairTiles_24k.md)"},
                     "three_body_kernels_ms": atm_ms, "ops_per_triple": F_TRIPLE,
                     "three_body_achieved": triples_per_launch * F_TRIPLE / (atm_ms * 1e-3) / 1e12},
        "cpu_baseline": base,
        "oracle_error": oracle_error,
        "general_path": general,
        "batched": batched,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": n * 3 * 8,
                "d2h_bytes_per_step": n * 3 * 8 + 4 * 8 + 8},
        "gpu_launches": int(launches1.value - launches0.value),
        "clocks": clocks.summary(),
    }
    print(json.dumps(line))


def run_clusters(args, rank, world):
    line = clusters_measure(args, rank, world)
    if rank == 0:
        print(json.dumps(line))


def clusters_measure(args, rank, world, num_clusters=4096, plain_sample=128):
    """Batched configuration: 4,096 water clusters of 2..32 waters (NoCutoff pair forces, ATM without cutoff), one
    energy+force evaluation of all of them per step through one CUDA graph, against the plain per-system path (one
    Context per cluster, evaluated one after the other) on a sample of the same clusters.  With several GPUs the
    4,096 clusters are partitioned over the ranks by a greedy balance of their work (interaxplugin.partition; no
    collective on the data path) and each rank's energies are gathered on rank 0's host after the timed steps."""
    import torch
    from interaxplugin import BatchContext, Context
    from interaxplugin import partition as PT
    from interaxplugin import workloads as W

    device = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(device)
    sizes = W.cluster_sizes(num_clusters, args.seed)
    shares = PT.assign([PT.cluster_cost(3 * int(w), int(w)) for w in sizes], world)
    mine = shares[rank]
    systems, positions = [], []
    for k in mine:
        s, p = W.cluster_of_set(k, sizes, args.seed)
        systems.append(s)
        positions.append(p)
    batch = BatchContext(systems, device=device)
    L = batch._lib
    pos = np.ascontiguousarray(np.concatenate(positions))
    hpos = torch.from_numpy(pos).pin_memory()
    hfor = torch.empty(pos.shape, dtype=torch.float64).pin_memory()
    hen = torch.empty((len(mine), 4), dtype=torch.float64).pin_memory()
    batch.compute(positions)
    pairs, triples = batch.getCounts()
    dpos = torch.from_numpy(pos).cuda()
    dfor = torch.empty(pos.shape, dtype=torch.float64, device="cuda")
    den = torch.empty((len(mine), 4), dtype=torch.float64, device="cuda")
    stream = torch.cuda.ExternalStream(L.ix_batch_get_stream(batch._batch))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def device_step():
        with torch.cuda.stream(stream):
            flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        batch._check(L.ix_batch_compute_device(batch._batch, ctypes.c_void_p(dpos.data_ptr()),
                                               ctypes.c_void_p(dfor.data_ptr()), ctypes.c_void_p(den.data_ptr())))
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b)

    for _ in range(args.warmup):
        device_step()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(device) as clocks:
        ms = [device_step() for _ in range(args.steps)]
    step_ms = float(np.sum(ms))
    step_ms = rank_max(step_ms, world)
    pairs = int(rank_sum(pairs, world))
    triples = int(rank_sum(triples, world))
    value = num_clusters * args.steps / (step_ms * 1e-3)
    # e2e: host positions in, host forces and energies out, per step
    e2e_t = 0.0
    for k in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        batch._check(L.ix_batch_compute(batch._batch, ctypes.c_void_p(hpos.data_ptr()),
                                        ctypes.c_void_p(hfor.data_ptr()), ctypes.c_void_p(hen.data_ptr())))
        if k >= args.warmup:
            e2e_t += time.perf_counter() - t0
    e2e = num_clusters * args.steps / rank_max(e2e_t, world)
    # the systems' energies gathered on rank 0's host, in cluster order
    gathered = PT.gather(list(hen.numpy().sum(1)), shares, rank, world, PT.host_group(world))
    # the plain per-system drop-in: one Context per cluster, host API, on a sample of the clusters
    ctxs = [Context(systems[k], properties={"DeviceIndex": device}) for k in range(plain_sample)]
    for k, c in enumerate(ctxs):
        c.setPositions(positions[k])
        c.getState()
    t0 = time.perf_counter()
    for rep in range(3):
        for k, c in enumerate(ctxs):
            c.setPositions(positions[k])
            c.getState()
    plain = 3 * plain_sample / (time.perf_counter() - t0)
    if rank != 0:
        return
    line = {
        "metric": "evaluations/s", "value": value, "unit": "evaluations/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{num_clusters} non-periodic water clusters of 2..32 waters in all, all four forces "
                               "(NoCutoff pairs, ATM without cutoff), one batched evaluation per step",
                   "atoms_rank0": int(pos.shape[0]), "pairs_per_step": pairs, "triples_per_step": triples,
                   "l2": "flushed between steps (256 MB write)",
                   "parallelism": f"clusters partitioned over {world} GPUs by work" if world > 1 else "1 GPU"},
        "gathered_systems": len(gathered),
        "plain_per_system": {"value": plain, "unit": "evaluations/s",
                             "sample": f"{plain_sample} of the clusters, one Context each, positions in and "
                                       "forces out per evaluation"},
        "batched_over_plain": e2e / plain,
        "e2e": {"value": e2e, "unit": "evaluations/s", "h2d_bytes_per_step": int(pos.nbytes),
                "d2h_bytes_per_step": int(pos.nbytes + num_clusters * 4 * 8)},
        "interactions_per_s": (pairs + triples) / (step_ms / args.steps * 1e-3),
        "clocks": clocks.summary(),
    }
    return line


def run_lambda(args, rank, world, num_windows=16, num_alchemical=30):
    """Alchemical windows: a 96,000-atom water box (32,000 waters, 9.855 nm, pair cutoff 1.0 nm, ATM on 32,000 sites
    with cutoff 0.8 nm) with 30 waters decoupled by lambda_sterics, evaluated at 16 windows linspace(0, 1, 16) per step
    (energies and forces of every window).  --config lambda has no soft core, so every window is E0 + lambda E1 and
    the 16 windows cost two evaluations plus an interpolation kernel; --config lambda-softcore (R = 0.1 nm) evaluates
    the pair terms once at 0 (where the alchemical pairs contribute nothing), each window's alchemical pairs, and the
    three-body term (linear in lambda) at 0 and 1.  Each counts 16 full
    energy+force evaluations per step.  Compared with the plain path: setParameter + getState
    per window.  With several GPUs the windows are partitioned over the ranks (each rank holds the whole box and
    evaluates its share of the windows; the window energies are gathered on rank 0's host)."""
    import torch
    from interaxplugin import Context, _capi
    from interaxplugin import partition as PT
    from interaxplugin import workloads as W

    softcore = 0.1 if args.config == "lambda-softcore" else 0.0
    device = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(device)
    cfg = W.CONFIGS["96k"]
    system, pos, box = W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=args.seed,
                                   three_body_cutoff=cfg["three_body_cutoff"],
                                   alchemical_waters=range(num_alchemical), softcore_radius=softcore)
    ctx = Context(system, properties={"DeviceIndex": device})
    L = _capi.lib()
    n = system.getNumParticles()
    ctx.setPositions(pos)
    all_values = np.linspace(0.0, 1.0, num_windows)
    shares = PT.assign([1.0] * num_windows, world)
    values = np.ascontiguousarray(all_values[shares[rank]])
    local_windows = len(values)
    energies = np.zeros((local_windows, 4))
    dfor = torch.empty((local_windows, n, 3), dtype=torch.float64, device="cuda")
    stream = torch.cuda.ExternalStream(L.ix_get_stream(ctx._ctx))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    name = b"lambda_sterics"

    def device_step():
        with torch.cuda.stream(stream):
            flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx._check(L.ix_compute_windows_device(ctx._ctx, name, local_windows, _capi.ptr(values),
                                               _capi.ptr(energies), ctypes.c_void_p(dfor.data_ptr())))
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b)

    for _ in range(args.warmup):
        device_step()
    pairs, triples = ctx.getCounts()
    launches0 = ctypes.c_longlong()
    ctx._check(L.ix_get_launch_count(ctx._ctx, ctypes.byref(launches0)))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(device) as clocks:
        ms = [device_step() for _ in range(args.steps)]
    launches1 = ctypes.c_longlong()
    ctx._check(L.ix_get_launch_count(ctx._ctx, ctypes.byref(launches1)))
    step_ms = float(np.sum(ms))
    step_ms = rank_max(step_ms, world)
    value = num_windows * args.steps / (step_ms * 1e-3)
    # e2e: host positions in (pinned), every window's energies and forces out to host memory, per step
    hpos = torch.from_numpy(np.ascontiguousarray(pos)).pin_memory()
    hfor = np.zeros((local_windows, n, 3))
    e2e_t = 0.0
    for k in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx._check(L.ix_set_positions(ctx._ctx, ctypes.c_void_p(hpos.data_ptr()), None))
        ctx._check(L.ix_compute_windows(ctx._ctx, name, local_windows, _capi.ptr(values), _capi.ptr(energies),
                                        _capi.ptr(hfor)))
        if k >= args.warmup:
            e2e_t += time.perf_counter() - t0
    e2e = num_windows * args.steps / rank_max(e2e_t, world)
    window_energies = PT.gather(list(energies.sum(1)), shares, rank, world, PT.host_group(world))
    # the plain path: one setParameter + getState per window
    reps = 2
    ctx.setParameter("lambda_sterics", 0.5)
    ctx.getState()
    t0 = time.perf_counter()
    for _ in range(reps):
        for lam in all_values:
            ctx.setParameter("lambda_sterics", lam)
            ctx.getState()
    plain = reps * num_windows / (time.perf_counter() - t0)
    if rank != 0:
        return
    line = {
        "metric": "evaluations/s", "value": value, "unit": "evaluations/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"96,000-atom water box (32,000 waters, 9.855 nm, cutoff 1.0 nm, ATM on 32,000 sites "
                               f"cutoff 0.8 nm), {num_alchemical} waters alchemical, {num_windows} lambda_sterics "
                               f"windows per step, soft-core radius {softcore} nm",
                   "windows_method": "two evaluations + linear interpolation (exact: no soft core)" if softcore == 0
                   else "pair terms once at 0 plus each window's alchemical pairs (soft core); ATM and LRC from 0 "
                        "and 1, interpolated",
                   "pairs_per_window": pairs, "triples_per_window": triples,
                   "l2": "flushed between steps (256 MB write)",
                   "parallelism": f"windows partitioned over {world} GPUs" if world > 1 else "1 GPU"},
        "gathered_windows": len(window_energies),
        "plain_per_window": {"value": plain, "unit": "evaluations/s",
                             "sample": "setParameter + getState (forces to host) per window"},
        "windows_over_plain": e2e / plain,
        "interactions_per_s": num_windows * (pairs + triples) / (step_ms / args.steps * 1e-3),
        "e2e": {"value": e2e, "unit": "evaluations/s", "h2d_bytes_per_step": int(n * 3 * 8),
                "d2h_bytes_per_step": int(num_windows * (n * 3 + 4) * 8)},
        "gpu_launches": int(launches1.value - launches0.value),
        "clocks": clocks.summary(),
    }
    print(json.dumps(line))


def served_pool(seed, levels=24):
    """Request templates of the served stream: relaxed periodic water boxes of 1,000..20,000 atoms (cutoff 1.0 nm,
    ATM cutoff 0.6 nm, box edge >= 2.15 nm) and water clusters of 50..999 atoms (NoCutoff, ATM without cutoff),
    log-spaced sizes, with 300 K velocities."""
    from interaxplugin import Context
    from interaxplugin import workloads as W
    boxes, clusters = [], []
    for k, w in enumerate(np.unique(np.round(np.geomspace(1000, 20000, levels) / 3).astype(int))):
        system, pos, _ = W.water_box(int(w), W.box_length_for(int(w)), 1.0, seed=seed + k, three_body_cutoff=0.6)
        pos = relax(Context(system), system, pos, iterations=30)
        boxes.append((system, pos, W.initial_velocities(system, 300.0, seed=seed + k)))
    for k, w in enumerate(np.unique(np.round(np.geomspace(50, 999, levels) / 3).astype(int))):
        system, pos, _ = W.water_cluster(int(w), seed=seed + 1000 + k)
        pos = relax(Context(system), system, pos, iterations=30)
        clusters.append((system, pos, W.initial_velocities(system, 300.0, seed=seed + 1000 + k)))
    return boxes, clusters


def run_served(args, rank, world, num_requests=20000, budget=120e9, plain_sample=150):
    """Served stream: 20,000 energy+force requests, sizes log-uniform in 50..20,000 atoms (water boxes from 1,000
    atoms, clusters below), each 1..50 velocity-Verlet steps of 1 fs, through the request server with a 120 GB device
    budget.  Evaluations = initial evaluation + one per step.  Throughput (`value`): the whole stream arriving at once.
    Latency: Poisson arrivals at --rate (below the capacity) for the first --latency-requests requests, from the
    scheduled arrival to the completion seen by the server.  With several GPUs the stream's requests are partitioned
    over the ranks by a greedy balance of their estimated work (interaxplugin.partition), each rank serving its share
    with its own server; throughput is the whole stream over the slowest rank's time."""
    import torch
    from interaxplugin import Context, Server
    from interaxplugin import partition as PT

    device = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(device)
    rng = np.random.default_rng(args.seed)
    boxes, clusters = served_pool(args.seed)
    sizes_b = np.log([s.getNumParticles() for s, _, _ in boxes])
    sizes_c = np.log([s.getNumParticles() for s, _, _ in clusters])
    reqs = []
    for _ in range(num_requests):
        a = math.log(50) + rng.random() * (math.log(20000) - math.log(50))
        if a >= math.log(1000):
            tpl = boxes[int(np.abs(sizes_b - a).argmin())]
        else:
            tpl = clusters[int(np.abs(sizes_c - a).argmin())]
        reqs.append((tpl, int(rng.integers(1, 51))))
    all_requests = len(reqs)
    all_evals = sum(n + 1 for _, n in reqs)
    shares = PT.assign([PT.request_cost(t[0].getNumParticles(), n, t[0] in [b[0] for b in boxes]) for t, n in reqs],
                       world)
    reqs = [reqs[i] for i in shares[rank]]
    num_requests = len(reqs)
    evals = sum(n + 1 for _, n in reqs)
    atoms = sum(t[0].getNumParticles() for t, _ in reqs)
    srv = Server(device=device, budget_bytes=budget, max_running=args.max_running, threads=args.server_threads,
                 window_seconds=args.cohort_window)
    # warm-up: a few requests of each kind (graph captures, pinned staging)
    for tpl in boxes[:2] + clusters[:2]:
        srv.submit(tpl[0], tpl[1], tpl[2], steps=2, dt=0.001)
    srv.run_all()

    def stream(requests, arrivals):
        """Submit `requests` at their arrival times (seconds from now), collect every result; returns the wall
        seconds and the latencies from the scheduled arrivals."""
        lag, done, order = {}, {}, []
        t0 = time.perf_counter()
        for i, ((system, pos, vel), n) in enumerate(requests):
            due = t0 + arrivals[i]
            while time.perf_counter() < due:
                for rid in srv.poll():
                    done[rid] = srv.result(rid)
                if due - time.perf_counter() > 2e-3:
                    time.sleep(1e-3)
            rid = srv.submit(system, pos, vel, steps=n, dt=0.001)
            lag[rid] = time.perf_counter() - due
            order.append(rid)
        while len(done) < len(requests):
            got = srv.wait(60.0)
            if not got:
                raise RuntimeError("served stream timed out")
            for rid in got:
                done[rid] = srv.result(rid)
        wall = time.perf_counter() - t0
        failed = [r for r in done.values() if r.status != 0]
        if failed:
            raise RuntimeError(f"{len(failed)} requests failed: {failed[0].error}")
        return wall, np.array([done[rid].latency + max(lag[rid], 0.0) for rid in order])   # in request order

    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    # throughput: the whole stream at once, the server admitting as memory and slots allow
    with ClockSampler(device) as clocks:
        wall, sat_lat = stream(reqs, np.zeros(num_requests))
    # latency: Poisson arrivals at a rate below the capacity, on the first `latency_requests` of the same stream
    m = min(args.latency_requests, num_requests)
    wall_p, lat = stream(reqs[:m], np.cumsum(rng.exponential(1.0 / args.rate, m)))
    box_ids = {id(b[0]) for b in boxes}
    box_mask = np.array([id(t[0]) in box_ids for t, _ in reqs[:m]])
    stats = srv.stats()
    srv.close()
    wall = rank_max(wall, world)
    value = all_evals / wall
    # the plain per-system path on a sample of the same requests: one Context per request, positions and
    # velocities in, steps, state out
    t_plain, e_plain = 0.0, 0
    for (system, pos, vel), n in reqs[:plain_sample]:
        ta = time.perf_counter()
        ctx = Context(system, properties={"DeviceIndex": device})
        ctx.setPositions(pos)
        ctx.runVelocityVerlet(n, 0.001, vel)
        ctx.getState()
        del ctx
        t_plain += time.perf_counter() - ta
        e_plain += n + 1
    plain = e_plain / t_plain
    if rank != 0:
        return
    line = {
        "metric": "evaluations/s", "value": value, "unit": "evaluations/s", "n_gpus": world, "steps": all_requests,
        "warmup": 4, "ms_per_step": 1000 * wall / all_requests, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"served stream of {all_requests} energy+force requests, sizes log-uniform 50..20,000 "
                               "atoms (periodic water boxes from 1,000 atoms, cutoff 1.0 nm, ATM 0.6 nm; clusters "
                               "below, NoCutoff), 1..50 velocity-Verlet steps of 1 fs each, 120 GB device budget; "
                               "throughput with the whole stream arriving at once; a step = one request",
                   "evaluations": all_evals, "atoms_rank0": atoms, "wall_s": wall,
                   "templates": f"{len(boxes)} box and {len(clusters)} cluster sizes, relaxed",
                   "max_running": args.max_running, "server_threads": args.server_threads,
                   "cohort_window_s": args.cohort_window,
                   "parallelism": f"requests partitioned over {world} GPUs by work" if world > 1 else "1 GPU"},
        "latency_ms": {"arrivals": f"Poisson at {args.rate:g} requests/s, the first {m} requests of the stream",
                       "p50": 1000 * float(np.percentile(lat, 50)), "p99": 1000 * float(np.percentile(lat, 99)),
                       "mean": 1000 * float(lat.mean()), "max": 1000 * float(lat.max()),
                       "requests_per_s": m / wall_p},
        "latency_by_kind_ms": {
            kind: {"requests": int(sel.sum()), "p50": 1000 * float(np.percentile(lat[sel], 50)),
                   "p99": 1000 * float(np.percentile(lat[sel], 99))}
            for kind, sel in (("periodic boxes", box_mask), ("clusters", ~box_mask)) if sel.any()},
        "latency_at_saturation_ms": {"p50": 1000 * float(np.percentile(sat_lat, 50)),
                                     "p99": 1000 * float(np.percentile(sat_lat, 99))},
        "requests_per_s": all_requests / wall,
        "server": {k: stats[k] for k in ("contexts", "cohorts", "peak_reserved_bytes", "peak_arena_bytes",
                                         "worker_seconds")},
        "plain_per_system": {"value": plain, "unit": "evaluations/s",
                             "sample": f"the first {plain_sample} requests, one Context each, sequentially"},
        "served_over_plain": value / world / plain,
        "e2e": {"value": value, "unit": "evaluations/s", "h2d_bytes_per_step": int(48 * atoms / max(num_requests, 1)),
                "d2h_bytes_per_step": int(72 * atoms / max(num_requests, 1) + 32)},
        "clocks": clocks.summary(),
    }
    print(json.dumps(line))


def main():
    args = parse()
    rank, world = dist_init(args)
    try:
        if args.config == "clusters":
            run_clusters(args, rank, world)
        elif args.config in ("lambda", "lambda-softcore"):
            run_lambda(args, rank, world)
        elif args.config == "served":
            run_served(args, rank, world, num_requests=args.requests)
        elif args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world)
        if world > 1:
            # the ranks leave together only when every rank succeeded; a failing rank skips this barrier, and the
            # others' next collective ends with the process group's timeout instead of hiding its traceback
            import torch.distributed as dist
            dist.barrier()
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
