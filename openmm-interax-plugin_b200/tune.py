"""Autotuner of the kernels' tile and schedule constants (the IX_TUNE_* macros of csrc/ix_tuning.h).

Run on the GPU:  python openmm-interax-plugin_b200/tune.py [--out tuning.json] [--steps 200]

Each candidate set of values is compiled into its own copy of the library (in parallel, with nvcc), and timed in a
fresh process that loads that copy (IX_B200_LIBRARY) on the benchmark's shapes:

* the 24,000-atom rigid-water box with the three-body term: the mean velocity-Verlet step time over `--steps` steps
  (list rebuilds included, so the pair skin's trade-off between candidate pairs and rebuild frequency is measured),
  and the pair kernel's and the three-body kernels' own times (CUDA events, the chains serialised);
* the 4,096 water clusters of the batched workload: the time of one batched evaluation.

A candidate counts only if it computes what the shipped build computes.  Before the search, the shipped (in-tree)
library relaxes the box once and records its energy and forces at that frame, and the clusters' batched energies and
forces, in a fresh process of its own.  Each candidate evaluates the same frame and clusters, and its results must
agree with the recorded ones to within half the accuracy bar (1e-6 relative energy, 1e-5 relative RMS force) that the
tests hold the shipped build to against the FP64 oracle; every candidate's MD run then starts from that frame.

The search is coordinate-wise: starting from the current values, each group of constants is varied over its
candidates with the others fixed, and the best by the objective (the MD step time, plus the batched evaluation time
for the groups that change it) is kept before the next group if it beats the current values by more than MARGIN (the
spread of repeated measurements of one build; a smaller gain is noise).  The chosen values and every measurement are
written to tuning.json, which the build (build_lib.py) turns into compiler definitions.  `--reselect FILE` applies the
selection again to the measurements recorded in FILE (no GPU).
"""
import argparse
import concurrent.futures
import hashlib
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

PKG = Path(__file__).resolve().parent
sys.path.insert(0, str(PKG))
import build_lib  # noqa: E402

DEFAULTS = {"IX_TUNE_PAIR_WARPS": 4, "IX_TUNE_PAIR_ROUND": 128, "IX_TUNE_PAIR_MIN_BLOCKS": 8,
            "IX_TUNE_PAIR_COLUMN_LISTS": 0, "IX_TUNE_PAIR_COLUMN_TRANSPOSE": 0, "IX_TUNE_PAIR_ILP": 0,
            "IX_TUNE_PAIR_SHARED_TABLE_BYTES": 0,
            "IX_TUNE_PAIR_MAX_CLASSES": 16,
            "IX_TUNE_PAIR_SKIN": 0.1,
            "IX_TUNE_SITE_SKIN": 0.1, "IX_TUNE_ATM_FAST": 64, "IX_TUNE_ATM_ROUND": 64, "IX_TUNE_ATM_MIN_BLOCKS": 7,
            "IX_TUNE_ATM_ACCUM": 0}

# groups of constants searched together, each with its candidate values (dicts of the group's macros)
GROUPS = [
    ("pair tiles", [dict(IX_TUNE_PAIR_WARPS=w, IX_TUNE_PAIR_ROUND=r, IX_TUNE_PAIR_MIN_BLOCKS=b,
                         IX_TUNE_PAIR_COLUMN_LISTS=c, IX_TUNE_PAIR_ILP=i)
                    for w, r, b, c, i in ((4, 128, 8, 0, 0), (4, 64, 8, 0, 0), (4, 256, 6, 0, 0), (2, 128, 16, 0, 0),
                                          (4, 128, 6, 1, 0), (4, 128, 5, 0, 1), (4, 128, 6, 0, 1), (4, 64, 5, 0, 1),
                                          (2, 128, 10, 0, 1), (4, 256, 4, 0, 1))]),
    ("pair table", [dict(IX_TUNE_PAIR_SHARED_TABLE_BYTES=b) for b in (0, 1024, 2048)]),
    ("pair columns", [dict(IX_TUNE_PAIR_COLUMN_TRANSPOSE=v) for v in (0, 1)]),
    ("pair skin", [dict(IX_TUNE_PAIR_SKIN=s) for s in (0.06, 0.08, 0.1, 0.12)]),
    ("three-body", [dict(IX_TUNE_ATM_FAST=f, IX_TUNE_ATM_ROUND=r, IX_TUNE_ATM_MIN_BLOCKS=b, IX_TUNE_ATM_ACCUM=acc)
                    for f, r, b, acc in ((64, 64, 7, 0), (64, 64, 8, 0), (64, 64, 10, 0), (32, 32, 12, 0),
                                         (64, 32, 8, 0), (64, 128, 7, 0), (64, 128, 8, 0), (64, 256, 5, 0),
                                         (64, 128, 7, 1))]),
    ("site skin", [dict(IX_TUNE_SITE_SKIN=s) for s in (0.05, 0.1, 0.15)]),
]


def _key(values):
    return hashlib.sha1(json.dumps(sorted(values.items())).encode()).hexdigest()[:12]


def compile_candidates(candidates, workdir, jobs=4):
    """Compile each candidate (a full dict of values) into workdir; returns {key: path}."""
    out = {}
    Path(workdir).mkdir(parents=True, exist_ok=True)

    def one(values):
        path = Path(workdir) / f"libinterax_b200_{_key(values)}.so"
        if not path.exists():
            build_lib.compile_library(path, values)
        return _key(values), path

    with concurrent.futures.ThreadPoolExecutor(jobs) as pool:
        for key, path in pool.map(one, candidates):
            out[key] = path
    return out


# a candidate's energy (relative) and forces (relative RMS) against the shipped build's: half the accuracy bar, so
# that a candidate within it stays within the bar against the FP64 oracle too
AGREEMENT_ENERGY = 5e-7
AGREEMENT_FORCE = 5e-6


def _box_system():
    from interaxplugin import workloads as W
    cfg = W.CONFIGS["24k"]
    return W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=1,
                       three_body_cutoff=cfg["three_body_cutoff"], rigid=True)


def force_error(f, ref):
    """Relative RMS difference of two force arrays."""
    import numpy as np
    f, ref = np.asarray(f, dtype=np.float64), np.asarray(ref, dtype=np.float64)
    return float(np.sqrt(((f - ref) ** 2).mean() / (ref ** 2).mean()))


def batch_energy_error(energies, ref):
    """The largest difference of a cluster's total energy, relative to the sum of its terms' magnitudes (a cluster's
    terms can cancel to a small total)."""
    import numpy as np
    energies, ref = np.asarray(energies, dtype=np.float64), np.asarray(ref, dtype=np.float64)
    scale = np.maximum(np.abs(ref).sum(1), 1e-300)
    return float((np.abs(energies.sum(1) - ref.sum(1)) / scale).max())


def reference_frame(path):
    """With the library this process loads (the shipped in-tree build): relax the 24k box once and record the frame
    with its energy and forces, and the 4,096 clusters' batched energies and forces, in `path` (.npz)."""
    import numpy as np

    sys.path.insert(0, str(PKG.parent))
    import bench  # the benchmark's relaxation
    from interaxplugin import BatchContext, Context
    from interaxplugin import workloads as W

    system, pos, _ = _box_system()
    ctx = Context(system)
    pos = bench.relax(ctx, system, pos, iterations=30)
    st = ctx.getState()
    systems, positions = W.cluster_set(4096, seed=1)
    energies, forces = BatchContext(systems).compute(positions)
    np.savez(path, pos=pos, energy=st.getPotentialEnergy(), forces=st.getForces(), batch_energies=energies,
             batch_forces=np.concatenate(forces))


def measure(steps, frame, clusters=True):
    """Agreement with the shipped build at the recorded frame (`frame`, from reference_frame) and timings of the
    library named by IX_B200_LIBRARY (run in a fresh process)."""
    import ctypes

    import numpy as np
    import torch

    from interaxplugin import BatchContext, Context, _capi
    from interaxplugin import workloads as W

    ref = np.load(frame)
    system, _, _ = _box_system()
    ctx = Context(system)
    L = _capi.lib()
    pos = ref["pos"]
    ctx.setPositions(pos)
    st = ctx.getState()
    err_e = abs(st.getPotentialEnergy() - float(ref["energy"])) / abs(float(ref["energy"]))
    err_f = force_error(st.getForces(), ref["forces"])
    vel = np.ascontiguousarray(W.initial_velocities(system, 300.0, seed=0))
    masses = np.array([system.getParticleMass(i) for i in range(system.getNumParticles())])
    ctx._check(L.ix_md_set_masses(ctx._ctx, _capi.ptr(masses)))
    ctx._check(L.ix_md_run(ctx._ctx, 20, 0.001, None, _capi.ptr(vel), None))
    stream = torch.cuda.ExternalStream(L.ix_get_stream(ctx._ctx))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    ctx._check(L.ix_md_steps_async(ctx._ctx, steps, 0.001))
    b.record(stream)
    ctx._check(L.ix_md_finish(ctx._ctx, None, None, None))
    step_ms = a.elapsed_time(b) / steps
    # the kernels alone: the three-body chain after the pair chain, events around each
    ctx._check(L.ix_set_profiling(ctx._ctx, 2))
    pair, atm = [], []
    for _ in range(30):
        ctx._check(L.ix_md_steps_async(ctx._ctx, 1, 0.001))
        ctx._check(L.ix_md_finish(ctx._ctx, None, None, None))
        p, t = ctypes.c_double(), ctypes.c_double()
        ctx._check(L.ix_get_kernel_times(ctx._ctx, ctypes.byref(p), ctypes.byref(t)))
        pair.append(p.value)
        atm.append(t.value)
    out = {"md_step_ms": step_ms, "pair_kernel_ms": float(np.median(pair)), "three_body_ms": float(np.median(atm)),
           "energy_error": err_e, "force_error": err_f}
    if clusters:
        systems, positions = W.cluster_set(4096, seed=1)
        batch = BatchContext(systems)
        energies, forces = batch.compute(positions)
        out["clusters_energy_error"] = batch_energy_error(energies, ref["batch_energies"])
        out["clusters_force_error"] = force_error(np.concatenate(forces), ref["batch_forces"])
        dpos = torch.from_numpy(np.ascontiguousarray(np.concatenate(positions))).cuda()
        dfor = torch.empty_like(dpos)
        den = torch.empty((4096, 4), dtype=torch.float64, device="cuda")
        bstream = torch.cuda.ExternalStream(L.ix_batch_get_stream(batch._batch))
        times = []
        for k in range(13):
            torch.cuda.synchronize()
            a.record(bstream)
            batch._check(L.ix_batch_compute_device(batch._batch, ctypes.c_void_p(dpos.data_ptr()),
                                                   ctypes.c_void_p(dfor.data_ptr()), ctypes.c_void_p(den.data_ptr())))
            b.record(bstream)
            b.synchronize()
            if k >= 3:
                times.append(a.elapsed_time(b))
        out["clusters_ms"] = float(np.median(times))
    return out


def record_reference_frame(path):
    """reference_frame(path) in a fresh process with the in-tree library (no IX_B200_LIBRARY)."""
    env = {k: v for k, v in os.environ.items() if k != "IX_B200_LIBRARY"}
    cmd = [sys.executable, str(Path(__file__).resolve()), "--reference-frame", str(path)]
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        raise RuntimeError("recording the shipped build's reference frame failed:\n" + r.stderr[-2000:])


def run_candidate(path, steps, frame, clusters):
    env = dict(os.environ, IX_B200_LIBRARY=str(path))
    cmd = [sys.executable, str(Path(__file__).resolve()), "--measure", "--steps", str(steps), "--frame", str(frame)]
    if not clusters:
        cmd.append("--no-clusters")
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        return {"error": r.stderr[-2000:]}
    return json.loads(r.stdout.strip().splitlines()[-1])


# a candidate must beat the group's current values by this fraction of the objective to replace them
MARGIN = 0.01


def agrees(m):
    """Whether a measurement's results meet the bar: agreement with the shipped build (energy_error, force_error and,
    with the clusters, clusters_*), or, in measurements recorded by an earlier form of the tuner, the error against
    the FP64 oracle (oracle_*, against the full bar)."""
    if "oracle_energy_error" in m:
        return m["oracle_energy_error"] <= 1e-6 and m["oracle_force_error"] <= 1e-5
    ok = m["energy_error"] <= AGREEMENT_ENERGY and m["force_error"] <= AGREEMENT_FORCE
    if "clusters_energy_error" in m:
        ok = ok and m["clusters_energy_error"] <= AGREEMENT_ENERGY and m["clusters_force_error"] <= AGREEMENT_FORCE
    return ok


def objective(m, with_clusters):
    if "error" in m or not agrees(m):
        return float("inf")
    return m["md_step_ms"] + (m["clusters_ms"] if with_clusters else 0.0)


def select(results, current, margin=MARGIN):
    """The values kept after a group: `results` holds (objective, values) per candidate, one of them `current`."""
    best = min(results, key=lambda r: r[0])
    base = [r[0] for r in results if r[1] == current]
    if base and not best[0] < (1.0 - margin) * base[0]:
        return dict(current)
    return dict(best[1])


def reselect(path):
    """Apply select() again to the measurements recorded in a tuning.json, group by group, and rewrite its choice."""
    data = json.loads(Path(path).read_text())
    current = dict(DEFAULTS)
    groups = []
    for entry in data["measurements"]:
        if not groups or groups[-1][0] != entry["group"]:
            groups.append((entry["group"], []))
        groups[-1][1].append(entry)
    for name, entries in groups:
        clusters = "clusters_ms" in entries[0]["measured"]
        results = [(objective(e["measured"], clusters), dict(current, **e["values"])) for e in entries]
        current = select(results, current)
    data["chosen"] = current
    data["selection"] = f"best of each group if it beats the current values by more than {MARGIN:.0%}"
    Path(path).write_text(json.dumps(data, indent=1) + "\n")
    return current


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--out", default=str(build_lib.TUNING))
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--measure", action="store_true", help=argparse.SUPPRESS)
    p.add_argument("--frame", help=argparse.SUPPRESS)
    p.add_argument("--reference-frame", metavar="NPZ", help=argparse.SUPPRESS)
    p.add_argument("--no-clusters", action="store_true", help=argparse.SUPPRESS)
    p.add_argument("--reselect", metavar="FILE")
    p.add_argument("--groups", help="comma-separated names of the groups to search (default: all)")
    args = p.parse_args()
    if args.reselect:
        print("chosen", reselect(args.reselect))
        return
    if args.reference_frame:
        reference_frame(args.reference_frame)
        return
    if args.measure:
        print(json.dumps(measure(args.steps, args.frame, clusters=not args.no_clusters)))
        return
    import torch
    current = dict(DEFAULTS)
    current.update(build_lib.tuned_values())
    record = []
    workdir = tempfile.mkdtemp(prefix="ix_tune_")
    t0 = time.time()
    frame = Path(workdir) / "reference_frame.npz"
    record_reference_frame(frame)
    groups = GROUPS if not args.groups else [g for g in GROUPS if g[0] in args.groups.split(",")]
    for name, options in groups:
        # the batched workload has no pair list and no site lists to rebuild: the skins do not change it
        clusters = name not in ("pair skin", "site skin", "pair table")
        candidates = [dict(current, **o) for o in options]
        libs = compile_candidates(candidates, workdir)
        results = []
        for values in candidates:
            m = run_candidate(libs[_key(values)], args.steps, frame, clusters)
            results.append((objective(m, clusters), values))
            record.append({"group": name, "values": {k: values[k] for k in options[0]}, "measured": m})
            print(name, {k: values[k] for k in options[0]}, m, flush=True)
        current = select(results, current)
    out = {"chosen": current, "device": torch.cuda.get_device_name(0), "steps": args.steps,
           "objective": "mean velocity-Verlet step of the 24,000-atom rigid-water box (ms), plus one batched "
                        "evaluation of the 4,096 clusters (ms) for the groups that change it",
           "selection": f"best of each group if it beats the current values by more than {MARGIN:.0%}",
           "command": "python openmm-interax-plugin_b200/tune.py", "seconds": time.time() - t0,
           "measurements": record}
    Path(args.out).write_text(json.dumps(out, indent=1) + "\n")
    print("chosen", current)


if __name__ == "__main__":
    main()
