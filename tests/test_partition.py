"""Multi-GPU partition of independent work (interaxplugin.partition) on the host.

* assign(): every item on exactly one rank, the loads balanced to within one item of the ideal, per-rank memory
  budgets honoured, deterministic.
* Two gloo ranks: each evaluates its share of a batch of water clusters (with the FP64 oracle standing in for the GPU
  evaluation, which a CPU host cannot run) and rank 0 gathers them; the merged results equal the one-rank results
  exactly, item by item.
"""
import os
import socket
import subprocess
import sys
import textwrap
from pathlib import Path

import numpy as np
import pytest

from interaxplugin import partition as P

ROOT = Path(__file__).resolve().parents[1]


def test_assign_covers_every_item_once_and_balances():
    rng = np.random.default_rng(0)
    costs = list(rng.lognormal(0.0, 1.5, size=500))
    for world in (1, 2, 3, 8):
        shares = P.assign(costs, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(costs)))
        assert all(s == sorted(s) for s in shares)
        load = P.loads(costs, shares)
        assert max(load) <= sum(costs) / world + max(costs) + 1e-9
        assert shares == P.assign(costs, world)          # deterministic


def test_assign_cluster_costs_of_the_batched_workload():
    from interaxplugin import workloads as W
    sizes = W.cluster_sizes(4096, seed=1)
    costs = [P.cluster_cost(3 * int(w), int(w)) for w in sizes]
    shares = P.assign(costs, 8)
    load = P.loads(costs, shares)
    assert max(load) / min(load) < 1.001                 # many small items: near-perfect balance


def test_assign_honours_memory_budgets():
    costs = [5.0, 4.0, 3.0, 3.0, 1.0]
    memory = [60, 50, 40, 30, 10]
    shares = P.assign(costs, 2, memory=memory, budget=100)
    for s in shares:
        assert sum(memory[i] for i in s) <= 100
    assert sorted(i for s in shares for i in s) == list(range(5))
    with pytest.raises(ValueError, match="fits no rank"):
        P.assign([1.0, 1.0], 2, memory=[10, 200], budget=100)


def test_request_costs_grow_with_size_and_steps():
    assert P.request_cost(3000, 10, True) > P.request_cost(3000, 0, True) > P.request_cost(300, 0, True)
    assert P.request_cost(96, 0, False) == P.cluster_cost(96, 32)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_gather_the_same_results_as_one(tmp_path):
    script = tmp_path / "share.py"
    script.write_text(textwrap.dedent(f"""
        import sys
        for p in ({str(ROOT)!r}, {str(ROOT / "openmm-interax-plugin_b200")!r}, {str(ROOT / "oracle")!r}):
            sys.path.insert(0, p)
        import pickle
        import bench
        import pyoracle
        from interaxplugin import partition as P
        from interaxplugin import workloads as W
        rank, world = bench.dist_init(None)
        sizes = W.cluster_sizes(40, seed=3)
        costs = [P.cluster_cost(3 * int(w), int(w)) for w in sizes]
        shares = P.assign(costs, world)
        systems, positions = W.cluster_set(40, seed=3)
        local = []
        for i in shares[rank]:
            e, f = pyoracle.evaluate(systems[i], positions[i])
            local.append((e, f))
        merged = P.gather(local, shares, rank, world, P.host_group(world))
        if rank == 0:
            with open(sys.argv[1], "wb") as out:
                pickle.dump((shares, merged), out)
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    """))
    out = tmp_path / "merged.pkl"
    port = str(_free_port())
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", MASTER_ADDR="127.0.0.1", MASTER_PORT=port, WORLD_SIZE="2")
    procs = [subprocess.Popen([sys.executable, str(script), str(out)], stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                              text=True, env=dict(env, RANK=str(r), LOCAL_RANK=str(r))) for r in range(2)]
    res = [p.communicate(timeout=300) for p in procs]
    for p, (_, err) in zip(procs, res):
        assert p.returncode == 0, err[-2000:]
    import pickle
    import pyoracle
    from interaxplugin import workloads as W
    shares, merged = pickle.loads(out.read_bytes())
    assert len(shares) == 2 and all(len(s) > 0 for s in shares)
    systems, positions = W.cluster_set(40, seed=3)
    for i in range(40):
        e, f = pyoracle.evaluate(systems[i], positions[i])
        assert merged[i][0] == e and np.array_equal(merged[i][1], f)
