"""The bench's multi-rank logic on the host, with two gloo ranks (on the GPU box every rank drives one GPU over NCCL;
the rank logic is the same).

* `rank_max` / `rank_sum`: a multi-rank number is timed over the slowest rank and counts the work of every rank.
* The reference arm under torchrun: rank 0 alone runs it and prints one JSON line; the other rank exits 0 without
  work.
"""
import json
import os
import socket
import subprocess
import sys
import textwrap
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _host_env(**extra):
    # no GPU in these processes, so the ranks take gloo
    return dict(os.environ, CUDA_VISIBLE_DEVICES="", MASTER_ADDR="127.0.0.1", **extra)


def test_rank_max_and_sum_over_two_gloo_ranks(tmp_path):
    script = tmp_path / "ranks.py"
    script.write_text(textwrap.dedent(f"""
        import sys
        sys.path.insert(0, {str(ROOT)!r})
        import bench
        import torch.distributed as dist
        rank, world = bench.dist_init(None)
        slowest = bench.rank_max(1.5 + rank, world)
        total = bench.rank_sum(10.0 * (rank + 1), world)
        print(rank, world, dist.get_backend(), slowest, total, flush=True)
        dist.barrier()
        dist.destroy_process_group()
    """))
    port = str(_free_port())
    procs = [subprocess.Popen([sys.executable, str(script)], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                              env=_host_env(RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2", MASTER_PORT=port))
             for r in range(2)]
    outs = [p.communicate(timeout=300) for p in procs]
    for p, (_, err) in zip(procs, outs):
        assert p.returncode == 0, err[-2000:]
    for r, (out, _) in enumerate(outs):
        rank, world, backend, slowest, total = out.split()
        assert (int(rank), int(world), backend) == (r, 2, "gloo")
        assert float(slowest) == 2.5
        assert float(total) == 30.0


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.rank_max(3.25, 1) == 3.25
    assert bench.rank_sum(7.0, 1) == 7.0


def test_reference_arm_prints_once_under_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), str(ROOT / "bench.py"), "--impl", "reference", "--gpus",
           "2", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, env=_host_env(), capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [line for line in r.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["steps"] == 1
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
