"""Spreading independent work over the GPUs of one node: whole systems of a batch, requests of a served stream and
windows of a lambda scan are assigned to ranks (one process per GPU) by a greedy balance of estimated work under a
per-rank device-memory budget; each rank evaluates its share on its own GPU and the results are gathered on the host
of rank 0.  Nothing is exchanged between the GPUs: the only traffic is the gather of finished results over the
process group's host transport.

The reference evaluates one System per Context on one device (platforms/cuda/src/CudaInteraxKernelFactory.cpp:75
takes the context's first device); this is the multi-GPU form of its batched and served workloads.
"""
import heapq
from math import comb

# Operations per interacting pair and per interacting triple of the reference's FP64 terms, fixed by counting the
# oracle's operations over the 24,000-atom water box (the same figures as the bench's roofline).
F_PAIR = 612.4
F_TRIPLE = 151.0


def cluster_cost(num_particles, num_sites):
    """Estimated work of one evaluation of a cluster with no cutoff: every pair and every triple of sites."""
    return F_PAIR * comb(num_particles, 2) + F_TRIPLE * comb(num_sites, 3)


def request_cost(num_particles, steps, periodic, pairs_per_particle=210.0, triples_per_site=57.0):
    """Estimated work of a served request: (steps + 1) evaluations; a periodic box costs about pairs_per_particle
    pairs per particle and triples_per_site triples per water site (the 24,000-atom box's figures at cutoffs 1.0 and
    0.6 nm), a cluster every pair and triple."""
    evaluations = steps + 1
    if periodic:
        per = F_PAIR * pairs_per_particle * num_particles + F_TRIPLE * triples_per_site * num_particles / 3.0
        return evaluations * per
    return evaluations * cluster_cost(num_particles, num_particles // 3)


def assign(costs, world, memory=None, budget=None):
    """Greedy balance of independent items over `world` ranks: the items in decreasing cost, each to the rank with the
    least work so far (ties to the lower rank) among those whose memory still has room (`memory[i]` bytes against
    `budget` bytes per rank; both None = no memory limit).  Deterministic.  Returns one list of item indices per
    rank, each in increasing order.  Raises ValueError when an item fits no rank."""
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    work = [(0.0, r) for r in range(world)]
    used = [0.0] * world
    share = [[] for _ in range(world)]
    heapq.heapify(work)
    for i in order:
        need = 0.0 if memory is None else float(memory[i])
        skipped = []
        while work:
            load, r = heapq.heappop(work)
            if budget is None or used[r] + need <= budget:
                share[r].append(i)
                used[r] += need
                heapq.heappush(work, (load + float(costs[i]), r))
                break
            skipped.append((load, r))
        else:
            raise ValueError(f"item {i} ({need:.0f} bytes) fits no rank's memory budget")
        for entry in skipped:
            heapq.heappush(work, entry)
    return [sorted(s) for s in share]


def loads(costs, shares):
    """Work assigned to each rank."""
    return [sum(costs[i] for i in s) for s in shares]


def gather(local, shares, rank, world, group=None):
    """Merge per-rank results into item order on rank 0: `local` holds this rank's results in the order of
    shares[rank].  Returns the full list on rank 0 and None elsewhere.  With world = 1 nothing is communicated.  The
    results travel as host objects over `group` (a gloo group, so the GPUs take no part)."""
    if world == 1:
        return list(local)
    import torch.distributed as dist
    parts = [None] * world if rank == 0 else None
    dist.gather_object(list(local), parts, dst=0, group=group)
    if rank != 0:
        return None
    total = sum(len(s) for s in shares)
    out = [None] * total
    for r in range(world):
        if len(parts[r]) != len(shares[r]):
            raise RuntimeError(f"rank {r} returned {len(parts[r])} results for {len(shares[r])} items")
        for i, value in zip(shares[r], parts[r]):
            out[i] = value
    return out


def host_group(world):
    """A gloo process group over every rank for the host gathers (None when there is one rank)."""
    if world == 1:
        return None
    import torch.distributed as dist
    return dist.new_group(backend="gloo")
