"""Sharding one G2 grid over ranks (one GPU each) by block chains.

The G2 of a component is a sum over its block chains (parts), each evaluated
on the whole frequency grid.  The chains are cut into `nbatch` batches of
about equal cost (largest first, each to the lightest batch), and step k of
rank r evaluates batch (k * world + r) mod nbatch.  Batch b belongs to rank
b mod world; a rank adds the values of the batches it owns, once each, to its
partial sum (after the scheduled steps it evaluates those of its batches that
no step reached), and one all-reduce (sum) over the ranks assembles the full
G2 -- the reference farms
parts over MPI ranks and sums the frequency values with MPI_Allreduce
(TwoParticleGF.cpp:171-188).  Sharding the frequencies instead would repeat
the per-frequency anchored products of every chain on every rank, since each
rank would need all values of z1 and z3 of its slab's triples.
"""
from __future__ import annotations

import numpy as np


def lpt_batches(costs, nbatch):
    """Chain indices split into nbatch lists of about equal total cost:
    largest first, each to the list with the least cost so far.  Lists keep
    the chains' order; a list may be empty when there are fewer chains."""
    if nbatch < 1:
        raise ValueError("nbatch must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    load = [0.0] * nbatch
    out = [[] for _ in range(nbatch)]
    for k in order:
        b = min(range(nbatch), key=lambda i: (load[i], i))
        out[b].append(k)
        load[b] += costs[k]
    return [sorted(b) for b in out]


class ChainShards:
    """Batches of chains dealt round-robin to the ranks of a job."""

    def __init__(self, costs, nbatch, rank=0, world=1):
        if world < 1 or not 0 <= rank < world:
            raise ValueError("bad rank/world")
        self.batches = lpt_batches(costs, nbatch)
        self.rank, self.world = rank, world
        self.done = set()

    def batch_of(self, step):
        """Batch that this rank evaluates at step `step`."""
        return (step * self.world + self.rank) % len(self.batches)

    def owns(self, batch):
        """Batch b belongs to rank b mod world: only its owner sums it."""
        return batch % self.world == self.rank

    def first_visit(self, batch):
        """True the first time this rank evaluates a batch it owns (its values
        then go into the partial sum; other visits only repeat work)."""
        if not self.owns(batch) or batch in self.done:
            return False
        self.done.add(batch)
        return True

    def own_batches(self):
        """Every batch this rank owns in one pass over the grid."""
        return list(range(self.rank, len(self.batches), self.world))


def allreduce_sum(local: np.ndarray, group=None) -> np.ndarray:
    """Sum of the ranks' complex partial results (torch.distributed: NCCL on
    GPUs, gloo on CPUs)."""
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(np.ascontiguousarray(local, dtype=complex).view(np.float64).copy()).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy().view(complex)


def evaluate_shard(shards: ChainShards, evaluate, nfreq, steps=None):
    """Run this rank's batches: `evaluate(batch_index)` returns the batch's
    values on the grid.  `steps` steps of the round-robin schedule (none with
    steps=None), then the rank's own batches that no step reached.  Returns
    the partial sum over the batches this rank owns, each once."""
    acc = np.zeros(nfreq, dtype=complex)
    plan = [] if steps is None else [shards.batch_of(k) for k in range(steps)]
    for b in plan:
        v = evaluate(b)
        if shards.first_visit(b):
            acc += v
    for b in shards.own_batches():
        if b not in shards.done:
            acc += evaluate(b)
            shards.done.add(b)
    return acc
