"""Frequency-slab sharding of a G2 evaluation across ranks (one GPU each).

Frequency triples are independent and the chains (block quadruples) are
replicated on every rank, so the work splits with no exchange inside the
Lehmann sum: rank r evaluates a contiguous slab of the triple list and, when
the caller needs the whole result, one all-gather assembles it
(the reference's counterpart is the MPI job farm over parts plus
MPI_Allreduce, TwoParticleGF.cpp:171-188).
"""
from __future__ import annotations

import numpy as np


def slab(n_items: int, rank: int, world: int) -> tuple[int, int]:
    """[begin, end) of rank's share: sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n_items, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def gather_slabs(local: np.ndarray, n_items: int, world: int, group=None) -> np.ndarray:
    """All-gather the complex slabs of every rank into the full result
    (torch.distributed; pads to the largest slab)."""
    import torch
    import torch.distributed as dist

    width = max(e - b for b, e in (slab(n_items, r, world) for r in range(world)))
    buf = torch.zeros(width, 2, dtype=torch.float64)
    loc = torch.from_numpy(np.stack([local.real, local.imag], 1))
    buf[: len(local)] = loc
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    buf = buf.to(dev)
    out = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(out, buf, group=group)
    parts = []
    for r in range(world):
        b, e = slab(n_items, r, world)
        t = out[r][: e - b].cpu().numpy()
        parts.append(t[:, 0] + 1j * t[:, 1])
    return np.concatenate(parts)
