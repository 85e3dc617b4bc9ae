"""Multi-rank path on CPU (gloo, world_size 2): the chain sharding of
pomerol_b200.shard (cost-balanced batches dealt round-robin, partial sums of
first visits, one all-reduce) reproduces the single-rank G2.  The per-batch
evaluator is injected: here the CPU oracle, on GPUs libpgx (bench.py)."""
import os
import socket

import numpy as np
import pytest

from pomerol_b200.shard import ChainShards, evaluate_shard, lpt_batches


def test_batches_cover_every_chain_once_and_balance():
    rng = np.random.default_rng(0)
    for n, nb in ((0, 3), (1, 4), (7, 3), (304, 20)):
        costs = rng.uniform(1, 100, n).tolist()
        b = lpt_batches(costs, nb)
        assert len(b) == nb and sorted(k for x in b for k in x) == list(range(n))
        if n >= 10 * nb:
            load = [sum(costs[k] for k in x) for x in b]
            assert max(load) - min(load) <= max(costs)
    with pytest.raises(ValueError):
        lpt_batches([1.0], 0)


def test_round_robin_schedule_visits_each_batch_once_per_pass():
    for world in (1, 2, 3, 8):
        seen = []
        for r in range(world):
            s = ChainShards([1.0] * 40, 20, r, world)
            seen += [s.batch_of(k) for k in range(-(-20 // world))]
            assert s.own_batches() == list(range(r, 20, world))
        assert sorted(set(seen)) == list(range(20))
    with pytest.raises(ValueError):
        ChainShards([1.0], 1, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _problem():
    from oracle import ed as EDm
    from oracle import lehmann as L
    from oracle import model as M
    beta = 10.0
    m = M.make_model(M.plaquette())
    ed = EDm.ED(m, beta)
    u, d = m.info.getIndex("A", 0, 1), m.info.getIndex("A", 0, 0)
    parts = L.g2_parts(ed, ed.c(u), ed.c(d), ed.cdag(u), ed.cdag(d))
    trip = [(a, b, x) for a in range(-2, 2) for b in range(-2, 2) for x in range(-2, 2)]
    fz = [tuple(L.fermionic(np.array(t), beta)) for t in trip]
    costs = [float(np.prod([len(ed.E[b]) for b in p["b"]])) for p in parts]
    return ed, parts, fz, costs


def _worker(rank, world, port, out_path, steps):
    import torch.distributed as dist

    from oracle import lehmann as L
    from pomerol_b200.shard import allreduce_sum

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ed, parts, fz, costs = _problem()
        shards = ChainShards(costs, 5, rank, world)

        def evaluate(b):
            return L.g2_exact(ed, [parts[k] for k in shards.batches[b]], fz)

        local = evaluate_shard(shards, evaluate, len(fz), steps=steps)
        full = allreduce_sum(local)
        if rank == 0:
            np.save(out_path, full)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("steps", [None, 4])
def test_two_rank_chain_shards_match_single_rank(tmp_path, steps):
    """One pass over each rank's batches, and a timed-style schedule of 4
    steps per rank (8 visits of 5 batches: repeats are not summed twice)."""
    import torch.multiprocessing as mp

    from oracle import lehmann as L

    out = str(tmp_path / "g2.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out, steps), nprocs=2, start_method="spawn")
    got = np.load(out)
    ed, parts, fz, _ = _problem()
    ref = L.g2_exact(ed, parts, fz)
    assert np.abs(got - ref).max() < 1e-12 * np.abs(ref).max()
