"""Multi-rank path on CPU (gloo, world_size 2): frequency slabs evaluated on
separate ranks and all-gathered equal the single-rank evaluation.  The
per-slab evaluation here is the CPU oracle; on GPUs each rank runs libpgx on
its slab (bench.py --gpus N)."""
import os
import socket

import numpy as np
import pytest

from pomerol_b200.shard import slab


def test_slab_partition_covers_everything_once():
    for n in (0, 1, 7, 4096, 13824):
        for world in (1, 2, 3, 8):
            edges = [slab(n, r, world) for r in range(world)]
            assert edges[0][0] == 0 and edges[-1][1] == n
            assert all(edges[r][1] == edges[r + 1][0] for r in range(world - 1))
            sizes = [e - b for b, e in edges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        slab(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path):
    import torch.distributed as dist

    from oracle import ed as EDm
    from oracle import lehmann as L
    from oracle import model as M
    from pomerol_b200.shard import gather_slabs

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        beta = 10.0
        m = M.make_model(M.plaquette())
        ed = EDm.ED(m, beta)
        u, d = m.info.getIndex("A", 0, 1), m.info.getIndex("A", 0, 0)
        parts = L.g2_parts(ed, ed.c(u), ed.c(d), ed.cdag(u), ed.cdag(d))
        trip = [(a, b, x) for a in range(-2, 2) for b in range(-2, 2) for x in range(-2, 2)]
        fz = [tuple(L.fermionic(np.array(t), beta)) for t in trip]
        b, e = slab(len(fz), rank, world)
        local = L.g2_exact(ed, parts, fz[b:e])
        full = gather_slabs(local, len(fz), world)
        if rank == 0:
            np.save(out_path, full)
    finally:
        dist.destroy_process_group()


def test_two_rank_slabs_match_single_rank(tmp_path):
    import torch.multiprocessing as mp

    from oracle import ed as EDm
    from oracle import lehmann as L
    from oracle import model as M

    out = str(tmp_path / "g2.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    got = np.load(out)
    beta = 10.0
    m = M.make_model(M.plaquette())
    ed = EDm.ED(m, beta)
    u, d = m.info.getIndex("A", 0, 1), m.info.getIndex("A", 0, 0)
    parts = L.g2_parts(ed, ed.c(u), ed.c(d), ed.cdag(u), ed.cdag(d))
    trip = [(a, b, x) for a in range(-2, 2) for b in range(-2, 2) for x in range(-2, 2)]
    ref = L.g2_exact(ed, parts, [tuple(L.fermionic(np.array(t), beta)) for t in trip])
    assert np.abs(got - ref).max() < 1e-12 * np.abs(ref).max()
