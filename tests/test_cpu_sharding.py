"""Batch sharding over ranks (the multi-GPU layout of independent boxes),
run as two gloo ranks on the CPU: each rank computes its share from the same
inputs, and the shares are disjoint, complete and balanced; the timing
reduction takes the maximum over ranks, and the end-of-run gather collects
per-box scalars in box order."""

import os

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp


def test_shard_is_deterministic_disjoint_and_balanced():
    from sponge_b200 import sharding, systems
    sizes = [systems.batch_member_size(s) for s in range(256)]
    costs = [sharding.box_cost(n, k) for n, k in sizes]
    for world in (1, 2, 3, 4, 8):
        parts = sharding.shard(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        assert parts == sharding.shard(costs, world)
        assert sharding.imbalance(costs, parts) < 1.02


def test_batch_member_size_matches_the_built_box():
    from sponge_b200 import systems
    for seed in (0, 7, 31):
        n, k = systems.batch_member_size(seed)
        b = systems.config_batch_member(seed)
        assert n == b.n
        assert k == systems.fft_size(b.box)


def _rank(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch
    from sponge_b200 import sharding, systems
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sizes = [systems.batch_member_size(s) for s in range(64)]
        costs = [sharding.box_cost(n, k) for n, k in sizes]
        mine = sharding.shard(costs, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        # device-time stand-in: this rank's load; the job time is the max
        t = torch.tensor([sum(costs[i] for i in mine)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        # per-box scalars (e.g. energies) gathered and put back in box order
        vals = {i: float(i) * 0.5 for i in mine}
        allv = [None] * world
        dist.all_gather_object(allv, vals)
        merged = {}
        for d in allv:
            merged.update(d)
        if rank == 0:
            np.save(os.path.join(out_dir, "result.npy"), np.array(
                [sorted(i for p in gathered for i in p) == list(range(64)),
                 len(set(gathered[0]) & set(gathered[1])) == 0,
                 abs(t.item() - max(sum(costs[i] for i in p) for p in gathered)) < 1e-9,
                 [merged[i] for i in range(64)] == [i * 0.5 for i in range(64)]]))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_with_gloo(tmp_path):
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mp.spawn(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    res = np.load(tmp_path / "result.npy")
    assert res.all(), res
