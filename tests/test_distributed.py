"""Host logic of the multi-GPU ensemble, run as 2 gloo ranks on the CPU."""
import os

import numpy as np
import torch.multiprocessing as mp

from sph_2_b200 import ic
from sph_2_b200.distributed import local_ensemble, shard_clouds


def test_shard_clouds_balances_and_partitions():
    counts = np.array([500, 20, 300, 300, 90, 10, 250, 40])
    for world in (1, 2, 3, 8):
        owner = shard_clouds(counts, world)
        assert owner.min() >= 0 and owner.max() < world
        load = np.bincount(owner, weights=counts, minlength=world)
        # LPT bound: max load <= mean + largest job
        assert load.max() <= counts.sum() / world + counts.max()
    assert np.array_equal(shard_clouds(counts, 2), shard_clouds(counts, 2))


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from sph_2_b200.distributed import all_sum, shared_dt
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    e = ic.ensemble(n_clouds=6, nmin=200, nmax=2000, seed=3)
    owner = shard_clouds(e["counts"], world)
    mine = local_ensemble(e, owner, rank)
    n_local = len(mine["m"])
    total = all_sum([n_local, len(mine["clouds"])])
    dt = shared_dt([0.01 * (rank + 1), 0.02])
    out[rank] = (tuple(mine["clouds"].tolist()), n_local, tuple(total.tolist()), dt,
                 int(mine["cloud"].max()) + 1 if n_local else 0)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_partition_the_ensemble():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = 29500 + os.getpid() % 1000
        ps = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    e = ic.ensemble(n_clouds=6, nmin=200, nmax=2000, seed=3)
    clouds = sorted(res[0][0] + res[1][0])
    assert clouds == list(range(6))
    assert res[0][1] + res[1][1] == len(e["m"])
    assert res[0][2] == res[1][2] == (len(e["m"]), 6)
    assert res[0][3] == res[1][3] == 0.01
    assert res[0][4] == len(res[0][0]) and res[1][4] == len(res[1][0])
