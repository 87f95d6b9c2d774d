"""The ensemble sharded over ranks: two processes on cuda:0, joined by a gloo
process group, each advance the clouds that the longest-processing-time
assignment gives them (no data-path collective), and sum their diagnostics.
Every cloud ends exactly where a single context advancing the whole
ensemble puts it: clouds share no data, and their Morton keys, trees, groups
and sums do not depend on which other clouds share the context (cloud ids
take the keys' top bits; 20 bits per dimension remain for 2 to 8 clouds).
The two ranks only ever run independent kernels, so they never wait on each
other on the GPU."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

CLOUDS, SEED, STEPS = 6, 17, 3
FIELDS = ("x", "y", "z", "vx", "vy", "vz", "u", "h", "rho")


def advance(e, n_cloud):
    """Prologue and STEPS steps of an ensemble in FP64 with per-cloud Courant
    steps; fields in the given order and the energy totals."""
    from sph_2_b200 import Config, Context
    from sph_2_b200 import _lib as L
    n = len(e["m"])
    ctx = Context(Config(n_max=n, n_cloud_max=n_cloud, precision="fp64", theta=0.5,
                         flags=L.FLAG_POTENTIAL))
    ctx.load(e["pos"], e["vel"], e["m"], e["h"], e["u"], cloud=e["cloud"])
    ctx.prologue()
    ctx.step(STEPS)
    ctx.sync()
    out = {f: ctx.get(f) for f in FIELDS}
    out["dt"] = ctx.dt
    en = ctx.energies()
    out["energy"] = np.array([en["KE"], en["U"], en["PE"], en["M"]])
    out["status"] = ctx.status()
    ctx.close()
    return out


def _rank(rank, world, port, path):
    import torch
    import torch.distributed as dist
    from sph_2_b200 import ic
    from sph_2_b200.distributed import all_sum, local_ensemble, shard_clouds
    torch.cuda.set_device(0)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    e = ic.ensemble(n_clouds=CLOUDS, nmin=3000, nmax=12000, seed=SEED)
    owner = shard_clouds(e["counts"], world)
    mine = local_ensemble(e, owner, rank)
    r = advance(mine, len(mine["counts"]))
    tot = all_sum(r["energy"])
    np.savez(os.path.join(path, f"rank{rank}.npz"), clouds=mine["clouds"], total=tot,
             **{f: r[f] for f in FIELDS + ("dt",)},
             bad=np.array([r["status"]["h_noconv"], r["status"]["ngb_overflow"],
                           r["status"]["stack_overflow"]]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_advance_their_shards_like_one_context(tmp_path):
    from sph_2_b200 import ic
    from sph_2_b200.distributed import shard_clouds
    ctx = mp.get_context("spawn")
    port = 29600 + os.getpid() % 1000
    ps = [ctx.Process(target=_rank, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(300)
        assert p.exitcode == 0
    e = ic.ensemble(n_clouds=CLOUDS, nmin=3000, nmax=12000, seed=SEED)
    whole = advance(e, CLOUDS)
    owner = shard_clouds(e["counts"], 2)
    assert set(owner.tolist()) == {0, 1}
    totals = []
    for rank in range(2):
        r = dict(np.load(tmp_path / f"rank{rank}.npz"))
        assert not r["bad"].any()
        totals.append(r["total"])
        sel = np.isin(e["cloud"], r["clouds"])
        for f in FIELDS:
            a, b = r[f], whole[f][sel]
            assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b)), f
        assert np.allclose(r["dt"], whole["dt"][r["clouds"]], rtol=1e-12, atol=0)
    # the summed diagnostics are the whole ensemble's
    assert np.array_equal(totals[0], totals[1])
    assert np.allclose(totals[0], whole["energy"], rtol=1e-12, atol=0)
