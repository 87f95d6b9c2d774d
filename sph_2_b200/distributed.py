"""Multi-GPU use of the step: one process per GPU, no data-path collective.

A single sphere does not shard without a halo exchange and a distributed tree
(SPH needs neighbours across any cut, gravity needs the global tree), so it
runs as replicas.  An ensemble of independent clouds shards naturally: clouds
are assigned to ranks by longest-processing-time order on particle count, each
rank advances its clouds with the same batched launches as on one GPU, and the
only collectives are scalar ones -- the sum of the diagnostics and, when the
ranks must share one time step, a min-reduction of dt.  (The reference's
multi-GPU code gathers every array to GPU 0 and broadcasts it back each phase,
GPU_sph_Type_cooling_II/hfvGpuSph_mgpu_v5.cu:339-568; nothing like that is
needed here.)
"""
from __future__ import annotations

import numpy as np


def shard_clouds(counts, world: int) -> np.ndarray:
    """owner[k] = rank of cloud k, greedy longest-processing-time by size."""
    counts = np.asarray(counts, np.int64)
    owner = np.empty(len(counts), np.int64)
    load = np.zeros(world, np.int64)
    for k in np.argsort(-counts, kind="stable"):
        r = int(np.argmin(load))
        owner[k] = r
        load[r] += counts[k]
    return owner


def local_ensemble(ens: dict, owner: np.ndarray, rank: int) -> dict:
    """The particles of the clouds this rank owns, cloud ids renumbered 0..K-1."""
    mine = np.nonzero(owner == rank)[0]
    remap = -np.ones(len(owner), np.int64)
    remap[mine] = np.arange(len(mine))
    sel = np.isin(ens["cloud"], mine)
    out = {k: v[sel] for k, v in ens.items() if k not in ("counts",)}
    out["cloud"] = remap[ens["cloud"][sel]].astype(np.int32)
    out["counts"] = np.asarray(ens["counts"])[mine]
    out["clouds"] = mine
    return out


def all_sum(values, device=None):
    """Sum a float64 vector over the ranks of the default process group."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(np.asarray(values, np.float64), device=device)
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def shared_dt(local_dt, device=None) -> float:
    """One step for all ranks: the minimum of the ranks' Courant steps."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(np.min(local_dt))], dtype=torch.float64, device=device)
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
    return float(t.item())
