"""Partitioning of a batch of independent scenes over the ranks of a job.

pe distributes ONE scene over MPI processes by domain decomposition (src/core/domaindecomp,
MPISystem); its batches of independent simulations are separate runs.  Here every scene is
stepped whole by one GPU, and a batch of scenes is split between the ranks of a
torch.distributed job: each rank advances its own share and no data crosses between ranks
during a step (weak scaling, no data-path collective).
"""
from __future__ import annotations

from typing import List, Optional, Sequence


def shard_scenes(scenes: Sequence, rank: int, world: int) -> List:
    """The scenes rank `rank` of `world` advances: largest first, each onto the rank with the
    fewest spheres so far (ties: the lower rank).  Every scene lands on exactly one rank; the
    order is deterministic, so all ranks compute the same partition without communicating."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    load = [0] * world
    mine = []
    for k in sorted(range(len(scenes)), key=lambda k: (-scenes[k].n, k)):
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += scenes[k].n
        if r == rank:
            mine.append(scenes[k])
    return mine


def local_scenes(scenes: Sequence, group: Optional[object] = None) -> List:
    """shard_scenes for the calling process of an initialised torch.distributed job (all scenes
    when no process group is initialised)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return list(sorted(scenes, key=lambda s: -s.n))
    return shard_scenes(scenes, dist.get_rank(group), dist.get_world_size(group))
