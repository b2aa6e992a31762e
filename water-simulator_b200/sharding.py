"""Spreading independent basins over ranks (one process per GPU).

Basins of an ensemble are independent, so the ensemble shards with no
collective on the data path: each rank advances its own basins.  The
assignment is longest-processing-time first (largest basin onto the least
loaded rank, ties to the lower rank), computed identically on every rank
from the basin sizes alone.  The only collectives are the timing ones:
a barrier around the timed region and the maximum of the ranks' times.

torch.distributed carries those collectives; it is imported only by the
functions that need a process group, so the assignment itself (and the
rest of the package) imports without torch.
"""
import datetime
import os


def assign_basins(cells, world):
    """Basin indices per rank: LPT over `cells` (the work of each basin).
    Every basin appears on exactly one rank; the result depends only on the
    arguments."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(cells)), key=lambda q: (-cells[q], q))
    load = [0] * world
    out = [[] for _ in range(world)]
    for q in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(q)
        load[r] += cells[q]
    for r in range(world):
        out[r].sort()
    return out


def rank_env():
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def _dist():
    import torch.distributed as dist
    return dist


def init_ranks(backend, device=None, timeout_s=120):
    """The process group for a multi-rank run (nothing for one rank).  The
    rendezvous address comes from MASTER_ADDR / MASTER_PORT; the short
    timeout makes ranks that wait on a missing peer fail instead of hang."""
    rank, world, _ = rank_env()
    if world <= 1:
        return False
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if device is not None:
        kw["device_id"] = device
    _dist().init_process_group(backend, **kw)
    return True


def _active():
    dist = _dist()
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def max_over_ranks(value, device=None):
    """The largest of the ranks' values (the job's time is its slowest rank)."""
    if not _active():
        return float(value)
    import torch
    dist = _dist()
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    if _active():
        _dist().barrier()
