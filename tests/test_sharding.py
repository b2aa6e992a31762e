"""The multi-rank plumbing on CPU: the basin assignment (longest first onto
the least loaded rank) and, with two `gloo` ranks in child processes, that
every rank computes the same assignment, that the basins split with none
shared, and that the job's time is the maximum over the ranks."""
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _sharding():
    sys.path.insert(0, ROOT)
    import __graft_entry__
    __graft_entry__.load_package()
    from water_simulator_b200 import sharding
    return sharding


def test_assignment_covers_every_basin_once():
    sh = _sharding()
    from water_simulator_b200 import workloads
    cells = [b["nx"] * b["ny"] for b in workloads.ensemble()]
    for world in (1, 2, 3, 4, 8):
        parts = sh.assign_basins(cells, world)
        flat = sorted(q for p in parts for q in p)
        assert flat == list(range(len(cells)))
        loads = [sum(cells[q] for q in p) for p in parts]
        # LPT: no rank exceeds the lightest by more than the largest basin
        assert max(loads) - min(loads) <= max(cells)
        assert parts == sh.assign_basins(cells, world)          # deterministic


def test_assignment_small_cases():
    sh = _sharding()
    assert sh.assign_basins([5, 4, 3, 3], 2) == [[0, 3], [1, 2]]
    assert sh.assign_basins([1, 1, 1], 4) == [[0], [1], [2], []]
    with pytest.raises(ValueError):
        sh.assign_basins([1], 0)


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sh = _sharding()
    import torch.distributed as dist
    assert sh.init_ranks("gloo", timeout_s=60)
    cells = [37, 5, 90, 12, 64, 64, 3, 41]
    mine = sh.assign_basins(cells, world)[rank]
    every = [None] * world
    dist.all_gather_object(every, sh.assign_basins(cells, world))
    sh.barrier()
    t = sh.max_over_ranks(1.5 + rank)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"mine": mine, "every": every, "tmax": t}, f)
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_gloo_ranks(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert res[0]["every"][0] == res[0]["every"][1] == res[1]["every"][0]
    assert set(res[0]["mine"]).isdisjoint(res[1]["mine"])
    assert sorted(res[0]["mine"] + res[1]["mine"]) == list(range(8))
    assert res[0]["tmax"] == res[1]["tmax"] == 2.5
