"""Host logic of multi-GPU replica runs, as world_size-2 gloo process groups on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from zoomy_amrex_b200.replicas import shard, shard_by_cells


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world_size, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world_size),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    from zoomy_amrex_b200 import replicas
    from zoomy_amrex_b200.workloads import dam_break_ensemble
    ws, r, _ = replicas.init("gloo", timeout_s=30)
    ens = dam_break_ensemble(10, seed=3)
    cells = [c.nx * c.ny for c, _, _ in ens]
    mine = replicas.shard_by_cells(cells, ws)[r]
    my_cells = sum(cells[k] for k in mine)
    t = 1.5 + r            # stand-in for this rank's device time
    replicas.barrier()
    out[r] = (replicas.max_over_ranks(t), replicas.sum_over_ranks(my_cells), mine, sum(cells))
    replicas.finish()


def test_replica_reductions_gloo():
    ws = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(ws, _free_port(), out), nprocs=ws, join=True)
    res = [out[r] for r in range(ws)]
    for tmax, total, _, all_cells in res:
        assert tmax == 2.5                     # the slowest rank's time
        assert total == all_cells              # every cell on exactly one rank
    assert sorted(res[0][2] + res[1][2]) == list(range(10))


def test_shard_helpers():
    assert shard(list(range(7)), 0, 3) == [0, 1, 2]
    assert shard(list(range(7)), 2, 3) == [5, 6]
    parts = shard_by_cells([100, 90, 10, 10, 5], 2)
    loads = [sum([100, 90, 10, 10, 5][k] for k in p) for p in parts]
    assert sorted(sum(parts, [])) == [0, 1, 2, 3, 4]
    assert max(loads) - min(loads) <= 15
