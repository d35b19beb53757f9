"""The multi-process plumbing of bench.py on CPU: two ranks over torch.distributed's gloo backend,
rendezvous on 127.0.0.1.

The single solve runs as independent replicas (one per GPU, no collective on the data path) and the
batched workload shards by case; the only collectives are the timing reductions. This checks them
with world size 2: the max and the sum over ranks, and that the case sharding gives every case to
exactly one rank with the cells balanced.
"""
import json
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), LOCAL_RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, REPO)
    import bench
    from brae_b200 import cases
    w, r, _ = bench.dist_setup("gloo")
    assert (w, r) == (world, rank)
    cells = [d["n"][0] * d["n"][1] * d["n"][2] for d in cases.mixed_batch_sizes(64)]
    res = {
        "max": bench.barrier_max(1.5 + rank, world),
        "sum": bench.sum_over_ranks(1.0 + rank, world),
        "mine": bench.cases_for_rank(cells, rank, world),
        "cells": cells,
    }
    bench.barrier(world)
    import torch.distributed as dist
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


def test_two_ranks_over_gloo(tmp_path):
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r in res:
        assert r["max"] == 2.5
        assert r["sum"] == 3.0
    cells = res[0]["cells"]
    mine = [set(r["mine"]) for r in res]
    assert not (mine[0] & mine[1])
    assert mine[0] | mine[1] == set(range(len(cells)))
    loads = [sum(cells[i] for i in m) for m in mine]
    assert abs(loads[0] - loads[1]) <= max(cells)


def test_case_sharding_single_rank():
    sys.path.insert(0, REPO)
    import bench
    cells = [5, 1, 9, 3]
    assert bench.cases_for_rank(cells, 0, 1) == [0, 1, 2, 3]
    # the largest first to the least-loaded rank
    assert bench.cases_for_rank(cells, 0, 2) == [2]
    assert bench.cases_for_rank(cells, 1, 2) == [0, 1, 3]
