"""bench.py's multi-rank plumbing on CPU: two ranks over gloo.

On a GPU box ``bench.py --gpus N`` runs one process per GPU under torchrun
(NCCL); every rank runs an independent replica, and rank 0 reports all ranks'
work over the slowest rank's device time.  Here the same helpers run as two
spawned CPU processes with the gloo backend (rendezvous on 127.0.0.1): the
barrier, the max over ranks and the round-robin sharding of independent work
units.
"""

from __future__ import annotations

import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench

    w, r, _ = bench.dist_setup(world, backend="gloo")
    bench.barrier(w)
    slowest = bench.max_over_ranks(10.0 * (r + 1), w)
    units = bench.shard(list(range(11)), r, w)
    bench.barrier(w)
    dist.destroy_process_group()
    out.put((r, w, slowest, units))


def test_two_ranks_time_max_and_shard():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, *_ in results] == [0, 1]
    assert all(w == 2 for _, w, _, _ in results)
    # both ranks see the slowest rank's time
    assert all(t == pytest.approx(20.0) for _, _, t, _ in results)
    # every unit on exactly one rank
    units = results[0][3] + results[1][3]
    assert sorted(units) == list(range(11)) and results[0][3] == [0, 2, 4, 6, 8, 10]


def test_single_process_needs_no_group():
    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.pop("WORLD_SIZE", None)
    assert bench.dist_setup(1)[0] == 1
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.shard([1, 2, 3], 0, 1) == [1, 2, 3]
