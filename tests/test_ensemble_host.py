"""Ensemble sharding on the host: the partition of members across ranks and the
gather of per-member summaries over a world-size-2 gloo group."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from impes_b200 import scenarios
from impes_b200.ensemble import gather, partition


def test_partition_covers_every_member_once_and_balances():
    cases = scenarios.ensemble(seed=4, members=64, steps=30)
    cells = [c[0]["reservoir"]["dimensions"][0] * c[0]["reservoir"]["dimensions"][1]
             * c[0]["reservoir"]["dimensions"][2] for c in cases]
    assert min(cells) >= 32 * 32 * 4 and max(cells) <= 128 * 128 * 16
    for world in (1, 2, 3, 4, 8):
        parts = partition(cells, world)
        flat = sorted(m for p in parts for m in p)
        assert flat == list(range(len(cells)))
        loads = [sum(cells[m] for m in p) for p in parts]
        # greedy largest-first: the spread is at most the largest member
        assert max(loads) - min(loads) <= max(cells)
        assert parts == partition(cells, world)          # deterministic


def test_partition_edge_cases():
    assert partition([], 3) == [[], [], []]
    assert partition([5], 2) == [[0], []]
    assert partition([3, 3, 3, 3], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        partition([1], 0)


def _rank_main(rank, world, port, cells, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = partition(cells, world)[rank]
        local = [{"member": m, "cells": cells[m], "rank": rank} for m in mine]
        full = gather(local, world)
        out[rank] = full
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_gather_over_gloo_world_two():
    cells = [4096, 262144, 16384, 65536, 8192, 131072, 32768]
    with mp.get_context("spawn").Manager() as man:
        out = man.dict()
        mp.spawn(_rank_main, args=(2, _free_port(), cells, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1]
    assert [s["member"] for s in res[0]] == list(range(len(cells)))
    parts = partition(cells, 2)
    for s in res[0]:
        assert s["member"] in parts[s["rank"]]
