"""Replica scheduling: disjoint units per rank and the max-over-ranks timing (gloo, 2 ranks)."""

from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pyticc_b200.replicas import Unit, all_units, max_over_ranks, rank_units


def test_units_cover_the_workload_once():
    units = all_units(2, 256, 16)
    assert len(units) == 32
    assert len(set(units)) == 32
    assert units[0] == Unit(0, 0, 16) and units[-1] == Unit(1, 240, 256)
    ragged = all_units(1, 10, 4)
    assert ragged[-1] == Unit(0, 8, 10)


@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_ranks_get_disjoint_units(world):
    per_rank = [rank_units(2, 256, 16, r, world, 32 // world) for r in range(world)]
    flat = [u for units in per_rank for u in units]
    assert len(flat) == len(set(flat)) == 32


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, results):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        mine = rank_units(2, 256, 16, rank, world, 4)
        slowest = max_over_ranks(1.0 + rank, dist)
        results[rank] = (slowest, [(u.block, u.start) for u in mine])
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_take_the_max_and_split_units():
    world = 2
    manager = mp.get_context("spawn").Manager()
    results = manager.dict()
    mp.start_processes(_worker, args=(world, _free_port(), results), nprocs=world, start_method="spawn")
    assert results[0][0] == results[1][0] == 2.0
    assert not set(results[0][1]) & set(results[1][1])


def test_single_process_max_is_identity():
    assert max_over_ranks(3.5) == 3.5
    assert torch.tensor([1.0]).item() == 1.0
