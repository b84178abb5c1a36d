"""Sharding of the batched ensemble over ranks (host logic, CPU): the
greedy cost balance, and two gloo ranks that each take their shard and
gather the per-member results, as bench.py's ensemble mode does across
GPUs."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fs2_b200 import ensemble as E


def test_config5_members():
    m = E.config5_members()
    assert len(m) == 48
    assert [x.seed for x in m] == list(range(100, 148))
    sizes = {(x.nc, x.n, x.boxsize) for x in m}
    assert sizes == {(32, 64, 32.0), (64, 128, 64.0), (96, 192, 96.0)}
    # the scope's per-step figure for the 48 members: 9.55 GB
    assert abs(sum(E.step_bytes(x) for x in m) / 1e9 - 9.54) < 0.02


@pytest.mark.parametrize("world", [1, 2, 3, 4, 5, 8])
def test_assignment_is_a_balanced_partition(world):
    m = E.config5_members()
    parts = E.assignment(m, world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(m)))
    loads = [sum(E.step_bytes(m[i]) for i in p) for p in parts]
    # greedy longest-first: the heaviest rank exceeds the mean by less than
    # one member's cost
    assert max(loads) - sum(loads) / world < max(E.step_bytes(x) for x in m)
    for r in range(world):
        assert E.shard(m, world, r) == [m[i] for i in parts[r]]


def test_assignment_rejects_empty_world():
    with pytest.raises(ValueError):
        E.assignment(E.config5_members(), 0)


def _member_value(m):
    # a deterministic stand-in for a member's loss
    return float(np.random.default_rng(m.seed).standard_normal(m.nc).sum())


def _rank_main(rank, world, port, out):
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port,
                            rank=rank, world_size=world)
    try:
        members = E.config5_members()
        mine = E.shard(members, world, rank)
        idx = E.assignment(members, world)[rank]
        local = [(i, _member_value(m)) for i, m in zip(idx, mine)]
        gathered = [None] * world
        dist.all_gather_object(gathered, local)
        t = torch.tensor([float(sum(E.step_bytes(m) for m in mine))],
                         dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            res = dict(kv for part in gathered for kv in part)
            np.save(out, np.array([res[i] for i in range(len(members))]))
            np.save(out + ".max.npy", t.numpy())
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_cover_every_member(tmp_path):
    out = str(tmp_path / "vals.npy")
    mp.spawn(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True)
    vals = np.load(out)
    members = E.config5_members()
    assert np.array_equal(vals, [_member_value(m) for m in members])
    loads = [sum(E.step_bytes(members[i]) for i in p)
             for p in E.assignment(members, 2)]
    assert float(np.load(out + ".max.npy")[0]) == max(loads)


def test_eval_bytes_model():
    # the evaluation's byte model: forward steps, backward steps, the 2LPT
    # both ways and the loss; the backward step moves more than the forward
    from fs2_b200.ensemble import (Member, adjoint_step_bytes, eval_bytes,
                                   lpt_bytes, step_bytes)
    m = Member(32, 64, 32.0, 1)
    N, n = 32 ** 3, 64
    R, K = n ** 3, n * n * (n // 2 + 1)
    assert step_bytes(m) == 120 * N + 32 * R + 32 * K
    assert adjoint_step_bytes(m) == 240 * N + 68 * R + 64 * K
    assert adjoint_step_bytes(m) > step_bytes(m)
    assert eval_bytes(m, 5) == (5 * (step_bytes(m) + adjoint_step_bytes(m)) +
                                3 * lpt_bytes(m) + 16 * R)
