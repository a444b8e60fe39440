"""Data-parallel training of the learned corrector, host side: the batch
shard of every rank and the gradient average over ranks, the latter on two
gloo ranks on the CPU (the training kernels themselves need the GPU)."""

import os
import socket

import numpy as np

from hexdyn.corrector import average_gradients, global_mean_loss, rank_batches


def test_rank_batches_cover_each_batch_once():
    for n in (0, 1, 7, 8, 33):
        for world in (1, 2, 3, 4):
            per = n // world
            shards = [rank_batches(n, r, world) for r in range(world)]
            assert all(len(s) == per for s in shards)  # the same step count on every rank
            assert sorted(b for s in shards for b in s) == list(range(per * world))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    grads = [torch.full((3, 2), float(rank + 1)), torch.arange(4, dtype=torch.float32) * (rank + 1)]
    average_gradients(grads)
    dist.destroy_process_group()
    q.put((rank, [g.numpy().copy() for g in grads]))


def test_average_gradients_on_two_gloo_ranks():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, (a, b) in out:
        np.testing.assert_array_equal(a, np.full((3, 2), 1.5, dtype=np.float32))
        np.testing.assert_array_equal(b, np.arange(4, dtype=np.float32) * 1.5)


def _rank_loss(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    # 5 batches over 2 ranks: each runs 2 (batch 4 is left out); rank r's
    # batches r and r + 2 have squared-error sums 10 (r + 1) and 20 (r + 1)
    mine = rank_batches(5, rank, world)
    loss = sum(10.0 * (rank + 1) * (i + 1) for i in range(len(mine)))
    out = global_mean_loss(loss, 100 * len(mine), dist.group.WORLD)
    dist.destroy_process_group()
    q.put((rank, mine, out))


def test_epoch_loss_is_the_mean_over_ranks_with_a_ragged_batch_count():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_loss, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [[0, 2], [1, 3]]
    want = (10 + 20 + 20 + 40) / 400.0
    assert [o[2] for o in out] == [want, want]
    assert global_mean_loss(30.0, 200) == 0.15
