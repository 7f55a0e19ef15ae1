"""Worlds across ranks, on the CPU: the cell-balanced partition, and two
gloo ranks that each serve their own share of a request stream (the fake
device of the serving tests) and together serve every request exactly
once, with no collective but the host-side gathers."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from worldinagrain_b200 import serve, shard

from .test_serve_cpu import FakeBackend, FakeClock


def _sizes(n, seed):
    rng = np.random.default_rng(seed)
    return [int(16 * round(64 * 8 ** rng.uniform() / 16)) ** 2 for _ in range(n)]


@pytest.mark.parametrize("n_ranks", [1, 2, 3, 8])
def test_partition_covers_once_and_balances(n_ranks):
    cells = _sizes(512, 4)
    shares = shard.partition(cells, n_ranks)
    flat = sorted(k for s in shares for k in s)
    assert flat == list(range(512))
    loads = [sum(cells[k] for k in s) for s in shares]
    assert max(loads) - min(loads) <= max(cells)
    assert shares == shard.partition(cells, n_ranks)  # deterministic


def test_partition_more_ranks_than_worlds():
    shares = shard.partition([5, 3], 4)
    assert sorted(k for s in shares for k in s) == [0, 1]
    assert sum(1 for s in shares if not s) == 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world_size, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        sizes = [10 + (k % 5) for k in range(24)]
        mine = shard.share_of(sizes, rank, world_size)
        owner = shard.owners(shard.partition(sizes, world_size))
        arrivals = serve.poisson_arrivals(3000.0, 200, len(sizes), seed=11)
        # each rank takes the requests routed to it, worlds renumbered locally
        local = {k: i for i, k in enumerate(mine)}
        my_arr = [(t, local[w]) for t, w in arrivals if shard.route(w, owner) == rank]
        clock = FakeClock()
        be = FakeBackend([sizes[k] for k in mine], step_s=0.002, clock=clock)
        srv = serve.Server(be, len(mine), 10_000, clock=clock)
        srv.preload()
        done = srv.run(my_arr)
        served = torch.tensor(sorted(mine[r.world] for r in done) + [-1] * (200 - len(done)), dtype=torch.int64)
        gathered = [torch.zeros(200, dtype=torch.int64) for _ in range(world_size)]
        dist.all_gather(gathered, served)
        if rank == 0:
            allw = torch.cat(gathered)
            np.save(os.path.join(out_dir, "served.npy"), allw[allw >= 0].numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_serve_every_request_once(tmp_path):
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    served = np.sort(np.load(tmp_path / "served.npy"))
    arrivals = serve.poisson_arrivals(3000.0, 200, 24, seed=11)
    want = np.sort(np.array([w for _, w in arrivals]))
    assert np.array_equal(served, want)
