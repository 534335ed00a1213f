"""Replicas across GPUs, host side, on the CPU: the request router, and a
world_size-2 gloo process group that serves a request list with a stand-in
server (no GPU), gathers the summaries and uses the bench's rank helpers."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pyclesperanto_prototype_b200.replicas import route, serve_replicated


def test_route_balances_by_capacity():
    sizes = [10, 10, 10, 10, 40, 5, 5]
    a = route(sizes, [100.0, 100.0])
    assert a == route(sizes, [100.0, 100.0])          # deterministic
    load = [sum(s for s, g in zip(sizes, a) if g == k) for k in range(2)]
    assert abs(load[0] - load[1]) <= max(sizes)
    b = route([1] * 30, [300.0, 100.0])               # a GPU with 3x the budget gets ~3x the work
    assert 21 <= b.count(0) <= 24 and b.count(0) + b.count(1) == 30
    with pytest.raises(ValueError):
        route([1], [])


class _Req:
    def __init__(self, rid, nbytes, arrival):
        self.rid, self.nbytes, self.arrival = rid, nbytes, arrival
        self.num_labels, self.done, self.table = 0, -1.0, None


class _FakeServer:
    """Stands in for SegmentationServer: 'labels' a request by its id."""

    def __init__(self, rank):
        self.rank = rank

    def run(self, reqs, realtime=True):
        for r in reqs:
            r.num_labels = 1000 * self.rank + r.rid
            r.done = r.arrival + 0.001 * (r.rid + 1)
        return reqs


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        reqs = [_Req(i, 10 + (i % 3) * 7, 0.01 * i) for i in range(17)]
        out = serve_replicated(reqs, _FakeServer, lambda r: r.nbytes, 1e3)
        expected = route([r.nbytes for r in reqs], [1e3] * world)
        ok = (sorted(s.rid for s in out) == list(range(17))
              and all(s.rank == expected[s.rid] for s in out)
              and all(s.num_labels == 1000 * s.rank + s.rid for s in out))
        import bench
        bench.barrier(world)
        m = bench.max_over_ranks(float(rank + 1), world)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{int(ok)} {m}\n")
    finally:
        dist.destroy_process_group()


def test_serve_replicated_two_ranks_gloo(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    for r in range(2):
        ok, m = open(tmp_path / f"rank{r}.txt").read().split()
        assert ok == "1"
        assert float(m) == 2.0
