"""Replicas across GPUs: one process per GPU, requests routed on the host.

Volumes are independent, so several GPUs serve a request stream as replicas:
each process (one per GPU, started by torch.distributed's launcher) runs its
own SegmentationServer on its own GPU.  Routing needs no communication: every
rank computes the same assignment from the same request list (`route`,
deterministic), and takes its share.  No collective runs on the data path;
only the small per-request summaries (label count, latency, the statistics
table if wanted) are gathered to rank 0 for reporting (`all_gather_object`,
any backend -- gloo on CPU, NCCL on GPUs).
"""
from __future__ import annotations

import dataclasses


def route(request_bytes, capacities):
    """GPU index per request: each request, in order, goes to the GPU whose
    assigned bytes so far, relative to its capacity (free HBM budget), are
    lowest (ties to the lower index).  Deterministic, so every rank computes
    the same assignment."""
    if not capacities:
        raise ValueError("route: no GPUs")
    load = [0.0] * len(capacities)
    out = []
    for b in request_bytes:
        k = min(range(len(capacities)), key=lambda i: ((load[i] + b) / capacities[i], i))
        load[k] += b
        out.append(k)
    return out


@dataclasses.dataclass
class Summary:
    rid: int
    rank: int
    num_labels: int
    arrival: float
    done: float
    table: object = None


def serve_replicated(requests, server_factory, request_bytes_fn, capacity_bytes: float,
                     keep_tables: bool = False):
    """Serves `requests` on all ranks of the default process group.

    server_factory(rank) builds this rank's server (a SegmentationServer on
    the rank's GPU); request_bytes_fn(request) is a request's device memory.
    Every rank gets the list of all Summary records, sorted by request id."""
    import torch.distributed as dist
    rank, world = dist.get_rank(), dist.get_world_size()
    assignment = route([request_bytes_fn(r) for r in requests], [float(capacity_bytes)] * world)
    mine = [r for r, g in zip(requests, assignment) if g == rank]
    if mine:
        server_factory(rank).run(mine, realtime=True)
    local = [Summary(r.rid, rank, int(r.num_labels), float(r.arrival), float(r.done),
                     r.table if keep_tables else None) for r in mine]
    gathered = [None] * world
    dist.all_gather_object(gathered, local)
    return sorted((s for part in gathered for s in part), key=lambda s: s.rid)
