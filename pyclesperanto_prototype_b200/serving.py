"""Served form: continuous batching of segmentation requests on one GPU.

A request is a volume in (pinned) host memory.  The server admits a waiting
request as soon as one of its `slots` (requests in flight) is free and the
request's device memory fits in the HBM budget, and enqueues all of its work
at once, on three kinds of streams:

  * the copy-in stream uploads the volume (requests in admission order);
  * a compute stream waits for that upload and runs the pipeline
    (voronoi_otsu_labeling, then statistics_of_labelled_pixels reading the
    label count the pipeline left on the device -- no host round trip) and
    copies the loop status and label count (8 bytes) to the host;
  * once those 8 bytes are on the host, the copy-out stream brings back the
    statistics of exactly that many labels.

So uploads and downloads overlap the computation of other requests, while
the computations themselves run one after another on the whole GPU (one
compute stream, the default) or two at a time (compute_streams=2, each
cooperative launch then capped at half the SMs).  With express_voxels > 0,
requests of at most that many voxels take an express lane (their own upload
and compute streams, cooperative launches on express_ctas SMs), so small
requests do not queue behind large ones.  Device buffers (input,
labels, workspaces, tables) are kept per shape and reused, so after warm-up
no request allocates.  Completion is detected by polling CUDA events;
latency = completion - arrival.  Each request's result is the same as the
per-call path's (tests/test_batch_serve_gpu.py).
"""
from __future__ import annotations

import collections
import dataclasses
import time

import numpy as np
import torch

from . import _lib
from .batch import vol_into, vol_workspace_bytes
from ._ops import STAT_KEYS


@dataclasses.dataclass
class Request:
    rid: int
    volume: torch.Tensor          # host tensor (pinned for overlap), uint8/uint16/float32
    arrival: float                # seconds since the start of the trace
    admitted: float = -1.0
    done: float = -1.0
    labels: torch.Tensor = None   # device uint32 labels
    num_labels: int = 0
    table: np.ndarray = None      # statistics table [35, num_labels]

    @property
    def latency(self) -> float:
        return self.done - self.arrival

    def statistics(self) -> dict:
        L = self.num_labels
        out = {"label": np.arange(1, L + 1), "original_label": np.arange(1, L + 1)}
        for i, k in enumerate(STAT_KEYS):
            out[k] = self.table[i, :L].copy()
        return out


class _Buffers:
    """Device buffers for one shape, reused across requests of that shape."""

    def __init__(self, shape, dtype, device):
        n = int(np.prod(shape))
        self.src = torch.empty(shape, dtype=dtype, device=device)
        self.labels = torch.empty(shape, dtype=torch.uint32, device=device)
        self.ws = torch.empty(vol_workspace_bytes(shape, dtype), dtype=torch.uint8, device=device)
        # statistics: label capacity = one label per 64 voxels (labels need voxels)
        self.capacity = max(1024, n // 64)
        self.table = torch.empty((len(STAT_KEYS), self.capacity), dtype=torch.float32, device=device)
        lib = _lib.load()
        d = _lib.tensor_desc(self.labels)
        self.stats_ws = torch.empty(int(lib.cle_statistics_workspace_bytes(_lib.ref(d), self.capacity)),
                                    dtype=torch.uint8, device=device)
        # pinned host copy of the statistics, grown when a request has more labels
        self.host_table = torch.empty(len(STAT_KEYS) * min(self.capacity, 1 << 16),
                                      dtype=torch.float32).pin_memory()
        self.host_count = torch.empty(2, dtype=torch.int32).pin_memory()
        self.bytes = sum(t.numel() * t.element_size() for t in
                         (self.src, self.labels, self.ws, self.table, self.stats_ws))


def request_bytes(shape, dtype) -> int:
    """Device bytes a request of this shape holds while admitted."""
    n = int(np.prod(shape))
    es = torch.empty(0, dtype=dtype).element_size()
    cap = max(1024, n // 64)
    return n * es + n * 4 + vol_workspace_bytes(shape, dtype) + cap * (35 * 4 + 200)


class SegmentationServer:
    def __init__(self, budget_bytes: float = 60e9, slots: int = 4, spot_sigma: float = 2.0,
                 outline_sigma: float = 2.0, device=None, keep_labels: bool = False,
                 compute_streams: int = 1, express_voxels: int = 0, express_ctas: int = 16):
        _lib.load()
        self.keep_labels = keep_labels
        self.device = torch.device(device or "cuda", torch.cuda.current_device()) \
            if device is None else torch.device(device)
        self.budget = float(budget_bytes)
        self.slots = int(slots)
        self.spot, self.outline = float(spot_sigma), float(outline_sigma)
        self.copy_in = torch.cuda.Stream(device=self.device)
        self.copy_out = torch.cuda.Stream(device=self.device)
        self.computes = [torch.cuda.Stream(device=self.device) for _ in range(max(1, int(compute_streams)))]
        self._next = 0
        self.pool = collections.defaultdict(list)    # (shape, dtype) -> [_Buffers] free
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        # express lane: requests of at most express_voxels get their own upload
        # and compute streams, so they never wait behind a large request; its
        # cooperative growth launches use express_ctas SMs, the others the rest
        self.express_voxels = int(express_voxels)
        self.express = None
        reserve = 0
        if self.express_voxels > 0:
            self.express = (torch.cuda.Stream(device=self.device), torch.cuda.Stream(device=self.device))
            self.express_ctas = max(1, min(int(express_ctas), sms // 2))
            reserve = self.express_ctas
        multi = len(self.computes) > 1 or self.express is not None
        self.coop = max(1, (sms - reserve) // len(self.computes)) if multi else 0

    # -- buffers ----------------------------------------------------------
    def _take(self, shape, dtype):
        key = (tuple(shape), dtype)
        if self.pool[key]:
            return self.pool[key].pop()
        return _Buffers(tuple(shape), dtype, self.device)

    def _give(self, shape, dtype, b):
        self.pool[(tuple(shape), dtype)].append(b)

    # -- one request on one slot -------------------------------------------
    def _start(self, req: Request, k: int, t_ref: float):
        b = self._take(req.volume.shape, req.volume.dtype)
        lib = _lib.load()
        if self.express is not None and req.volume.numel() <= self.express_voxels:
            up, s = self.express
            lib.cle_set_cooperative_ctas(self.express_ctas)
        else:
            up, s = self.copy_in, self.computes[self._next]
            self._next = (self._next + 1) % len(self.computes)
            lib.cle_set_cooperative_ctas(self.coop)
        with torch.cuda.stream(up):
            b.src.copy_(req.volume, non_blocking=True)
            uploaded = torch.cuda.Event()
            uploaded.record(up)
        s.wait_event(uploaded)
        with torch.cuda.stream(s):
            vol_into(b.src, b.labels, b.ws, self.spot, self.outline, s.cuda_stream)
            count = lib.cle_workspace_label_count(b.ws.data_ptr())
            i, l = _lib.tensor_desc(b.src), _lib.tensor_desc(b.labels)
            _lib.check(lib.cle_statistics_of_labelled_pixels_device_count(
                _lib.ref(i), _lib.ref(l), count, b.capacity, b.table.data_ptr(), b.stats_ws.data_ptr(),
                b.stats_ws.numel(), s.cuda_stream), "statistics_of_labelled_pixels")
            # loop status and label count back to the host first (8 bytes)
            status_count = torch.stack([b.ws[0:4].view(torch.int32)[0], b.ws[8:12].view(torch.int32)[0]])
            b.host_count.copy_(status_count, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
        req.admitted = time.perf_counter() - t_ref
        return b, ev

    def _copy_table(self, req: Request, b: _Buffers, done_compute):
        """Second half of a request: checks status and count, then copies the
        statistics of the request's labels only; returns the event to poll."""
        status, count = int(b.host_count[0]), int(b.host_count[1])
        if status:
            raise _lib.ERRORS.get(status, RuntimeError)(f"request {req.rid}: device status {status}")
        if count > b.capacity:
            raise RuntimeError(f"request {req.rid}: {count} labels exceed the table capacity {b.capacity}")
        req.num_labels = count
        s = self.copy_out
        s.wait_event(done_compute)
        if len(STAT_KEYS) * count > b.host_table.numel():
            b.host_table = torch.empty(len(STAT_KEYS) * count * 2, dtype=torch.float32).pin_memory()
        with torch.cuda.stream(s):
            if count:
                b.host_table[:len(STAT_KEYS) * count].copy_(b.table[:, :count].contiguous().view(-1),
                                                             non_blocking=True)
            if self.keep_labels:
                req.labels = b.labels.clone()  # the pooled buffer is reused by later requests
            ev = torch.cuda.Event()
            ev.record(s)
        return ev

    def _finish(self, req: Request, b: _Buffers):
        n = req.num_labels
        req.table = b.host_table[:len(STAT_KEYS) * n].view(len(STAT_KEYS), n).numpy().copy()

    # -- trace replay --------------------------------------------------------
    def run(self, requests, realtime: bool = True):
        """Serves `requests` (sorted by arrival).  With realtime, a request is
        not admitted before its arrival time.  Returns the requests with their
        admitted / done times (seconds since the start)."""
        lib = _lib.load()
        lib.cle_set_cooperative_ctas(self.coop)
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        running = {}       # slot -> [req, buffers, event, bytes, stage]
        in_use = 0.0
        t0 = time.perf_counter()
        try:
            while pending or running:
                now = time.perf_counter() - t0
                for k in list(running):
                    req, b, ev, nbytes, stage = running[k]
                    if not ev.query():
                        continue
                    if stage == 0:                 # status and count arrived: copy the table
                        running[k] = [req, b, self._copy_table(req, b, ev), nbytes, 1]
                        continue
                    req.done = time.perf_counter() - t0
                    self._finish(req, b)
                    self._give(req.volume.shape, req.volume.dtype, b)
                    in_use -= nbytes
                    del running[k]
                free = [k for k in range(self.slots) if k not in running]
                while pending and free and (not realtime or pending[0].arrival <= now):
                    req = pending[0]
                    nbytes = request_bytes(req.volume.shape, req.volume.dtype)
                    if in_use + nbytes > self.budget and running:
                        break                      # wait for memory to free up
                    pending.popleft()
                    k = free.pop(0)
                    b, ev = self._start(req, k, t0)
                    running[k] = [req, b, ev, nbytes, 0]
                    in_use += nbytes
                if running and not free:
                    time.sleep(20e-6)
                elif pending and realtime and pending[0].arrival > now and not running:
                    time.sleep(min(1e-3, pending[0].arrival - now))
        finally:
            lib.cle_set_cooperative_ctas(0)
        return requests


def per_call_loop(requests, spot_sigma: float, outline_sigma: float, realtime: bool = True,
                  keep_labels: bool = False):
    """The plain per-call path on the same trace: one request at a time through
    the public API (voronoi_otsu_labeling, then statistics_of_labelled_pixels),
    each started at max(arrival, previous completion).  With keep_labels each
    request keeps its device label image (memory grows with the trace)."""
    from . import _ops
    from ._tier0 import push_native
    t0 = time.perf_counter()
    for req in sorted(requests, key=lambda r: r.arrival):
        if realtime:
            while time.perf_counter() - t0 < req.arrival:
                time.sleep(50e-6)
        req.admitted = time.perf_counter() - t0
        img = push_native(req.volume)
        lab = _ops.voronoi_otsu_labeling(img, spot_sigma=spot_sigma, outline_sigma=outline_sigma)
        stats = _ops.statistics_of_labelled_pixels(img, lab)
        torch.cuda.synchronize()
        req.done = time.perf_counter() - t0
        req.num_labels = len(stats["label"])
        req.table = np.stack([stats[k] for k in STAT_KEYS]) if req.num_labels else np.zeros((35, 0), np.float32)
        if keep_labels:
            req.labels = lab.tensor
    return requests
