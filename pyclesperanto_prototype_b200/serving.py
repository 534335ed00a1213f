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
  * the copy-out stream brings the label image back into the request's own
    pinned host buffer (when it gives one), and, once the 8 bytes are on the
    host, the statistics of exactly that many labels.

So uploads and downloads overlap the computation of other requests, while
the computations themselves run one after another on the whole GPU (one
compute stream, the default) or two at a time (compute_streams=2, each
cooperative launch then capped at half the SMs).  With express_voxels > 0,
requests of at most that many voxels take an express lane (their own upload
and compute streams, cooperative launches on express_ctas SMs), so small
requests do not queue behind large ones.  The CTA cap and the loop limits
travel with each call (cle_call_options); nothing is set process-wide, so
several servers may run in one process.  Device buffers (input, labels,
workspaces, tables) are kept per shape and reused, so after warm-up no
request allocates.  Completion is detected by polling CUDA events;
latency = completion - arrival.

Failures stay with their request: a request whose volume the library
rejects (dtype, shape) or whose device loop stops at a limit records its
status and message, and the loop goes on with the others.  cancel(rid)
drops a waiting request, and stops an admitted one at its next growth step
through a cancel word in pinned host memory that the device loop reads.
Each request's result is the same as the per-call path's
(tests/test_batch_serve_gpu.py).
"""
from __future__ import annotations

import collections
import dataclasses
import threading
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
    labels: torch.Tensor = None   # device uint32 labels (keep_labels)
    labels_out: torch.Tensor = None   # optional pinned host uint32 tensor of the volume's shape:
                                      # the label image is copied there
    max_loop_steps: int = 0       # per-request limit of the growth loop (0: default)
    num_labels: int = 0
    table: np.ndarray = None      # statistics table [35, num_labels]
    status: int = 0               # 0, or the cle_status that ended the request
    error: str = None             # message of a failed request
    cancelled: bool = False

    @property
    def ok(self) -> bool:
        return self.status == 0 and self.error is None and not self.cancelled

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
        # the request's cancel word, read by the device loop once per step
        self.cancel = torch.zeros(1, dtype=torch.int32).pin_memory()
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
        # the statistics tables on a stream of their own: behind the label
        # images of other requests on copy_out, a finished request's table
        # would hold its slot until those downloads end
        self.copy_table = torch.cuda.Stream(device=self.device)
        self.computes = [torch.cuda.Stream(device=self.device) for _ in range(max(1, int(compute_streams)))]
        self._next = 0
        self.pool = collections.defaultdict(list)    # (shape, dtype) -> [_Buffers] free
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        # express lane: requests of at most express_voxels get their own upload
        # and compute streams, so they never wait behind a large request; its
        # cooperative growth launches use express_ctas SMs, the others the rest
        self.express_voxels = int(express_voxels)
        self.express = None
        self.express_ctas = 0
        reserve = 0
        if self.express_voxels > 0:
            self.express = (torch.cuda.Stream(device=self.device), torch.cuda.Stream(device=self.device))
            self.express_ctas = max(1, min(int(express_ctas), sms // 2))
            reserve = self.express_ctas
        multi = len(self.computes) > 1 or self.express is not None
        self.coop = max(1, (sms - reserve) // len(self.computes)) if multi else 0
        self._lock = threading.Lock()
        self._cancel = set()          # rids asked to stop (cancel() may come from any thread)

    # -- buffers ----------------------------------------------------------
    def _take(self, shape, dtype):
        key = (tuple(shape), dtype)
        if self.pool[key]:
            return self.pool[key].pop()
        return _Buffers(tuple(shape), dtype, self.device)

    def _give(self, shape, dtype, b):
        self.pool[(tuple(shape), dtype)].append(b)

    def cancel(self, rid: int) -> None:
        """Asks the server to stop request `rid`: a request still waiting is
        dropped; an admitted one stops at the next step of its growth loop
        (its device work after the loop still runs, its results are
        discarded).  Either way the request ends with cancelled=True."""
        with self._lock:
            self._cancel.add(rid)

    def _cancel_requested(self, rid) -> bool:
        with self._lock:
            return rid in self._cancel

    # -- one request on one slot -------------------------------------------
    def _start(self, req: Request, t_ref: float):
        """Enqueues the request's work; returns (buffers, event) or raises
        (the caller records the failure)."""
        b = self._take(req.volume.shape, req.volume.dtype)
        try:
            return b, self._enqueue(req, b, t_ref)
        except Exception:
            self._give(req.volume.shape, req.volume.dtype, b)
            raise

    def _enqueue(self, req: Request, b: _Buffers, t_ref: float):
        lib = _lib.load()
        if req.volume.device.type != "cpu":
            raise ValueError(f"request {req.rid}: the volume must be in host memory")
        if req.labels_out is not None and (tuple(req.labels_out.shape) != tuple(req.volume.shape)
                                           or req.labels_out.dtype != torch.uint32):
            raise ValueError(f"request {req.rid}: labels_out must be uint32 of the volume's shape")
        if self.express is not None and req.volume.numel() <= self.express_voxels:
            up, s = self.express
            coop = self.express_ctas
        else:
            up, s = self.copy_in, self.computes[self._next]
            self._next = (self._next + 1) % len(self.computes)
            coop = self.coop
        b.cancel.zero_()
        opts = _lib.call_options(max_loop_steps=req.max_loop_steps, cooperative_ctas=coop,
                                 cancel_ptr=b.cancel.data_ptr())
        # validate before anything is enqueued (a rejected volume leaves no work behind)
        _lib.tensor_desc(b.src)
        if b.src.dtype not in (torch.uint8, torch.uint16, torch.float32):
            raise KeyError(f"request {req.rid}: Type {b.src.dtype} is currently unsupported for buffers/arrays")
        with torch.cuda.stream(up):
            b.src.copy_(req.volume, non_blocking=True)
            uploaded = torch.cuda.Event()
            uploaded.record(up)
        s.wait_event(uploaded)
        with torch.cuda.stream(s):
            vol_into(b.src, b.labels, b.ws, self.spot, self.outline, s.cuda_stream, opts)
            count = lib.cle_workspace_label_count(b.ws.data_ptr())
            i, l = _lib.tensor_desc(b.src), _lib.tensor_desc(b.labels)
            _lib.check(lib.cle_statistics_of_labelled_pixels_device_count(
                _lib.ref(i), _lib.ref(l), count, b.capacity, b.table.data_ptr(), b.stats_ws.data_ptr(),
                b.stats_ws.numel(), s.cuda_stream), "statistics_of_labelled_pixels")
            computed = torch.cuda.Event()
            computed.record(s)
            # loop status and label count back to the host first (8 bytes)
            status_count = torch.stack([b.ws[0:4].view(torch.int32)[0], b.ws[8:12].view(torch.int32)[0]])
            b.host_count.copy_(status_count, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
        b.labels_done = None
        if req.labels_out is not None:
            self.copy_out.wait_event(computed)
            with torch.cuda.stream(self.copy_out):
                req.labels_out.copy_(b.labels, non_blocking=True)
                b.labels_done = torch.cuda.Event()
                b.labels_done.record(self.copy_out)
        req.admitted = time.perf_counter() - t_ref
        return ev

    def _copy_table(self, req: Request, b: _Buffers, done_compute):
        """Second half of a request: checks status and count, then copies the
        statistics of the request's labels only; returns the event to poll
        (recorded after every copy that reads the request's buffers)."""
        status, count = int(b.host_count[0]), int(b.host_count[1])
        s = self.copy_table
        s.wait_event(done_compute)
        if b.labels_done is not None:
            s.wait_event(b.labels_done)   # the buffers stay busy until the labels are out
        if status == _lib.CLE_ERR_CANCELLED or (status == 0 and self._cancel_requested(req.rid)):
            req.cancelled = True
        elif status:
            req.status = status
            req.error = f"request {req.rid}: device status {status} ({_lib.ERRORS.get(status, RuntimeError).__name__})"
        elif count > b.capacity:
            req.status = _lib.CLE_ERR_TOO_LARGE
            req.error = f"request {req.rid}: {count} labels exceed the table capacity {b.capacity}"
        else:
            req.num_labels = count
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
        if not req.ok:
            req.num_labels = 0
            req.table = np.zeros((len(STAT_KEYS), 0), np.float32)
            return
        n = req.num_labels
        req.table = b.host_table[:len(STAT_KEYS) * n].view(len(STAT_KEYS), n).numpy().copy()

    # -- trace replay --------------------------------------------------------
    def run(self, requests, realtime: bool = True):
        """Serves `requests` (sorted by arrival).  With realtime, a request is
        not admitted before its arrival time.  Returns the requests with their
        admitted / done times (seconds since the start), results, or status /
        error / cancelled for the ones that did not finish."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        running = {}       # slot -> [req, buffers, event, bytes, stage]
        in_use = 0.0
        t0 = time.perf_counter()
        while pending or running:
            now = time.perf_counter() - t0
            for k in list(running):
                req, b, ev, nbytes, stage = running[k]
                if stage == 0 and self._cancel_requested(req.rid):
                    b.cancel.fill_(1)              # the device loop stops at its next step
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
            # waiting requests that were cancelled leave the queue at once
            if pending and self._cancel:
                keep = collections.deque()
                for req in pending:
                    if self._cancel_requested(req.rid):
                        req.cancelled = True
                        req.done = time.perf_counter() - t0
                        req.table = np.zeros((len(STAT_KEYS), 0), np.float32)
                    else:
                        keep.append(req)
                pending = keep
            free = [k for k in range(self.slots) if k not in running]
            while pending and free and (not realtime or pending[0].arrival <= now):
                req = pending[0]
                try:
                    nbytes = request_bytes(req.volume.shape, req.volume.dtype)
                except Exception as e:          # a dtype torch or the library rejects
                    pending.popleft()
                    self._fail(req, e, t0)
                    continue
                if in_use + nbytes > self.budget and running:
                    break                      # wait for memory to free up
                pending.popleft()
                try:
                    b, ev = self._start(req, t0)
                except Exception as e:
                    self._fail(req, e, t0)
                    continue
                k = free.pop(0)
                running[k] = [req, b, ev, nbytes, 0]
                in_use += nbytes
            if running and not free:
                time.sleep(20e-6)
            elif running:
                time.sleep(20e-6)
            elif pending and realtime and pending[0].arrival > now:
                time.sleep(min(1e-3, pending[0].arrival - now))
        return requests

    @staticmethod
    def _fail(req: Request, e: Exception, t0: float):
        code = {KeyError: 1, ValueError: 3}.get(type(e), _lib.CLE_ERR_CUDA if isinstance(e, RuntimeError) else 3)
        req.status = code
        req.error = f"{type(e).__name__}: {e}"
        req.done = time.perf_counter() - t0
        req.table = np.zeros((len(STAT_KEYS), 0), np.float32)


def per_call_loop(requests, spot_sigma: float, outline_sigma: float, realtime: bool = True,
                  keep_labels: bool = False):
    """The plain per-call path on the same trace: one request at a time through
    the public API (voronoi_otsu_labeling, then statistics_of_labelled_pixels),
    each started at max(arrival, previous completion).  With keep_labels each
    request keeps its device label image (memory grows with the trace); a
    request with labels_out gets its label image copied there."""
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
        if req.labels_out is not None:
            req.labels_out.copy_(lab.tensor)
        torch.cuda.synchronize()
        req.done = time.perf_counter() - t0
        req.num_labels = len(stats["label"])
        req.table = np.stack([stats[k] for k in STAT_KEYS]) if req.num_labels else np.zeros((35, 0), np.float32)
        if keep_labels:
            req.labels = lab.tensor
    return requests
