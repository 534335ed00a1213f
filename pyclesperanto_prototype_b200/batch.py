"""Batched form: many independent volumes through voronoi_otsu_labeling as one
CUDA graph.

The plan and launch live in the C ABI (cle_vol_batch_plan /
cle_vol_batch_launch): tiles of any mix of 2D / 3D shapes are spread over K
lanes (CUDA streams forked from the caller's stream) by a longest-first
greedy schedule on voxel count; tiles in a lane run one after another on that
lane's workspace slice (sized for its largest tile), lanes run concurrently,
and K comes from the library's tuned table unless given.  The whole batch is
captured into one CUDA graph after one uncaptured warm-up run, so a batch is
a single graph launch with no host work per tile.  While several lanes run,
each cooperative launch of the growth loop is capped at SMs / K CTAs so the
concurrent grids always fit on the GPU together.  Results are the same labels
as the per-call path, tile by tile (tests/test_batch_serve_gpu.py).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._tier0 import B200Array


def _desc(t: torch.Tensor):
    return _lib.tensor_desc(t)


def vol_workspace_bytes(shape, dtype=torch.float32) -> int:
    d = _lib.CleTensor()
    d.data = 256
    d.ndim = len(shape)
    d.dtype = _lib._TORCH_TO_CODE[dtype]
    acc = 1
    strides = []
    for s in reversed(shape):
        strides.insert(0, acc)
        acc *= int(s)
    for i in range(3):
        d.shape[i] = int(shape[i]) if i < len(shape) else 1
        d.strides[i] = strides[i] if i < len(shape) else 1
    d.device = 0
    return int(_lib.load(require_gpu=False).cle_voronoi_otsu_labeling_workspace_bytes(_lib.ref(d)))


def vol_into(src: torch.Tensor, dst: torch.Tensor, ws: torch.Tensor, spot_sigma: float,
             outline_sigma: float, stream: int, options: "_lib.CallOptions" = None) -> None:
    """One voronoi_otsu_labeling on `stream` with an explicit workspace and
    per-call loop options (None: defaults)."""
    s, d = _desc(src), _desc(dst)
    lib = _lib.load()
    _lib.check(lib.cle_voronoi_otsu_labeling(_lib.ref(s), _lib.ref(d), float(spot_sigma),
                                             float(outline_sigma),
                                             _lib.ref(options) if options is not None else None,
                                             ws.data_ptr(), ws.numel(), stream),
               "voronoi_otsu_labeling")


def workspace_status(ws: torch.Tensor, stream: int) -> int:
    return int(_lib.load().cle_workspace_status(ws.data_ptr(), ws.numel(), stream))


def schedule(voxels, lanes: int):
    """Longest-first greedy assignment of tiles to lanes (lists of indices)."""
    order = sorted(range(len(voxels)), key=lambda i: -voxels[i])
    load = [0] * lanes
    out = [[] for _ in range(lanes)]
    for i in order:
        k = int(np.argmin(load))
        out[k].append(i)
        load[k] += voxels[i]
    return out


class VolBatch:
    """voronoi_otsu_labeling over a fixed set of device volumes through the C
    ABI's batched form (cle_vol_batch_plan / cle_vol_batch_launch), replayed
    as one CUDA graph.

        batch = VolBatch(inputs, spot_sigma=3.5, outline_sigma=1.0)
        batch.run()                 # labels in batch.outputs[i]

    lanes = 0 takes the lane count from the library's tuned table."""

    def __init__(self, inputs, spot_sigma: float = 2.0, outline_sigma: float = 2.0,
                 lanes: int = 0, use_graph: bool = True, max_loop_steps: int = 0, cooperative_ctas: int = 0):
        lib = _lib.load()
        self.inputs = [x.tensor if isinstance(x, B200Array) else x for x in inputs]
        for t in self.inputs:
            if not t.is_cuda or not t.is_contiguous():
                raise ValueError("VolBatch inputs must be contiguous CUDA tensors")
        self.spot, self.outline = float(spot_sigma), float(outline_sigma)
        self.device = self.inputs[0].device
        self.outputs = [torch.empty(t.shape, dtype=torch.uint32, device=self.device) for t in self.inputs]
        n = len(self.inputs)
        self._in = (_lib.CleTensor * n)(*[_desc(t) for t in self.inputs])
        self._out = (_lib.CleTensor * n)(*[_desc(t) for t in self.outputs])
        self.options = _lib.call_options(max_loop_steps=max_loop_steps, cooperative_ctas=cooperative_ctas)
        self._plan = ctypes.c_void_p()
        _lib.check(lib.cle_vol_batch_plan(self._in, n, self.spot, self.outline, int(lanes),
                                          _lib.ref(self.options), ctypes.byref(self._plan)), "vol_batch_plan")
        self.lanes = int(lib.cle_vol_batch_lanes(self._plan))
        self.ws = torch.empty(max(1, int(lib.cle_vol_batch_workspace_bytes(self._plan))), dtype=torch.uint8,
                              device=self.device)
        # the maximum of every tile's loop status, written on the device
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.graph = None
        self.use_graph = use_graph
        self.launches_per_run = 0     # library kernels one run launches

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value and _lib._lib is not None:
            _lib._lib.cle_vol_batch_free(plan)
            self._plan = None

    def _issue(self):
        lib = _lib.load()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(lib.cle_vol_batch_launch(self._plan, self._in, self._out, self.ws.data_ptr(), self.ws.numel(),
                                            self.status.data_ptr(), stream), "vol_batch_launch")

    def capture(self):
        lib = _lib.load()
        self._issue()                       # uncaptured warm-up (sets kernel attributes)
        torch.cuda.synchronize(self.device)
        self.check()
        if self.use_graph:
            g = torch.cuda.CUDAGraph()
            cap = torch.cuda.Stream(device=self.device)
            cap.wait_stream(torch.cuda.current_stream(self.device))
            n0 = lib.cle_kernel_launches()
            with torch.cuda.graph(g, stream=cap, capture_error_mode="thread_local"):
                self._issue()
            self.launches_per_run = int(lib.cle_kernel_launches() - n0)
            self.graph = g
        return self

    def run(self):
        """One batch on the current stream (graph replay when captured)."""
        lib = _lib.load()
        if self.graph is None and self.use_graph:
            self.capture()
        if self.graph is not None:
            self.graph.replay()
        else:
            n0 = lib.cle_kernel_launches()
            self._issue()
            self.launches_per_run = int(lib.cle_kernel_launches() - n0)
        return self.outputs

    def check(self):
        """Raises if any tile's device loop reported a limit (synchronises)."""
        st = int(self.status.max().item())
        if st:
            raise _lib.ERRORS.get(st, RuntimeError)(f"voronoi_otsu_labeling (batch): device status {st}")
