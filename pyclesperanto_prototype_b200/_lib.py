"""ctypes binding of libcle_b200.so (declarations in include/cle_b200.h).

There is no fallback: if the library is missing, cannot be loaded, or no CUDA
device is present, every op raises.  Status codes map to the exception types
the reference raises for the same conditions (see ``check``).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcle_b200.so")

CLE_U8, CLE_U16, CLE_U32, CLE_I32, CLE_F32 = 1, 2, 3, 4, 5
STATS_NCOLS = 35

_TORCH_TO_CODE = {
    torch.uint8: CLE_U8,
    torch.uint16: CLE_U16,
    torch.uint32: CLE_U32,
    torch.int32: CLE_I32,
    torch.float32: CLE_F32,
}

ERRORS = {
    1: KeyError,        # unsupported dtype (_tier0/_pycl.py:44-48 raises KeyError)
    2: ValueError,      # shape
    3: ValueError,      # argument
    4: RuntimeError,    # workspace
    5: RuntimeError,    # device loop limit
    6: RuntimeError,    # CUDA
    7: ValueError,      # too large
    8: RuntimeError,    # cancelled through the call's cancel word
}
CLE_ERR_ITER_LIMIT = 5
CLE_ERR_CANCELLED = 8


class CleTensor(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("ndim", ctypes.c_int32),
        ("dtype", ctypes.c_int32),
        ("shape", ctypes.c_int64 * 3),
        ("strides", ctypes.c_int64 * 3),
        ("device", ctypes.c_int32),
    ]


class CallOptions(ctypes.Structure):
    """cle_call_options: per-call limits of the device loops (0 = default)."""
    _fields_ = [
        ("struct_bytes", ctypes.c_uint32),
        ("max_loop_steps", ctypes.c_uint32),
        ("loop_time_limit_ms", ctypes.c_uint32),
        ("barrier_time_limit_ms", ctypes.c_uint32),
        ("cooperative_ctas", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("cancel", ctypes.c_void_p),
    ]


def call_options(max_loop_steps: int = 0, loop_time_limit_ms: int = 0, barrier_time_limit_ms: int = 0,
                 cooperative_ctas: int = 0, cancel_ptr: int = 0) -> CallOptions:
    """cancel_ptr: address of an int32 in pinned host memory (or 0): a nonzero
    value there stops the call's device loop with CLE_ERR_CANCELLED."""
    o = CallOptions()
    o.struct_bytes = ctypes.sizeof(CallOptions)
    o.max_loop_steps = int(max_loop_steps)
    o.loop_time_limit_ms = int(loop_time_limit_ms)
    o.barrier_time_limit_ms = int(barrier_time_limit_ms)
    o.cooperative_ctas = int(cooperative_ctas)
    o.reserved = 0
    o.cancel = int(cancel_ptr) or None
    return o


_lib = None

# name: (restype, argtypes)
_P = ctypes.c_void_p
_T = ctypes.POINTER(CleTensor)
_SZ = ctypes.c_size_t
_O = ctypes.POINTER(CallOptions)
_SIGS = {
    "cle_abi_version": (ctypes.c_int, []),
    "cle_version": (ctypes.c_char_p, []),
    "cle_last_error_message": (ctypes.c_char_p, []),
    "cle_kernel_launches": (ctypes.c_ulonglong, []),
    "cle_profile_enable": (ctypes.c_int, [ctypes.c_int]),
    "cle_profile_stage_ms": (ctypes.c_int, [_P, ctypes.c_int]),
    "cle_profile_trace": (ctypes.c_int, [_P, _SZ]),
    "cle_gaussian_blur_workspace_bytes": (_SZ, [_T]),
    "cle_gaussian_blur": (ctypes.c_int, [_T, _T, ctypes.c_double, ctypes.c_double, ctypes.c_double, _P, _SZ, _P]),
    "cle_minimum_maximum_workspace_bytes": (_SZ, [_T]),
    "cle_minimum_maximum": (ctypes.c_int, [_T, _P, _P, _SZ, _P]),
    "cle_histogram_workspace_bytes": (_SZ, [_T, ctypes.c_int]),
    "cle_histogram": (ctypes.c_int, [_T, _T, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, _P, _SZ, _P]),
    "cle_threshold_otsu_workspace_bytes": (_SZ, [_T]),
    "cle_threshold_otsu": (ctypes.c_int, [_T, _T, _P, _P, _SZ, _P]),
    "cle_threshold_otsu_noalloc": (ctypes.c_int, [_T, _T, _P]),
    "cle_threshold_otsu_noalloc_scratch_bytes": (_SZ, []),
    "cle_greater_constant": (ctypes.c_int, [_T, _T, ctypes.c_float, _P]),
    "cle_binary_and": (ctypes.c_int, [_T, _T, _T, _P]),
    "cle_erode_box": (ctypes.c_int, [_T, _T, _P]),
    "cle_add_image_and_scalar": (ctypes.c_int, [_T, _T, ctypes.c_float, _P]),
    "cle_replace_intensities": (ctypes.c_int, [_T, _T, _T, _P]),
    "cle_euclidean_distance_from_label_centroid_map": (ctypes.c_int, [_T, _T, _T, _P]),
    "cle_generate_distance_matrix": (ctypes.c_int, [_T, _T, _T, _P]),
    "cle_generate_touch_matrix": (ctypes.c_int, [_T, _T, _P]),
    "cle_average_distance_of_n_distances": (ctypes.c_int, [_T, ctypes.c_int, ctypes.c_int, _T, _P]),
    "cle_average_distance_of_touching_neighbors": (ctypes.c_int, [_T, _T, _T, _P]),
    "cle_average_distance_of_n_nearest_points": (ctypes.c_int, [_T, _T, ctypes.c_int, ctypes.c_int, _T, _P]),
    "cle_average_distance_of_touching_labels_workspace_bytes": (_SZ, [ctypes.c_int64]),
    "cle_average_distance_of_touching_labels": (ctypes.c_int, [_T, _T, _T, _P, _SZ, _P]),
    "cle_box_filter_workspace_bytes": (_SZ, [_T]),
    "cle_minimum_box": (ctypes.c_int, [_T, _T, ctypes.c_double, ctypes.c_double, ctypes.c_double, _P, _SZ, _P]),
    "cle_maximum_box": (ctypes.c_int, [_T, _T, ctypes.c_double, ctypes.c_double, ctypes.c_double, _P, _SZ, _P]),
    "cle_top_hat_box": (ctypes.c_int, [_T, _T, ctypes.c_double, ctypes.c_double, ctypes.c_double, _P, _SZ, _P]),
    "cle_mask": (ctypes.c_int, [_T, _T, _T, _P]),
    "cle_detect_maxima_box_workspace_bytes": (_SZ, [_T, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "cle_detect_maxima_box": (ctypes.c_int, [_T, _T, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _SZ, _P]),
    "cle_connected_components_labeling_box_workspace_bytes": (_SZ, [_T]),
    "cle_connected_components_labeling_box": (ctypes.c_int, [_T, _T, _P, _SZ, _P]),
    "cle_relabel_sequential_workspace_bytes": (_SZ, [_T, ctypes.c_uint32]),
    "cle_relabel_sequential": (ctypes.c_int, [_T, _T, ctypes.c_uint32, _P, _SZ, _P]),
    "cle_masked_voronoi_labeling_workspace_bytes": (_SZ, [_T]),
    "cle_masked_voronoi_labeling": (ctypes.c_int, [_T, _T, _T, _O, _P, _SZ, _P]),
    "cle_connected_components_labeling_diamond_workspace_bytes": (_SZ, [_T]),
    "cle_connected_components_labeling_diamond": (ctypes.c_int, [_T, _T, _P, _SZ, _P]),
    "cle_extend_labeling_via_voronoi_workspace_bytes": (_SZ, [_T]),
    "cle_extend_labeling_via_voronoi": (ctypes.c_int, [_T, _T, _O, _P, _SZ, _P]),
    "cle_voronoi_labeling_workspace_bytes": (_SZ, [_T]),
    "cle_voronoi_labeling": (ctypes.c_int, [_T, _T, _O, _P, _SZ, _P]),
    "cle_masked_voronoi_labeling_binary_workspace_bytes": (_SZ, [_T]),
    "cle_masked_voronoi_labeling_binary": (ctypes.c_int, [_T, _T, _T, _O, _P, _SZ, _P]),
    "cle_voronoi_otsu_labeling_workspace_bytes": (_SZ, [_T]),
    "cle_voronoi_otsu_labeling": (ctypes.c_int, [_T, _T, ctypes.c_double, ctypes.c_double, _O, _P, _SZ, _P]),
    "cle_vol_batch_plan": (ctypes.c_int, [_T, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, _O,
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "cle_vol_batch_workspace_bytes": (_SZ, [_P]),
    "cle_vol_batch_lanes": (ctypes.c_int, [_P]),
    "cle_vol_batch_launch": (ctypes.c_int, [_P, _T, _T, _P, _SZ, _P, _P]),
    "cle_vol_batch_free": (None, [_P]),
    "cle_workspace_status": (ctypes.c_int, [_P, _SZ, _P]),
    "cle_label_centroids_workspace_bytes": (_SZ, [_T, ctypes.c_int64]),
    "cle_label_centroids": (ctypes.c_int, [_T, ctypes.c_int64, _P, _P, _SZ, _P]),
    "cle_workspace_label_count": (_P, [_P]),
    "cle_statistics_of_labelled_pixels_device_count": (ctypes.c_int, [_T, _T, _P, ctypes.c_int64, _P, _P, _SZ, _P]),
    "cle_label_maximum_workspace_bytes": (_SZ, [_T]),
    "cle_label_maximum": (ctypes.c_int, [_T, _P, _P, _SZ, _P]),
    "cle_statistics_workspace_bytes": (_SZ, [_T, ctypes.c_int64]),
    "cle_statistics_of_labelled_pixels": (ctypes.c_int, [_T, _T, ctypes.c_int64, _P, _P, _SZ, _P]),
}


def exported_symbols():
    """Names the header declares (and the library must export)."""
    return list(_SIGS)


def load(require_gpu: bool = True):
    """Loads the library (once).  Raises when it is missing or, with
    require_gpu, when no CUDA device is visible."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is not built; run `python -m pyclesperanto_prototype_b200._build`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    if require_gpu and not torch.cuda.is_available():
        raise RuntimeError("pyclesperanto_prototype_b200 needs a CUDA device (sm_100a); none is visible")
    return _lib


def check(status: int, what: str = "") -> None:
    if status != 0:
        msg = load(require_gpu=False).cle_last_error_message().decode(errors="replace")
        raise ERRORS.get(status, RuntimeError)(f"{what}: {msg}" if what else msg)


def tensor_desc(t: torch.Tensor) -> CleTensor:
    if not t.is_cuda:
        raise ValueError("device tensor expected")
    code = _TORCH_TO_CODE.get(t.dtype)
    if code is None:
        raise KeyError(f"Type {t.dtype} is currently unsupported for buffers/arrays")
    d = CleTensor()
    d.data = t.data_ptr()
    d.ndim = t.dim()
    d.dtype = code
    for i in range(3):
        d.shape[i] = t.shape[i] if i < t.dim() else 1
        d.strides[i] = t.stride(i) if i < t.dim() else 1
    d.device = t.device.index if t.device.index is not None else torch.cuda.current_device()
    return d


def ref(d: CleTensor):
    return ctypes.byref(d)


def stream_ptr(device=None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def workspace(nbytes: int, device) -> torch.Tensor:
    """Caller-provided scratch (torch caching allocator, 512-byte aligned)."""
    if nbytes <= 0:
        return torch.empty(0, dtype=torch.uint8, device=device)
    return torch.empty(int(nbytes), dtype=torch.uint8, device=device)


def np_dtype_of(t: torch.Tensor):
    return {torch.uint8: np.uint8, torch.uint16: np.uint16, torch.uint32: np.uint32,
            torch.int32: np.int32, torch.float32: np.float32}[t.dtype]
