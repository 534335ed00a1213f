"""The drop-in boundary: array type, push/pull/create*, plugin_function.

Mirrors pyclesperanto_prototype/_tier0 (push _push.py:4-41, pull _pull.py:4-28,
create* _create.py:5-52, plugin_function _plugin_function.py:12-76, Image /
is_image _types.py:1-23, Backend _backends.py:2-20) with device buffers held
as PyTorch CUDA tensors.  Arrays exchange with other frameworks through
DLPack (``__dlpack__`` / ``from_dlpack``) and ``__cuda_array_interface__``.
"""
from __future__ import annotations

import inspect
from functools import wraps
from typing import Callable, Union

import numpy as np
import torch

from . import _lib


class B200Array:
    """Device image: a C-contiguous torch CUDA tensor plus the small numpy-like
    surface the reference's OCLArray offers (shape, dtype, get, __array__,
    astype, min/max/sum)."""

    __slots__ = ("tensor",)

    def __init__(self, tensor: torch.Tensor):
        if not tensor.is_cuda:
            raise ValueError("B200Array holds CUDA tensors only")
        self.tensor = tensor.contiguous()

    # numpy-like surface ------------------------------------------------
    @property
    def shape(self):
        return tuple(self.tensor.shape)

    @property
    def dtype(self):
        return np.dtype(_lib.np_dtype_of(self.tensor))

    @property
    def ndim(self):
        return self.tensor.dim()

    @property
    def size(self):
        return self.tensor.numel()

    @property
    def nbytes(self):
        return self.tensor.numel() * self.tensor.element_size()

    def get(self) -> np.ndarray:
        t = self.tensor.cpu()
        if t.dtype in (torch.uint16, torch.uint32):
            return t.numpy().copy()
        return t.numpy()

    def __array__(self, dtype=None, copy=None):
        a = self.get()
        return a.astype(dtype) if dtype is not None else a

    def astype(self, dtype):
        dt = np.dtype(dtype)
        tt = {np.dtype(np.float32): torch.float32, np.dtype(np.uint8): torch.uint8,
              np.dtype(np.uint16): torch.uint16, np.dtype(np.uint32): torch.uint32,
              np.dtype(np.int32): torch.int32}.get(dt)
        if tt is None:
            raise KeyError(f"Type {dt} is currently unsupported for buffers/arrays")
        return B200Array(self.tensor.to(tt))

    def min(self):
        return float(self.tensor.min().item()) if self.tensor.dtype == torch.float32 else self.tensor.to(torch.float64).min().item()

    def max(self):
        return float(self.tensor.max().item()) if self.tensor.dtype == torch.float32 else self.tensor.to(torch.float64).max().item()

    def sum(self):
        return float(self.tensor.to(torch.float64).sum().item())

    def __len__(self):
        return self.shape[0]

    def __repr__(self):
        return f"B200Array({self.get()!r}, dtype={self.dtype})"

    # interchange -------------------------------------------------------
    def __dlpack__(self, stream=None, **kw):
        return self.tensor.__dlpack__(stream=stream) if stream is not None else self.tensor.__dlpack__()

    def __dlpack_device__(self):
        return self.tensor.__dlpack_device__()

    @property
    def __cuda_array_interface__(self):
        return self.tensor.__cuda_array_interface__


Image = Union[np.ndarray, B200Array, torch.Tensor, list, tuple]


def is_image(obj) -> bool:
    """_tier0/_types.py:13-23: which arguments plugin_function pushes."""
    return isinstance(obj, (np.ndarray, tuple, list, B200Array, torch.Tensor)) or str(type(obj)) in [
        "<class 'cupy._core.core.ndarray'>",
        "<class 'dask.array.core.Array'>",
        "<class 'xarray.core.dataarray.DataArray'>",
        "<class 'resource_backed_dask_array.ResourceBackedDaskArray'>",
        "<class 'pyclesperanto._pyclesperanto._Array'>",
    ]


def _device():
    _lib.load()
    return torch.device("cuda", torch.cuda.current_device())


_NATIVE = (np.dtype(np.uint8), np.dtype(np.uint16))


def _to_numpy(any_array):
    if isinstance(any_array, (list, tuple)):
        return np.asarray(any_array)
    if hasattr(any_array, "shape") and hasattr(any_array, "dtype") and hasattr(any_array, "get"):
        return np.asarray(any_array.get())
    return np.asarray(any_array)


def push(any_array) -> B200Array:
    """Copies an image to device memory as float32 (_tier0/_push.py:4-41).
    Device tensors and arrays are converted on the device."""
    if isinstance(any_array, B200Array):
        return any_array
    dev = _device()
    if isinstance(any_array, torch.Tensor):
        t = any_array.detach().to(dev, dtype=torch.float32)
        return B200Array(t.contiguous())
    if hasattr(any_array, "__dlpack__") and hasattr(any_array, "__cuda_array_interface__"):
        t = torch.from_dlpack(any_array)
        return B200Array(t.to(dev, dtype=torch.float32).contiguous())
    a = _to_numpy(any_array)
    if a.dtype in _NATIVE:
        # copy the narrow type and widen on the device (exactly float32(x))
        t = torch.from_numpy(np.ascontiguousarray(a)).to(dev, non_blocking=False)
        return B200Array(t.to(torch.float32))
    return B200Array(torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(dev))


def push_native(any_array) -> B200Array:
    """Like push, but keeps uint8/uint16 data in its own type on the device.
    Used for inputs the kernels read in any of u8/u16/f32 (values identical to
    the float32 push, fewer bytes moved)."""
    if isinstance(any_array, B200Array):
        return any_array
    if isinstance(any_array, torch.Tensor) and any_array.dtype in (torch.uint8, torch.uint16):
        return B200Array(any_array.detach().to(_device()).contiguous())
    if isinstance(any_array, np.ndarray) and any_array.dtype in _NATIVE:
        return B200Array(torch.from_numpy(np.ascontiguousarray(any_array)).to(_device()))
    return push(any_array)


push_zyx = push
asarray = push


def pull(gpu_array) -> np.ndarray:
    """Device image to numpy (_tier0/_pull.py:4-28)."""
    if isinstance(gpu_array, B200Array):
        return gpu_array.get()
    if isinstance(gpu_array, torch.Tensor):
        return gpu_array.detach().cpu().numpy()
    return np.asarray(gpu_array)


pull_zyx = pull
nparray = pull

_NP_TO_TORCH = {np.dtype(np.float32): torch.float32, np.dtype(np.uint8): torch.uint8,
                np.dtype(np.uint16): torch.uint16, np.dtype(np.uint32): torch.uint32,
                np.dtype(np.int32): torch.int32}


def create(dimensions, dtype=np.float32) -> B200Array:
    """_tier0/_create.py:5-21 (uninitialised device image)."""
    if isinstance(dimensions, B200Array):
        dimensions = dimensions.shape
    else:
        dimensions = tuple(int(d) for d in dimensions)
    tt = _NP_TO_TORCH.get(np.dtype(dtype))
    if tt is None:
        raise KeyError(f"Type {np.dtype(dtype)} is currently unsupported for buffers/arrays")
    return B200Array(torch.empty(dimensions, dtype=tt, device=_device()))


create_zyx = lambda dimensions: create(dimensions[::-1])  # noqa: E731


def _dims(args, reverse_numpy: bool):
    d = args[0]
    if isinstance(d, B200Array):
        return d.shape
    if reverse_numpy and isinstance(d, np.ndarray):
        return d.shape[::-1]
    if hasattr(d, "shape"):
        return tuple(d.shape)
    return d


def create_like(*args) -> B200Array:
    return create(_dims(args, False))


def create_binary_like(*args) -> B200Array:
    return create(_dims(args, True), np.uint8)


def create_labels_like(*args) -> B200Array:
    return create(_dims(args, True), np.uint32)


def create_none(*args):
    return None


def plugin_function(function: Callable = None, output_creator: Callable = create_like,
                    categories: list = None, priority: int = 0, native_inputs=()):
    """_tier0/_plugin_function.py:12-76: binds the arguments (TypeError on a
    mismatch), pushes every Image-annotated argument, creates missing outputs
    with output_creator, calls the function.  Parameters named in
    native_inputs are pushed with push_native."""
    if function is None:
        return lambda f: plugin_function(f, output_creator=output_creator, categories=categories,
                                         priority=priority, native_inputs=native_inputs)
    function.fullargspec = inspect.getfullargspec(function)
    function.categories = categories
    function.priority = priority
    sig = inspect.signature(function)
    n_creator = len(inspect.signature(output_creator).parameters)

    @wraps(function)
    def worker_function(*args, **kwargs):
        bound = sig.bind(*args, **kwargs)
        bound.apply_defaults()
        for key, value in bound.arguments.items():
            if key in sig.parameters and sig.parameters[key].annotation in (Image, "Image"):
                if is_image(value):
                    bound.arguments[key] = (push_native if key in native_inputs else push)(value)
                if value is None:
                    bound.arguments[key] = output_creator(*bound.args[:n_creator])
        return function(*bound.args, **bound.kwargs)

    worker_function.__module__ = "pyclesperanto_prototype_b200"
    return worker_function


class Backend:
    """The reference's backend singleton (_tier0/_backends.py:2-20): this
    package has one backend, the B200 one."""

    def __init__(self):
        self._current_backend = B200Backend()

    def set(self, backend):
        self._current_backend = backend

    def get(self):
        return self._current_backend

    @classmethod
    def get_instance(cls):
        if not hasattr(cls, "instance"):
            cls.instance = Backend()
        return cls.instance


class B200Backend:
    """A backend with the reference's backend interface
    (_tier0/_opencl_backend.py:10-44, installed the way _tier0/_device.py:62-71
    installs the cupy backend: ``Backend.get_instance().set(B200Backend(...))``).

    Its arrays are B200Array (torch CUDA tensors): once installed in the
    reference, the reference's push / create / create_like return device
    arrays of this package, which the cle.* functions of this package take and
    return without a host round trip.  Kernels outside this package's path
    arrive at execute(); they are handed to `fallback` (another backend, e.g.
    the reference's OpenCL backend): every B200Array argument is copied into
    the fallback's arrays, the kernel runs there, and the arrays are copied
    back, so only those kernels pay a host round trip.  Without a fallback
    execute raises NotImplementedError."""

    def __init__(self, fallback=None):
        self.fallback = fallback

    def array_type(self):
        return B200Array

    def asarray(self, array):
        return pull(array)

    def empty(self, shape, dtype=np.float32):
        return create(shape, dtype)

    def from_array(self, array):
        return push(array)

    def empty_image_like(self, array):
        return create_like(array)

    def execute(self, anchor, opencl_kernel_filename, kernel_name, global_size, parameters, prog=None,
                constants=None, image_size_independent_kernel_compilation=None, device=None):
        if self.fallback is None:
            raise NotImplementedError(
                f"{kernel_name}: this kernel is outside the B200 path; construct B200Backend(fallback=...) "
                "with the backend that runs it")
        mine = {k: v for k, v in parameters.items() if isinstance(v, B200Array)}
        theirs = dict(parameters)
        for k, v in mine.items():
            theirs[k] = self.fallback.from_array(v.get())
        result = self.fallback.execute(anchor, opencl_kernel_filename, kernel_name, global_size, theirs,
                                       prog=prog, constants=constants,
                                       image_size_independent_kernel_compilation=image_size_independent_kernel_compilation,
                                       device=device)
        for k, v in mine.items():
            host = np.asarray(self.fallback.asarray(theirs[k]))
            v.tensor.copy_(torch.from_numpy(np.ascontiguousarray(host.astype(v.dtype, copy=False))).to(v.tensor.device))
        return result

    def __str__(self):
        return "B200 backend (sm_100a kernels of pyclesperanto_prototype_b200)"
