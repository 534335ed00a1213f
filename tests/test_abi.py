"""Host-side checks of the C ABI that need no GPU: the library loads, exports
every entry point include/cle_b200.h declares, and validates its arguments
(shape, dtype, contiguity, workspace) before touching the device."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    txt = open(os.path.join(ROOT, "include", "cle_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cle_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    from pyclesperanto_prototype_b200 import _build, _lib
    _build.build()
    return _lib.load(require_gpu=False)


def test_exports_every_declared_symbol(lib):
    names = _header_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n


def test_binding_table_matches_header():
    from pyclesperanto_prototype_b200 import _lib
    assert sorted(_lib.exported_symbols()) == _header_functions()


def test_no_process_wide_setters(lib):
    """The cooperative-CTA cap and the loop limits are per-call arguments; the
    header declares no setter that would change them for the whole process."""
    names = _header_functions()
    assert "cle_set_cooperative_ctas" not in names
    assert not [n for n in names if n.startswith("cle_set_")]


def test_version(lib):
    assert lib.cle_abi_version() == 2
    assert b"sm_100a" in lib.cle_version()


def _desc(shape, dtype, data=256, strides=None):
    from pyclesperanto_prototype_b200._lib import CleTensor
    d = CleTensor()
    d.data = data
    d.ndim = len(shape)
    d.dtype = dtype
    st = strides or []
    if not st:
        acc = 1
        for s in reversed(shape):
            st.insert(0, acc)
            acc *= s
    for i in range(3):
        d.shape[i] = shape[i] if i < len(shape) else 1
        d.strides[i] = st[i] if i < len(shape) else 1
    d.device = 0
    return d


def test_workspace_queries(lib):
    from pyclesperanto_prototype_b200._lib import CLE_F32, CLE_U16, ref
    s = _desc((128, 512, 512), CLE_U16)
    n = 128 * 512 * 512
    vol = lib.cle_voronoi_otsu_labeling_workspace_bytes(ref(s))
    # T (4 B) + spots, seg (1 B each) + seed list (4 B) + frontier arrays (8 B)
    assert 18 * n <= vol <= 19 * n
    assert lib.cle_gaussian_blur_workspace_bytes(ref(_desc((64, 64), CLE_F32))) >= 2 * 4 * 64 * 64
    assert lib.cle_statistics_workspace_bytes(ref(_desc((8, 8), CLE_F32)), 10) > 0


def test_argument_validation_errors(lib):
    from pyclesperanto_prototype_b200._lib import CLE_F32, CLE_U8, ref
    a = _desc((16, 16), CLE_F32)
    bad_dtype = _desc((16, 16), 99)
    assert lib.cle_gaussian_blur(ref(bad_dtype), ref(a), 1.0, 1.0, 0.0, None, 0, None) == 1
    assert b"dtype" in lib.cle_last_error_message()
    other = _desc((16, 17), CLE_F32)
    assert lib.cle_gaussian_blur(ref(a), ref(other), 1.0, 1.0, 0.0, None, 0, None) == 2
    assert b"shape mismatch" in lib.cle_last_error_message()
    u8 = _desc((16, 16), CLE_U8)
    assert lib.cle_gaussian_blur(ref(a), ref(u8), 1.0, 1.0, 0.0, None, 0, None) == 1
    strided = _desc((16, 16), CLE_F32, strides=[32, 1])
    assert lib.cle_gaussian_blur(ref(strided), ref(a), 1.0, 1.0, 0.0, None, 0, None) == 2
    assert b"contiguous" in lib.cle_last_error_message()
    # missing workspace is reported before any launch
    assert lib.cle_gaussian_blur(ref(a), ref(a), 1.0, 1.0, 0.0, None, 0, None) == 4
    huge = _desc((2048, 1024, 1025), CLE_F32)
    assert lib.cle_voronoi_otsu_labeling_workspace_bytes(ref(huge)) == 0
    assert lib.cle_voronoi_otsu_labeling(ref(huge), ref(huge), 2.0, 2.0, None, None, 0, None) == 7


def test_call_options_are_validated_per_call():
    """Loop limits travel with each call (cle_call_options); malformed options
    are rejected before anything touches a device."""
    from pyclesperanto_prototype_b200 import _lib
    from pyclesperanto_prototype_b200._lib import CLE_F32, ref
    lib = _lib.load(require_gpu=False)
    a = _desc((16, 16), CLE_F32)
    short = _lib.call_options(max_loop_steps=1)
    short.struct_bytes = 8          # a caller built against a smaller struct
    assert lib.cle_voronoi_otsu_labeling(ref(a), ref(a), 2.0, 2.0, ref(short), None, 0, None) == 3
    assert b"struct_bytes" in lib.cle_last_error_message()
    bad = _lib.call_options(cooperative_ctas=-1)
    assert lib.cle_masked_voronoi_labeling_binary(ref(a), ref(a), ref(a), ref(bad), None, 0, None) == 3
    ok = _lib.call_options(max_loop_steps=5, cooperative_ctas=4)
    assert ctypes.sizeof(ok) == 32 and ok.struct_bytes == 32
    # with valid options the call goes on to its own checks (no workspace here)
    assert lib.cle_voronoi_otsu_labeling(ref(a), ref(a), 2.0, 2.0, ref(ok), None, 0, None) == 4
    assert _lib.ERRORS[8] is RuntimeError


def test_status_maps_to_reference_exceptions():
    from pyclesperanto_prototype_b200 import _lib
    assert _lib.ERRORS[1] is KeyError and _lib.ERRORS[2] is ValueError
    assert _lib.ERRORS[5] is RuntimeError and _lib.ERRORS[6] is RuntimeError


def test_signature_binding_errors_before_device_use():
    # plugin_function binds with inspect.signature first (TypeError), as the
    # reference does (_tier0/_plugin_function.py:57)
    import pyclesperanto_prototype_b200 as cle
    with pytest.raises(TypeError):
        cle.voronoi_otsu_labeling(None, None, 1, 1, 1)
    with pytest.raises(TypeError):
        cle.gaussian_blur(sigma_q=3)


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    import numpy as np
    import pyclesperanto_prototype_b200 as cle
    with pytest.raises(RuntimeError):
        cle.voronoi_otsu_labeling(np.zeros((8, 8), np.float32))


def test_batch_plan_validates_before_device_use():
    """The batched form's plan rejects bad arguments on the host."""
    from pyclesperanto_prototype_b200 import _lib
    from pyclesperanto_prototype_b200._lib import CLE_F32, CLE_U32
    lib = _lib.load(require_gpu=False)
    plan = ctypes.c_void_p()
    tiles = (_lib.CleTensor * 2)(_desc((16, 16), CLE_F32), _desc((8, 16, 16), CLE_U32))
    assert lib.cle_vol_batch_plan(tiles, 0, 2.0, 2.0, 0, None, ctypes.byref(plan)) == 3
    assert lib.cle_vol_batch_plan(tiles, 1, 2.0, 2.0, 65, None, ctypes.byref(plan)) == 3
    assert lib.cle_vol_batch_plan(tiles, 2, 2.0, 2.0, 0, None, ctypes.byref(plan)) == 1   # uint32 tile
    assert b"tiles[1]" in lib.cle_last_error_message()
    assert not plan.value
    assert lib.cle_vol_batch_launch(None, tiles, tiles, None, 0, None, None) == 3
    assert lib.cle_vol_batch_workspace_bytes(None) == 0 and lib.cle_vol_batch_lanes(None) == 0
    lib.cle_vol_batch_free(None)
