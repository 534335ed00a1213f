"""cle_threshold_otsu_noalloc: the threshold_otsu entry point for callers that
cannot allocate device memory (it uses a scratch array built into the
library).  Checked through the C ABI against cle_threshold_otsu (which takes a
caller workspace) on two calls in a row; the second call uses a smaller image
so that anything left over from the first call in the shared array would
show.  This file is collected last so that a failure here does not hide the
other tests; it also passes run on its own in a fresh process."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from pyclesperanto_prototype_b200 import _build, _lib
    _build.build()
    return _lib


def _reference(img):
    import pyclesperanto_prototype_b200 as cle
    return cle.pull(cle.threshold_otsu(img))


def _noalloc(lib, img):
    import torch
    src = torch.from_numpy(np.ascontiguousarray(img, dtype=np.float32)).cuda()
    dst = torch.empty(img.shape, dtype=torch.uint8, device="cuda")
    s, d = lib.tensor_desc(src), lib.tensor_desc(dst)
    status = lib.load().cle_threshold_otsu_noalloc(lib.ref(s), lib.ref(d), lib.stream_ptr())
    lib.check(status, "threshold_otsu_noalloc")
    torch.cuda.synchronize()
    return dst.cpu().numpy()


def test_noalloc_matches_workspace_entry_point_twice(lib):
    rng = np.random.default_rng(40)
    first = rng.gamma(2.0, 40.0, size=(24, 300, 200)).astype(np.float32)
    second = (rng.normal(500.0, 90.0, size=(150, 130)) ** 1.1).astype(np.float32)
    for img in (first, second):
        got = _noalloc(lib, img)
        ref = _reference(img)
        assert got.dtype == np.uint8
        assert np.array_equal(got, ref)
        assert 0 < got.sum() < got.size


def test_noalloc_rejects_images_beyond_its_scratch(lib):
    import torch
    img = torch.zeros((8, 5000, 3), dtype=torch.float32, device="cuda")   # 5000 rows > 4096
    out = torch.empty(img.shape, dtype=torch.uint8, device="cuda")
    s, d = lib.tensor_desc(img), lib.tensor_desc(out)
    status = lib.load().cle_threshold_otsu_noalloc(lib.ref(s), lib.ref(d), lib.stream_ptr())
    assert status == 7
    assert b"4096 rows" in lib.load().cle_last_error_message()
    assert lib.load().cle_threshold_otsu_noalloc_scratch_bytes() >= 4 * 1024 * 1024
