"""erode_box, gauss_otsu_labeling, eroded_otsu_labeling,
connected_components_labeling_diamond, extend_labeling_via_voronoi and
voronoi_labeling on the device against the oracle: binary images and label
images bit for bit, on the reference's own fixtures, seeded random images of
ragged 2D/3D shapes and blob images."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cle():
    import pyclesperanto_prototype_b200 as m
    from pyclesperanto_prototype_b200 import _build
    _build.build()
    return m


SHAPES = [(1, 1), (1, 9), (9, 1), (5, 7), (33, 65), (130, 257),
          (1, 1, 1), (1, 6, 5), (4, 1, 9), (3, 40, 33), (17, 100, 70), (40, 64, 31)]


# ---------------------------------------------------------------- erode ---
def test_erode_box_reference_test(cle):
    # tests/test_erode_box.py:5-29 of the reference
    t = cle.push(np.asarray([[0, 0, 0, 0, 0], [0, 1, 1, 1, 0], [0, 1, 1, 1, 0], [0, 1, 1, 1, 0],
                             [0, 0, 0, 0, 0]]))
    r = cle.create(t)
    cle.erode_box(t, r)
    ref = np.zeros((5, 5))
    ref[2, 2] = 1
    assert np.array_equal(cle.pull(r), ref)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("density", [0.6, 0.9, 1.0])
def test_erode_box_matches_oracle(cle, oracle, shape, density):
    a = (np.random.default_rng(3).random(shape) < density).astype(np.uint8)
    got = cle.pull(cle.erode_box(cle.push_native(a)))
    assert got.dtype == np.uint8
    assert np.array_equal(got, oracle.erode_box(a))


@pytest.mark.parametrize("src_dtype", [np.uint8, np.uint16, np.uint32, np.int32, np.float32])
@pytest.mark.parametrize("dst_dtype", [np.uint8, np.uint16, np.uint32, np.float32])
def test_erode_box_dtypes(cle, oracle, src_dtype, dst_dtype):
    rng = np.random.default_rng(4)
    a = np.where(rng.random((6, 35, 41)) < 0.85, rng.integers(1, 100, (6, 35, 41)), 0).astype(src_dtype)
    if src_dtype == np.float32:
        a[0, 0, :5] = [0.5, -1.0, np.nan, -0.0, 2.0]     # nonzero test on floats (NaN != 0)
    dst = cle.create(a.shape, dst_dtype)
    cle.erode_box(cle.push_native(a), dst)
    got = cle.pull(dst)
    assert got.dtype == dst_dtype
    assert np.array_equal(got.astype(np.uint8), oracle.erode_box(a))


# ------------------------------------------------------- gauss_otsu -------
def test_gauss_otsu_labeling_reference_test(cle):
    # tests/test_gauss_otsu_labeling.py:4-41 of the reference
    src = np.asarray([[0, 0, 1, 1, 0, 0], [0, 1, 8, 9, 1, 0], [0, 1, 1, 0, 0, 0], [0, 0, 0, 0, 0, 0],
                      [0, 0, 0, 1, 1, 0], [0, 0, 1, 8, 7, 1], [0, 0, 1, 1, 1, 0]])
    ref = np.asarray([[0, 0, 1, 1, 0, 0], [0, 1, 1, 1, 1, 0], [0, 1, 1, 1, 0, 0], [0, 0, 0, 0, 0, 0],
                      [0, 0, 0, 2, 2, 0], [0, 0, 2, 2, 2, 2], [0, 0, 2, 2, 2, 0]])
    out = cle.gauss_otsu_labeling(cle.push(src), outline_sigma=1)
    assert out.dtype == np.uint32
    assert np.array_equal(cle.pull(out), ref)


def _blob_image(shape, seed):
    rng = np.random.default_rng(seed)
    img = rng.normal(10, 3, shape).clip(0)
    grids = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    for _ in range(max(3, int(np.prod(shape) / 1500))):
        c = [rng.uniform(0, s) for s in shape]
        r2 = sum((g - ci) ** 2 for g, ci in zip(grids, c))
        img += rng.uniform(100, 250) * np.exp(-r2 / (2 * rng.uniform(2, 5) ** 2))
    return rng.poisson(img).astype(np.float32)


@pytest.mark.parametrize("shape,sigma", [((64, 80), 1.0), ((200, 150), 2.0), ((256, 256), 5.0),
                                         ((20, 60, 70), 1.0), ((33, 80, 65), 2.0)])
def test_gauss_otsu_labeling_matches_oracle(cle, oracle, shape, sigma):
    img = _blob_image(shape, 11)
    got = cle.pull(cle.gauss_otsu_labeling(img, outline_sigma=sigma))
    ref = oracle.gauss_otsu_labeling(img, sigma)
    assert ref.max() > 0
    assert np.array_equal(got, ref)


def test_gauss_otsu_labeling_uint16_input(cle, oracle):
    # a uint16 volume is blurred in place of its float32 copy: same labels
    img = _blob_image((24, 70, 66), 12).clip(0, 65535).astype(np.uint16)
    got = cle.pull(cle.gauss_otsu_labeling(img, outline_sigma=2))
    assert np.array_equal(got, oracle.gauss_otsu_labeling(img.astype(np.float32), 2))


# ----------------------------------------------------- eroded_otsu --------
def test_eroded_otsu_labeling_reference_test(cle):
    # tests/test_eroded_otsu_labeling.py:4-41 of the reference
    src = np.asarray([[0, 0, 5, 5, 0, 0], [0, 5, 8, 9, 1, 0], [0, 5, 7, 6, 1, 1], [0, 0, 0, 5, 5, 1],
                      [0, 0, 0, 5, 5, 1], [0, 0, 5, 5, 5, 1], [0, 0, 5, 5, 5, 0]])
    ref = np.asarray([[0, 0, 1, 1, 0, 0], [0, 1, 1, 1, 1, 0], [0, 1, 1, 1, 1, 0], [0, 0, 1, 1, 1, 0],
                      [0, 0, 0, 2, 2, 0], [0, 0, 2, 2, 2, 0], [0, 0, 2, 2, 2, 0]])
    out = cle.eroded_otsu_labeling(cle.push(src), number_of_erosions=1.0, outline_sigma=1)
    assert np.array_equal(cle.pull(out), ref)


@pytest.mark.parametrize("shape,erosions,sigma", [((64, 80), 0, 1.0), ((200, 150), 2, 1.0),
                                                  ((256, 256), 5, 2.0), ((20, 60, 70), 1, 1.0),
                                                  ((33, 80, 65), 3, 2.0), ((30, 50, 40), 40, 1.0)])
def test_eroded_otsu_labeling_matches_oracle(cle, oracle, shape, erosions, sigma):
    img = _blob_image(shape, 13)
    got = cle.pull(cle.eroded_otsu_labeling(img, number_of_erosions=erosions, outline_sigma=sigma))
    assert np.array_equal(got, oracle.eroded_otsu_labeling(img, erosions, sigma))


# ------------------------------- diamond CCL and Voronoi labelling -------
def test_ccl_diamond_reference_test(cle):
    # tests/test_connected_components_labeling_diamond.py:4-27 of the reference
    src = cle.push(np.asarray([[[0, 1, 0, 1], [0, 1, 0, 0], [1, 0, 0, 1]]]))
    out = cle.connected_components_labeling_diamond(src)
    assert np.array_equal(cle.pull(out), [[[0, 2, 0, 3], [0, 2, 0, 0], [1, 0, 0, 4]]])


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("density", [0.3, 0.55, 0.8])
def test_ccl_diamond_matches_oracle(cle, oracle, shape, density):
    a = (np.random.default_rng(5).random(shape) < density).astype(np.uint8)
    got = cle.pull(cle.connected_components_labeling_diamond(cle.push_native(a)))
    assert np.array_equal(got, oracle.connected_components_labeling_diamond(a))


def test_extend_labeling_via_voronoi_reference_test(cle):
    # tests/test_extend_labeling_via_voronoi.py:4-37 of the reference
    src = cle.push(np.asarray([[[0, 0, 0, 0, 3, 3], [0, 4, 0, 0, 3, 3], [0, 0, 0, 0, 0, 0],
                                [0, 0, 0, 0, 0, 0], [0, 2, 0, 0, 1, 0], [0, 0, 0, 0, 0, 0]]]))
    ref = [[[4, 4, 4, 3, 3, 3], [4, 4, 4, 3, 3, 3], [4, 4, 4, 3, 3, 3], [2, 2, 2, 1, 1, 1],
            [2, 2, 2, 1, 1, 1], [2, 2, 2, 1, 1, 1]]]
    assert np.array_equal(cle.pull(cle.extend_labeling_via_voronoi(src)), ref)


def test_voronoi_labeling_reference_test(cle):
    # tests/test_voronoi_labeling.py:4-37 of the reference
    src = np.zeros((1, 6, 6))
    src[0, 1, 1] = src[0, 1, 4] = src[0, 4, 1] = src[0, 4, 4] = 1
    ref = [[[1, 1, 1, 3, 3, 3]] * 3 + [[2, 2, 2, 4, 4, 4]] * 3]
    assert np.array_equal(cle.pull(cle.voronoi_labeling(cle.push(src))), ref)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("density", [0.0005, 0.01, 0.2])
def test_voronoi_labeling_matches_oracle(cle, oracle, shape, density):
    a = (np.random.default_rng(6).random(shape) < density).astype(np.uint8)
    got = cle.pull(cle.voronoi_labeling(cle.push_native(a)))
    assert np.array_equal(got, oracle.voronoi_labeling(a))


@pytest.mark.parametrize("shape", [(70, 90), (20, 64, 50), (9, 130, 40)])
def test_extend_labeling_via_voronoi_any_label_values(cle, oracle, shape):
    # arbitrary uint32 label values, including ones at and above 2^31, held as
    # a uint32 device image (push would round them to float32 like the reference)
    import torch
    rng = np.random.default_rng(7)
    lab = np.zeros(shape, np.uint32)
    idx = rng.choice(lab.size, 25, replace=False)
    lab.flat[idx] = rng.integers(1, 2 ** 32 - 1, 25, dtype=np.uint64).astype(np.uint32)
    lab.flat[idx[:3]] = [2 ** 31, 2 ** 31 + 5, 2 ** 32 - 1]
    src = cle.B200Array(torch.from_numpy(lab).cuda())
    got = cle.pull(cle.extend_labeling_via_voronoi(src, cle.create_labels_like(src)))
    assert np.array_equal(got, oracle.extend_labeling_via_voronoi(lab))


# ---------------------------------- minimum / maximum box, top-hat -------
def test_box_reference_tests(cle):
    # tests/test_minimum_box.py, test_maximum_box.py, test_top_hat_box.py of the reference
    t = np.zeros((5, 5))
    t[1:4, 1:4] = 1
    ref = np.zeros((5, 5))
    ref[2, 2] = 1
    r = cle.create(cle.push(t))
    cle.minimum_box(cle.push(t), r, 1, 1, 0)
    assert np.array_equal(cle.pull(r), ref)
    cle.maximum_box(cle.push(ref), r, 1, 1, 0)
    assert np.array_equal(cle.pull(r), t)
    h = cle.push(np.asarray([[0, 0, 0, 0, 0], [0, 50, 50, 50, 0], [0, 50, 100, 50, 0], [0, 50, 50, 50, 0],
                             [0, 0, 0, 0, 0]]))
    out = cle.create(h)
    cle.top_hat_box(h, out, 1, 1, 0)
    a = cle.pull(out)
    assert a.min() == 0 and a.max() == 50


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("radii", [(1, 1, 1), (2.5, 0, 3.7), (0, 4, 1), (9, 7, 5), (40, 40, 40)])
def test_box_filters_match_oracle(cle, oracle, shape, radii):
    a = np.random.default_rng(8).normal(100, 30, shape).astype(np.float32)
    assert np.array_equal(cle.pull(cle.minimum_box(a, None, *radii)), oracle.minimum_box(a, *radii))
    assert np.array_equal(cle.pull(cle.maximum_box(a, None, *radii)), oracle.maximum_box(a, *radii))
    assert np.array_equal(cle.pull(cle.top_hat_box(a, None, *radii)), oracle.top_hat_box(a, *radii))


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16])
def test_top_hat_box_narrow_input_and_in_place(cle, oracle, dtype):
    a = np.random.default_rng(9).integers(0, np.iinfo(dtype).max, (13, 70, 61)).astype(dtype)
    assert np.array_equal(cle.pull(cle.top_hat_box(a, None, 5, 5, 2)), oracle.top_hat_box(a.astype(np.float32), 5, 5, 2))
    f = cle.push(a.astype(np.float32))
    cle.top_hat_box(f, f, 5, 5, 2)              # destination = source
    assert np.array_equal(cle.pull(f), oracle.top_hat_box(a.astype(np.float32), 5, 5, 2))


def test_backend_installs_and_delegates(cle):
    """B200Backend as the reference's backend: push / create give device arrays
    the cle.* functions take directly; a kernel outside the path goes to the
    fallback backend and its outputs come back into the device arrays."""
    import numpy as np

    class NumpyArray:
        def __init__(self, a):
            self.a = np.array(a)

        def get(self):
            return self.a

    class FakeFallback:
        """Stands in for the reference's OpenCL backend: runs one kernel in numpy."""
        calls = []

        def from_array(self, a):
            return NumpyArray(a)

        def asarray(self, a):
            return a.a

        def execute(self, anchor, filename, kernel_name, global_size, parameters, **kw):
            self.calls.append(kernel_name)
            assert kernel_name == "add_image_and_scalar"
            parameters["dst"].a[...] = parameters["src"].a + parameters["scalar"]

    be = cle.B200Backend(fallback=FakeFallback())
    backend = cle.Backend.get_instance()
    old = backend.get()
    backend.set(be)
    try:
        assert backend.get().array_type() is cle.B200Array
        src = be.from_array(np.arange(12, dtype=np.float32).reshape(3, 4))
        dst = be.empty_image_like(src)
        be.execute(None, "add_image_and_scalar_x.cl", "add_image_and_scalar", dst.shape,
                   {"src": src, "dst": dst, "scalar": 2.0})
        assert np.array_equal(cle.pull(dst), np.arange(12, dtype=np.float32).reshape(3, 4) + 2)
        # hot-path functions take the backend's arrays without a host copy
        lab = cle.voronoi_otsu_labeling(be.from_array(np.pad(np.ones((5, 5), np.float32), 4)), spot_sigma=1,
                                        outline_sigma=1)
        assert isinstance(lab, cle.B200Array) and cle.pull(lab).max() == 1
        with pytest.raises(NotImplementedError):
            cle.B200Backend().execute(None, "x.cl", "x", (1,), {})
    finally:
        backend.set(old)
