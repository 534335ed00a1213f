"""Parity of the CUDA path (through the cle.* API and the C ABI) with the
oracle on seeded inputs.  Labels, masks, maxima and histograms are compared
bit for bit; the blur is compared bit for bit as well (both sides use the
same float32 fused multiply-add chain); statistics within rtol 1e-5 with the
same NaN/inf pattern."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL_STATS = 1e-5


@pytest.fixture(scope="module")
def cle():
    import pyclesperanto_prototype_b200 as m
    from pyclesperanto_prototype_b200 import _build
    _build.build()
    return m


def rng(seed):
    return np.random.default_rng(seed)


SHAPES_2D = [(1, 1), (1, 7), (7, 1), (5, 6), (31, 33), (64, 100), (257, 130)]
SHAPES_3D = [(1, 1, 1), (1, 5, 6), (3, 1, 9), (7, 11, 13), (17, 40, 35), (33, 64, 70)]


# ---------------------------------------------------------------- blur -----
@pytest.mark.parametrize("shape", SHAPES_2D + SHAPES_3D)
@pytest.mark.parametrize("sig", [(1.0, 1.0, 1.0), (2.0, 0.5, 3.5), (0.0, 1.5, 0.0), (0.1, 0.1, 0.1)])
def test_gaussian_blur_bit_exact(cle, oracle, shape, sig):
    a = rng(1).uniform(0, 1000, size=shape).astype(np.float32)
    got = cle.pull(cle.gaussian_blur(a, None, *sig))
    ref = oracle.gaussian_blur(a, *sig)
    assert got.dtype == np.float32 and np.array_equal(got, ref)


@pytest.mark.parametrize("shape", [(3, 70, 33), (40, 130, 97), (1, 33, 31), (17, 64, 64), (250, 260), (5, 3)])
@pytest.mark.parametrize("sigma", [0.3, 1.0, 1.7, 2.0, 3.5])
def test_gaussian_blur_fused_bit_exact(cle, oracle, shape, sigma):
    # isotropic sigma with radius 1..14 takes the one-launch fused kernel
    a = rng(21).uniform(0, 5000, size=shape).astype(np.float32)
    got = cle.pull(cle.gaussian_blur(a, None, sigma, sigma, sigma))
    assert np.array_equal(got, oracle.gaussian_blur(a, sigma, sigma, sigma))


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16])
def test_gaussian_blur_narrow_input(cle, oracle, dtype):
    a = rng(2).integers(0, np.iinfo(dtype).max, size=(9, 40, 37)).astype(dtype)
    got = cle.pull(cle.gaussian_blur(a, None, 2, 2, 2))
    assert np.array_equal(got, oracle.gaussian_blur(a.astype(np.float32), 2, 2, 2))


# rows of a multiple of 16 bytes and grids of at least two waves of CTAs: the
# fused volume blur stages its planes with TMA copies (boxes starting left of /
# above the image, partial tiles at the right and bottom edges, volumes with
# fewer planes than the z window inside each chunk's halo)
TMA_CASES = [(np.uint16, (96, 700, 1000), 0.8), (np.uint16, (96, 700, 1000), 2.0),
             (np.uint16, (60, 700, 1000), 3.5), (np.uint16, (9, 1030, 4104), 1.7),
             (np.uint8, (80, 700, 1008), 1.0), (np.uint8, (80, 700, 1008), 2.0),
             (np.float32, (64, 700, 1004), 1.0), (np.float32, (64, 700, 1004), 0.3)]


@pytest.mark.parametrize("dtype,shape,sigma", TMA_CASES)
def test_gaussian_blur_tma_staging_bit_exact(cle, oracle, dtype, shape, sigma):
    import torch
    from pyclesperanto_prototype_b200 import _lib
    r = rng(23)
    a = (r.integers(0, np.iinfo(dtype).max, size=shape) if dtype != np.float32
         else r.uniform(0, 5000, size=shape)).astype(dtype)
    src = torch.from_numpy(a).cuda()
    dst = torch.empty(shape, dtype=torch.float32, device="cuda")
    lib = _lib.load()
    s, d = _lib.tensor_desc(src), _lib.tensor_desc(dst)
    ws = torch.empty(lib.cle_gaussian_blur_workspace_bytes(_lib.ref(s)), dtype=torch.uint8, device="cuda")
    stream = _lib.stream_ptr()
    _lib.check(lib.cle_gaussian_blur(_lib.ref(s), _lib.ref(d), sigma, sigma, sigma, ws.data_ptr(), ws.numel(),
                                     stream), "gaussian_blur")
    assert lib.cle_workspace_status(ws.data_ptr(), ws.numel(), stream) == 0
    assert np.array_equal(dst.cpu().numpy(), oracle.gaussian_blur(a.astype(np.float32), sigma, sigma, sigma))


def test_gaussian_blur_reference_test(cle):
    # tests/test_gaussian_blur.py:4-22 of the reference
    t = np.zeros((5, 5))
    t[2, 2] = 100
    r = cle.create(cle.push(t))
    cle.gaussian_blur(t, r, 1, 1, 0)
    a = cle.pull(r)
    assert a.min() > 0 and 15.9 < a.max() < 16


# -------------------------------------------------------------- maxima -----
@pytest.mark.parametrize("shape", SHAPES_2D + SHAPES_3D + [(40, 130, 97)])
@pytest.mark.parametrize("levels", [3, 1000])
def test_detect_maxima_exact(cle, oracle, shape, levels):
    a = rng(3).integers(0, levels, size=shape).astype(np.float32)
    got = cle.pull(cle.detect_maxima_box(a))
    assert got.dtype == np.uint8
    assert np.array_equal(got, oracle.detect_maxima(a))


def test_detect_maxima_reference_test(cle):
    a = np.array([[0, 0, 0, 0, 0], [1, 0, 0, 2, 0], [1, 2, 1, 3, 2], [0, 1, 0, 2, 0], [0, 0, 0, 0, 0]])
    r = np.zeros((5, 5), np.uint8)
    r[2, 1] = r[2, 3] = 1
    out = cle.create_like(cle.push(a))
    cle.detect_maxima_box(a, out)
    assert np.array_equal(cle.pull(out), r)


def test_detect_maxima_large_values(cle, oracle):
    # |v| >= 2^24: v - 1 == v in float32 changes the tie rule
    a = (rng(4).integers(0, 3, size=(6, 9, 8)) * 1.0 + 2.0 ** 25).astype(np.float32)
    assert np.array_equal(cle.pull(cle.detect_maxima_box(a)), oracle.detect_maxima(a))


# ------------------------------------------------- min/max, histogram ------
@pytest.mark.parametrize("shape", [(1, 1), (5, 6), (257, 130), (7, 11, 13), (33, 64, 70)])
def test_min_max_histogram_exact(cle, oracle, shape):
    a = rng(5).normal(100, 30, size=shape).astype(np.float32)
    assert cle.minimum_of_all_pixels(a) == a.min()
    assert cle.maximum_of_all_pixels(a) == a.max()
    h = cle.pull(cle.histogram(a, num_bins=256))
    assert np.array_equal(h, oracle.histogram(a, 256))


@pytest.mark.parametrize("shape", [(64, 100), (9, 50, 64), (3, 128, 256), (5, 7, 1028)])
@pytest.mark.parametrize("bins", [256, 7, 600])
def test_histogram_smooth_image_exact(cle, oracle, shape, bins):
    # rows of a multiple of 4 floats: lanes whose 8 voxels share a bin add
    # them at once, the others add runs of equal bins; plateaus, ramps,
    # noisy patches and values on bin edges exercise both
    r = rng(25)
    a = np.full(shape, 100.0, np.float32)
    ramp = np.linspace(0.0, 1000.0, shape[-1], dtype=np.float32)
    a[..., : shape[-1] // 3] += ramp[: shape[-1] // 3]
    a += (r.uniform(size=shape) < 0.02) * r.normal(0, 300, size=shape).astype(np.float32)
    a.reshape(-1)[:: 97] = 100.0 + 1000.0 * r.integers(0, 8, size=a.size)[:: 97].astype(np.float32) / 7.0
    h = cle.pull(cle.histogram(a, num_bins=bins))
    assert np.array_equal(h, oracle.histogram(a, bins))


@pytest.mark.parametrize("bins", [256, 9])
def test_histogram_nan_inf_given_range(cle, oracle, bins):
    # NaN / +-inf voxels among plateaus of equal values, with the range given
    # (NaN and -inf land in bin 0, +inf and values above the range in none)
    r = rng(26)
    a = np.full((6, 40, 128), 250.0, np.float32)
    a[:, :, 64:] = 700.0
    flat = a.reshape(-1)
    idx = r.choice(flat.size, 300, replace=False)
    flat[idx[:100]] = np.nan
    flat[idx[100:200]] = np.inf
    flat[idx[200:]] = -np.inf
    a[2, 5, :] = 5000.0   # above the range
    h = cle.pull(cle.histogram(a, num_bins=bins, minimum_intensity=100.0, maximum_intensity=1000.0,
                               determine_min_max=False))
    assert np.array_equal(h, oracle.histogram(a, bins, 100.0, 1000.0))


@pytest.mark.parametrize("img", [
    [[1, 2, 4, 4, 2, 3], [3, 3, 4, 4, 5, 5]],
    [[[1, 2, 4, 4, 2, 3]], [[3, 3, 4, 4, 5, 5]]],
    [[[1, 2, 4], [4, 2, 3]], [[3, 3, 4], [4, 5, 5]]],
])
def test_histogram_reference_tests(cle, img):
    assert np.allclose(cle.pull(cle.histogram(np.asarray(img), num_bins=5)), [1, 2, 3, 4, 2])


def test_histogram_row_sum_rounding(cle, oracle):
    # 2^24 + rows: float32 row sums round exactly as the reference's
    a = np.zeros((4100, 4100), np.float32)
    a[0, 0] = 1.0
    assert np.array_equal(cle.pull(cle.histogram(a, num_bins=256)), oracle.histogram(a, 256))


@pytest.mark.parametrize("shape", [(64, 100), (257, 130), (17, 40, 35), (1, 1)])
def test_threshold_otsu_exact(cle, oracle, shape):
    a = (rng(6).gamma(2.0, 40.0, size=shape)).astype(np.float32)
    got = cle.pull(cle.threshold_otsu(a))
    ref, _ = oracle.threshold_otsu(a)
    assert got.dtype == np.uint8 and np.array_equal(got, ref)


def test_threshold_constant_image(cle):
    a = np.full((9, 9), 7.0, np.float32)
    assert cle.pull(cle.threshold_otsu(a)).max() == 0


def test_elementwise(cle, oracle):
    a = rng(7).uniform(0, 10, size=(13, 17, 19)).astype(np.float32)
    b = (rng(8).uniform(size=a.shape) > 0.5).astype(np.float32)
    assert np.array_equal(cle.pull(cle.greater_constant(a, None, 4.5)), oracle.greater_constant(a, 4.5))
    assert np.array_equal(cle.pull(cle.binary_and(a > 5, b)), oracle.binary_and(a > 5, b))
    out = cle.create_labels_like(cle.push(a))
    cle.mask(a, b, out)
    assert np.array_equal(cle.pull(out), np.where(b != 0, a, 0).astype(np.uint32))


# ----------------------------------------------------------------- CCL -----
@pytest.mark.parametrize("shape", SHAPES_2D + SHAPES_3D)
@pytest.mark.parametrize("density", [0.2, 0.55])
def test_ccl_exact(cle, oracle, shape, density):
    b = (rng(9).uniform(size=shape) < density).astype(np.uint8)
    got = cle.pull(cle.connected_components_labeling_box(b))
    assert got.dtype == np.uint32
    assert np.array_equal(got, oracle.connected_components_labeling_box(b))


def test_ccl_reference_test(cle):
    a = np.array([[[1, 0, 1], [1, 0, 0], [0, 0, 1]]])
    assert np.array_equal(cle.pull(cle.connected_components_labeling_box(a)),
                          [[[1, 0, 2], [1, 0, 0], [0, 0, 3]]])


def test_ccl_float32_key_collisions(cle, oracle):
    # keys above 2^24 round in float32; components whose rounded keys collide
    # share a label in the reference -- and here
    shape = (64, 512, 600)
    b = (rng(10).uniform(size=shape) < 0.002).astype(np.uint8)
    ref = oracle.connected_components_labeling_box(b)
    got = cle.pull(cle.connected_components_labeling_box(b))
    assert np.array_equal(got, ref)
    assert ref.max() < len(np.unique(ref)) - 1 + 200000  # sanity
    # collisions do occur at this size
    from scipy.ndimage import label as sclabel
    n_components = sclabel(b, structure=np.ones((3, 3, 3)))[1]
    assert ref.max() < n_components


def test_relabel_sequential(cle, oracle):
    a = np.array([[[1, 2, 3], [1, 6, 6], [7, 8, 9]]])
    out = cle.create_like(cle.push(a))
    cle.relabel_sequential(a, out)
    assert np.array_equal(cle.pull(out), [[[1, 2, 3], [1, 4, 4], [5, 6, 7]]])
    r = rng(11).choice([0, 3, 17, 400, 401, 60000], size=(20, 30, 40)).astype(np.uint32)
    got = cle.pull(cle.relabel_sequential(cle.push_native(r.astype(np.uint16))))
    assert np.array_equal(got, oracle.relabel_sequential(r))


# -------------------------------------------------------- masked Voronoi ---
def test_masked_voronoi_reference_test(cle):
    seeds = np.zeros((1, 6, 6), int)
    seeds[0, 0, 0] = seeds[0, 0, 5] = seeds[0, 5, 0] = seeds[0, 5, 5] = 1
    mask = np.array([[[1, 1, 1, 1, 0, 1], [1, 0, 0, 1, 0, 1], [1, 0, 1, 1, 0, 1], [1, 0, 1, 1, 0, 1],
                      [1, 0, 0, 0, 0, 1], [1, 1, 1, 1, 1, 1]]])
    ref = [[[1, 1, 1, 1, 0, 3], [1, 0, 0, 1, 0, 3], [1, 0, 1, 1, 0, 3], [2, 0, 1, 1, 0, 4],
            [2, 0, 0, 0, 0, 4], [2, 2, 2, 4, 4, 4]]]
    assert np.array_equal(cle.pull(cle.masked_voronoi_labeling(seeds, mask)), ref)


@pytest.mark.parametrize("shape", [(40, 50), (9, 30, 31), (1, 20, 20)])
@pytest.mark.parametrize("mask_values", [(0, 1), (0, 2, 255)])
def test_masked_voronoi_general(cle, oracle, shape, mask_values):
    r = rng(12)
    mask = r.choice(mask_values, size=shape, p=None).astype(np.float32)
    seeds = (r.uniform(size=shape) < 0.03).astype(np.uint8)
    got = cle.pull(cle.masked_voronoi_labeling(seeds, mask))
    assert np.array_equal(got, oracle.masked_voronoi_labeling(seeds, mask))


# ---------------------------------------------------- voronoi_otsu_labeling --
def test_vol_reference_test(cle):
    img = np.array([[0, 0, 1, 1, 0, 0], [0, 1, 8, 9, 1, 0], [0, 1, 7, 6, 1, 0], [0, 0, 1, 1, 1, 0],
                    [0, 0, 1, 1, 1, 0], [0, 0, 1, 8, 7, 1], [0, 0, 1, 1, 1, 0]])
    ref = [[0, 0, 1, 1, 0, 0], [0, 1, 1, 1, 1, 0], [0, 1, 1, 1, 1, 0], [0, 0, 1, 2, 2, 0],
           [0, 0, 0, 2, 2, 0], [0, 0, 2, 2, 2, 0], [0, 0, 0, 2, 2, 0]]
    out = cle.voronoi_otsu_labeling(cle.push(img), spot_sigma=1, outline_sigma=1)
    assert out.dtype == np.uint32 and np.array_equal(cle.pull(out), ref)


@pytest.fixture(scope="module")
def blobs():
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    return np.load(os.path.join(here, "golden", "blobs.npz"))["blobs"]


@pytest.mark.parametrize("spot,outline", [(1, 1), (3.2, 1), (3.5, 2), (2, 2)])
def test_vol_blobs_exact(cle, oracle, blobs, spot, outline):
    got = cle.pull(cle.voronoi_otsu_labeling(blobs, spot_sigma=spot, outline_sigma=outline))
    assert np.array_equal(got, oracle.voronoi_otsu_labeling(blobs.astype(np.float32), spot, outline))


def test_vol_c1_synthetic_exact(cle, oracle):
    from pyclesperanto_prototype_b200 import synthetic
    img = synthetic.blobs_2d((256, 256), 60, seed=0)
    got = cle.pull(cle.voronoi_otsu_labeling(img, spot_sigma=3.5, outline_sigma=1.0))
    ref = oracle.voronoi_otsu_labeling(img, 3.5, 1.0)
    assert np.array_equal(got, ref) and ref.max() > 10


@pytest.mark.parametrize("shape,n", [((24, 96, 112), 40), ((40, 128, 128), 90)])
def test_vol_nuclei_3d_exact(cle, oracle, shape, n):
    from pyclesperanto_prototype_b200 import synthetic
    vol = synthetic.nuclei_volume(shape, n, seed=3)
    got = cle.pull(cle.voronoi_otsu_labeling(vol, spot_sigma=2, outline_sigma=1))
    ref = oracle.voronoi_otsu_labeling(vol.astype(np.float32), 2, 1)
    assert np.array_equal(got, ref) and ref.max() > 5
    # the float32 push path gives the same labels as the native uint16 path
    got32 = cle.pull(cle.voronoi_otsu_labeling(cle.push(vol), spot_sigma=2, outline_sigma=1))
    assert np.array_equal(got32, ref)


@pytest.mark.parametrize("shape,n", [((24, 96, 112), 40), ((9, 70, 62), 12), ((17, 65, 129), 30),
                                     ((5, 33, 31), 6)])
@pytest.mark.parametrize("sigma", [1.0, 2.0])
def test_vol_equal_sigmas_3d_exact(cle, oracle, shape, n, sigma):
    # equal spot and outline sigmas: one blur, maxima and seeds in one pass
    # (even and odd row lengths, partial warps at the right edge)
    from pyclesperanto_prototype_b200 import synthetic
    vol = synthetic.nuclei_volume(shape, n, seed=5)
    got = cle.pull(cle.voronoi_otsu_labeling(vol, spot_sigma=sigma, outline_sigma=sigma))
    ref = oracle.voronoi_otsu_labeling(vol.astype(np.float32), sigma, sigma)
    assert np.array_equal(got, ref) and ref.max() > 1


@pytest.mark.parametrize("shape", [(20, 60, 64), (9, 33, 45), (70, 90)])
def test_vol_equal_sigmas_into_dirty_or_aliased_destination(cle, oracle, shape):
    # equal sigmas with a uint32 destination: the blur clears the label buffer
    # and the seed pass writes only the seeds -- a destination full of other
    # values must come out exactly as a fresh one; a destination sharing the
    # float32 source's memory keeps the seed pass's full write
    import torch
    from pyclesperanto_prototype_b200 import synthetic
    vol = synthetic.nuclei_volume(shape if len(shape) == 3 else (1,) + shape, 12, seed=41)
    vol = vol.reshape(shape).astype(np.float32)
    ref = oracle.voronoi_otsu_labeling(vol, 2, 2)
    dirty = cle.B200Array(torch.full(shape, 0xFFFFFFF0, dtype=torch.uint32, device="cuda"))
    got = cle.pull(cle.voronoi_otsu_labeling(cle.push(vol), dirty, spot_sigma=2, outline_sigma=2))
    assert np.array_equal(got, ref) and ref.max() > 0
    src = torch.from_numpy(vol.copy()).cuda()
    alias = cle.B200Array(src.view(torch.uint32))
    got = cle.pull(cle.voronoi_otsu_labeling(cle.B200Array(src), alias, spot_sigma=2, outline_sigma=2))
    assert np.array_equal(got, ref)


def test_vol_edge_cases(cle):
    assert cle.pull(cle.voronoi_otsu_labeling(np.full((16, 16), 3.0, np.float32))).max() == 0
    assert cle.pull(cle.voronoi_otsu_labeling(np.zeros((1, 1), np.float32))).max() == 0
    out = cle.create_like(cle.push(np.zeros((5, 6))))
    img = np.array([[0, 0, 1, 1, 0, 0], [0, 1, 8, 9, 1, 0], [0, 1, 7, 6, 1, 0], [0, 0, 1, 1, 1, 0],
                    [0, 0, 1, 8, 7, 1]], np.float32)
    cle.voronoi_otsu_labeling(img, out, 1, 1)    # float32 destination
    assert cle.pull(out).dtype == np.float32 and cle.pull(out).max() >= 1


def test_vol_deterministic(cle):
    from pyclesperanto_prototype_b200 import synthetic
    vol = synthetic.nuclei_volume((32, 128, 128), 60, seed=5)
    a = cle.pull(cle.voronoi_otsu_labeling(vol, spot_sigma=2, outline_sigma=1))
    b = cle.pull(cle.voronoi_otsu_labeling(vol, spot_sigma=2, outline_sigma=1))
    assert np.array_equal(a, b)


# ----------------------------------------------------------- statistics ----
def _assert_stats(got, ref):
    assert list(got.keys()) == list(ref.keys())
    for k in ref:
        g, r = np.asarray(got[k]), np.asarray(ref[k])
        assert g.shape == r.shape, k
        assert np.array_equal(np.isnan(g), np.isnan(r)), k
        m = ~np.isnan(r)
        assert np.allclose(g[m], r[m], rtol=RTOL_STATS, atol=0), (k, g[m][:5], r[m][:5])


@pytest.mark.parametrize("shape", [(3, 3), (64, 100), (7, 11, 13), (20, 64, 70)])
def test_statistics_random(cle, oracle, shape):
    r = rng(13)
    lab = r.integers(0, 12, size=shape).astype(np.uint32)
    lab[lab == 5] = 0           # label 5 absent: reference sentinels
    inten = r.uniform(0, 1000, size=shape).astype(np.float32)
    _assert_stats(cle.statistics_of_labelled_pixels(inten, lab), oracle.statistics_of_labelled_pixels(inten, lab))


@pytest.mark.parametrize("shape", [(3, 5, 8), (40, 260), (6, 33, 132), (2, 9, 1024)])
@pytest.mark.parametrize("pattern", ["runs", "random", "stripes"])
@pytest.mark.parametrize("on_device", [True, False])
def test_statistics_row_segments(cle, oracle, shape, pattern, on_device):
    # uint32 rows of a multiple of 4 voxels take the 4-per-lane run passes:
    # runs that cross lanes and 128-voxel segments, single voxels, rows that
    # end inside a segment
    r = rng(27)
    if pattern == "runs":
        lab = np.repeat(r.integers(0, 9, size=shape[:-1] + (shape[-1] // 4 + 1,)), 4 + shape[-1] % 3, axis=-1)
        lab = lab[..., : shape[-1]]
        lab = np.ascontiguousarray(np.broadcast_to(lab, shape) if lab.shape != shape else lab)
    elif pattern == "random":
        lab = r.integers(0, 7, size=shape)
    else:
        lab = (np.arange(shape[-1]) // 37 % 5) * np.ones(shape, np.int64)
    lab = lab.astype(np.uint32)
    inten = r.integers(0, 4000, size=shape).astype(np.uint16)
    import torch
    # uint32 labels on the device, or a numpy label image (pushed as float32)
    dlab = cle.B200Array(torch.from_numpy(lab).cuda()) if on_device else lab
    _assert_stats(cle.statistics_of_labelled_pixels(inten, dlab),
                  oracle.statistics_of_labelled_pixels(inten.astype(np.float32), lab))


def test_statistics_reference_tables(cle, oracle):
    inten = np.array([[0, 1, 2], [1, 2, 3], [2, 3, 4]])
    lab = np.array([[1, 1, 2], [1, 2, 2], [3, 3, 3]])
    _assert_stats(cle.statistics_of_labelled_pixels(inten, lab), oracle.statistics_of_labelled_pixels(inten, lab))
    s = cle.statistics_of_labelled_pixels(inten, lab)
    assert np.allclose(s["standard_deviation_intensity"], [0.47140452, 0.4714045, 0.8164966], rtol=1e-4)


def test_statistics_on_vol_labels(cle, oracle, blobs):
    lab = cle.voronoi_otsu_labeling(blobs, spot_sigma=3.5)
    got = cle.statistics_of_labelled_pixels(blobs, lab)
    ref = oracle.statistics_of_labelled_pixels(blobs, cle.pull(lab))
    _assert_stats(got, ref)
    assert len(got["label"]) == 65


# ------------------------------------------ active-front (brick) growth -----
def _binary_case(shape, seed, density, seed_density):
    r = rng(seed)
    mask = (r.uniform(size=shape) < density).astype(np.uint8)
    seeds = ((r.uniform(size=shape) < seed_density) & (mask == 1)).astype(np.uint8)
    return seeds, mask


@pytest.mark.parametrize("shape", [(1, 1), (3, 40), (45, 70), (130, 97), (1, 33, 31), (9, 30, 31),
                                   (20, 65, 67), (33, 64, 96)])
@pytest.mark.parametrize("density", [0.35, 0.8, 1.0])
def test_masked_voronoi_binary_exact(cle, oracle, shape, density):
    seeds, mask = _binary_case(shape, 31, density, 0.002)
    got = cle.pull(cle.masked_voronoi_labeling_binary(seeds, mask))
    ref = oracle.masked_voronoi_labeling(seeds, mask)
    assert np.array_equal(got, ref)
    # the general dense path agrees as well
    assert np.array_equal(cle.pull(cle.masked_voronoi_labeling(seeds, mask)), ref)


def test_masked_voronoi_binary_diagonal_stop(cle, oracle):
    # a diagonal-only mask path: a face step changes nothing before the next
    # box step would, so the reference stops and the rest stays 0
    n = 40
    mask = np.zeros((n, n), np.uint8)
    for i in range(n):
        mask[i, i] = 1
    mask[0, 1] = 1
    seeds = np.zeros_like(mask)
    seeds[0, 0] = 1
    ref, steps = oracle.masked_voronoi_labeling(seeds, mask, return_steps=True)
    got = cle.pull(cle.masked_voronoi_labeling_binary(seeds, mask))
    assert np.array_equal(got, ref)
    assert (ref > 0).sum() < mask.sum()      # growth stopped early, as in the reference


def _snake(length, width=40):
    """A one-voxel-wide serpentine path of `length` voxels in plane z = 1 of a
    3-plane volume (rows y = 1, 3, 5, ... joined at alternating ends), seeded at
    its start: the growth needs about `length` steps."""
    rows = (length + width - 1) // width + 1
    mask = np.zeros((3, 2 * rows + 2, width), np.uint8)
    n, y, left = 0, 1, True
    while n < length:
        xs = range(width) if left else range(width - 1, -1, -1)
        for x in xs:
            if n == length:
                break
            mask[1, y, x] = 1
            n += 1
        if n < length:
            mask[1, y + 1, width - 1 if left else 0] = 1
            n += 1
        y += 2
        left = not left
    seeds = np.zeros_like(mask)
    seeds[1, 1, 0] = 1
    return seeds, mask


def _path_order(plane):
    # the path's voxels from its start (y 1, x 0), by walking face neighbours
    y, x = 1, 0
    seen, out = {(y, x)}, [(y, x)]
    while True:
        nxt = [(y + dy, x + dx) for dy, dx in ((0, 1), (0, -1), (1, 0), (-1, 0))
               if 0 <= y + dy < plane.shape[0] and 0 <= x + dx < plane.shape[1]
               and plane[y + dy, x + dx] and (y + dy, x + dx) not in seen]
        if not nxt:
            return out
        y, x = nxt[0]
        seen.add((y, x))
        out.append((y, x))


@pytest.mark.parametrize("length", [60, 247, 249, 252, 254, 257, 600])
def test_masked_voronoi_binary_long_path(cle, oracle, length):
    # paths around the arrival-step limit of the key growth (120 steps, above
    # which the step-by-step brick growth takes over), with a second seed a
    # few voxels before the path's end so two labels meet on the path
    seeds, mask = _snake(length)
    path = _path_order(mask[1])
    y, x = path[-6]
    seeds[1, y, x] = 1
    ref, steps = oracle.masked_voronoi_labeling(seeds, mask, return_steps=True)
    got = cle.pull(cle.masked_voronoi_labeling_binary(seeds, mask))
    assert np.array_equal(got, ref)
    assert (ref > 0).sum() == mask.sum()


def test_masked_voronoi_binary_many_seeds_3d(cle, oracle):
    seeds, mask = _binary_case((24, 100, 70), 32, 0.6, 0.02)
    got = cle.pull(cle.masked_voronoi_labeling_binary(seeds, mask))
    assert np.array_equal(got, oracle.masked_voronoi_labeling(seeds, mask))


def test_masked_voronoi_binary_dense_seeds(cle, oracle):
    # tens of thousands of seeds: many per CTA in the seed queueing round
    seeds, mask = _binary_case((32, 256, 256), 33, 0.7, 0.01)
    assert seeds.sum() > 10000
    got = cle.pull(cle.masked_voronoi_labeling_binary(seeds, mask))
    assert np.array_equal(got, oracle.masked_voronoi_labeling(seeds, mask))
