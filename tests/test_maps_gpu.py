"""Parametric label maps, replace_intensities, add_image_and_scalar and the
statistics table formats on the device: the reference's own fixtures, and the
maps against the oracle's statistics of labels + 1 on seeded label images
(rtol 1e-5 like every statistics comparison, same NaN / inf positions)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

RTOL = 1e-5


@pytest.fixture(scope="module")
def cle():
    import pyclesperanto_prototype_b200 as m
    from pyclesperanto_prototype_b200 import _build
    _build.build()
    return m


LAB2 = np.asarray([[1, 1, 2], [1, 0, 0], [3, 3, 0]])
INT2 = np.asarray([[1, 1, 2], [4, 0, 0], [5, 3, 0]])


def _close(a, b, rtol=1e-3):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.array_equal(np.isnan(a), np.isnan(b)) and np.allclose(a[~np.isnan(a)], b[~np.isnan(b)], rtol)


# ---- the reference's fixtures (tests/test_label_*_map.py and friends) -----
def test_replace_intensities_reference_test(cle):
    src = cle.push(np.asarray([[0, 0, 0, 0, 0], [0, 1, 2, 3, 0], [0, 2, 3, 4, 0], [0, 4, 4, 5, 0],
                               [0, 0, 0, 0, 0]]))
    vec = cle.push(np.asarray([[0, 9, 8, 7, 6, 5]]))
    out = cle.create(src)
    cle.replace_intensities(src, vec, out)
    ref = [[0, 0, 0, 0, 0], [0, 9, 8, 7, 0], [0, 8, 7, 6, 0], [0, 6, 6, 5, 0], [0, 0, 0, 0, 0]]
    assert np.allclose(cle.pull(out), ref)


@pytest.mark.parametrize("three_d", [False, True])
def test_label_maps_reference_tests(cle, three_d):
    lab, inten = LAB2, INT2
    if three_d:                         # the 3D fixtures are the 2D ones as 3 planes of one row
        lab, inten = lab[:, None, :], inten[:, None, :]
    lab_r = lab.copy()
    lab_r[1, ..., 2] = 2                # the extension-ratio fixture's labels
    cases = [
        (cle.label_mean_intensity_map(cle.push(inten), cle.push(lab)), [[2, 2, 2], [2, 0, 0], [4, 4, 0]]),
        (cle.label_pixel_count_map(cle.push(lab)), [[3, 3, 1], [3, 0, 0], [2, 2, 0]]),
        (cle.label_maximum_extension_map(cle.push(lab)),
         [[0.74535596, 0.74535596, 0], [0.74535596, 0, 0], [0.5, 0.5, 0]]),
        (cle.label_mean_extension_map(cle.push(lab)),
         [[0.65403885, 0.65403885, 0], [0.65403885, 0, 0], [0.5, 0.5, 0]]),
        (cle.label_maximum_extension_ratio_map(cle.push(lab_r)),
         [[1.1396203, 1.1396203, 1], [1.1396203, 0, 1], [1, 1, 0]]),
        (cle.label_standard_deviation_intensity_map(cle.push(inten), cle.push(lab)),
         [[1.4142, 1.4142, 0], [1.4142, 0, 0], [1, 1, 0]]),
    ]
    for out, ref in cases:
        ref = np.asarray(ref, np.float64)
        if three_d:
            ref = ref[:, None, :]
        assert np.allclose(cle.pull(out), ref, 0.001)


def test_statistics_of_background_and_labelled_pixels_reference_test(cle):
    # tests/test_statistics_of_background_and_labelled_pixels.py: the table through push_regionprops
    intensity = cle.push(np.asarray([[0, 1, 2], [1, 2, 3], [2, 3, 4]]))
    labels = cle.push(np.asarray([[0, 0, 1], [0, 1, 1], [2, 2, 2]]))
    ref = np.asarray([
        [0, 1, 2], [0, 1, 0], [0, 0, 2], [0, 0, 0], [1, 2, 2], [1, 1, 2], [0, 0, 0], [2, 2, 3], [2, 2, 1],
        [1, 1, 1], [0, 2, 2], [1, 3, 4], [0.6666667, 2.3333333, 3], [2, 7, 9],
        [0.47140452, 0.4714045, 0.8164966], [3, 3, 3], [1, 12, 11], [1, 5, 18], [0, 0, 0],
        [0.5, 1.7142857, 1.2222222], [0.5, 0.71428573, 2], [0, 0, 0], [1, 5, 3], [1, 2, 6], [0, 0, 0],
        [0.33333334, 1.6666666, 1], [0.33333334, 0.6666667, 2], [0, 0, 0],
        [2.1213202, 1.9426796, 2.2222223], [0.70710677, 0.6475599, 0.7407408],
        [0.70710677, 0.7693094, 1.2222222], [1, 1.1880127, 1.6499999], [1.9621165, 1.9621165, 2],
        [0.65403885, 0.65403885, 0.6666667], [0.74535596, 0.745356, 1], [1.1396203, 1.1396204, 1.5]])
    props = cle.statistics_of_background_and_labelled_pixels(intensity, labels)
    table = cle.pull(cle.push_regionprops(props, first_row_index=0))
    assert table.shape == (36, 3)
    assert np.allclose(table, ref, 0.0001)
    assert cle.STATISTICS_ENTRY.MEAN_DISTANCE_TO_CENTROID.value == 33


def test_push_regionprops_column_reference_test(cle):
    labels = cle.push(np.asarray([[[4, 4, 2]], [[4, 1, 2]], [[3, 3, 4]]]))
    props = cle.statistics_of_background_and_labelled_pixels(None, labels)
    assert np.allclose(cle.pull(cle.push_regionprops_column(props, "area")), [[0, 1, 2, 2, 4]])


def test_add_image_and_scalar(cle):
    a = np.random.default_rng(1).normal(0, 100, (7, 33, 40)).astype(np.float32)
    assert np.array_equal(cle.pull(cle.add_image_and_scalar(a, None, 2.5)), a + np.float32(2.5))


# ---- maps against the oracle ---------------------------------------------
MAPS = [("label_pixel_count_map", "area", False), ("label_mean_intensity_map", "mean_intensity", True),
        ("label_minimum_intensity_map", "min_intensity", True),
        ("label_maximum_intensity_map", "max_intensity", True),
        ("label_standard_deviation_intensity_map", "standard_deviation_intensity", True),
        ("label_mean_extension_map", "mean_distance_to_centroid", False),
        ("label_maximum_extension_map", "max_distance_to_centroid", False),
        ("label_maximum_extension_ratio_map", "mean_max_distance_to_centroid_ratio", False)]


def _oracle_map(oracle, inten, lab, key):
    temp = lab.astype(np.uint32) + 1
    props = oracle.statistics_of_labelled_pixels(inten if inten is not None else temp.astype(np.float32), temp)
    vec = np.asarray(props[key], np.float32).copy()
    vec[0] = 0
    return vec[lab.astype(np.int64)]


@pytest.mark.parametrize("shape", [(40, 70), (6, 33, 50), (1, 5, 7), (130, 97)])
@pytest.mark.parametrize("name,key,with_intensity", MAPS)
def test_label_maps_match_oracle(cle, oracle, shape, name, key, with_intensity):
    rng = np.random.default_rng(2)
    lab = rng.integers(0, 12, shape).astype(np.uint32)
    lab[lab == 5] = 0                   # a gap: label 5 absent
    inten = rng.normal(200, 50, shape).astype(np.float32)
    fn = getattr(cle, name)
    got = cle.pull(fn(inten, lab) if with_intensity else fn(lab))
    ref = _oracle_map(oracle, inten if with_intensity else None, lab, key)
    assert _close(got, ref, RTOL)


# ---- euclidean_distance_from_label_centroid_map ---------------------------
def test_euclidean_distance_from_label_centroid_map_reference_test(cle):
    # tests/test_euclidean_distance_from_label_centroid_map.py:4-34
    labels = np.asarray([[1, 1, 1, 2], [1, 1, 1, 2], [1, 1, 1, 2], [2, 2, 2, 2]])
    ref = np.asarray([[1.4142135, 1, 1.4142135, 2.3079278], [1, 0, 1, 1.4285713],
                      [1.4142135, 1, 1.4142135, 0.86896616], [2.3079278, 1.4285713, 0.86896616, 1.2121831]])
    got = cle.pull(cle.euclidean_distance_from_label_centroid_map(cle.push(labels)))
    assert np.allclose(got, ref, 0.001)


@pytest.mark.parametrize("shape", [(40, 70), (6, 33, 50), (1, 5, 7), (130, 97), (1, 1)])
def test_euclidean_distance_from_label_centroid_map_matches_oracle(cle, oracle, shape):
    rng = np.random.default_rng(3)
    lab = rng.integers(0, 9, shape).astype(np.uint32)
    lab[lab == 4] = 0                   # a gap: label 4 absent
    got = cle.pull(cle.euclidean_distance_from_label_centroid_map(lab))
    ref = oracle.euclidean_distance_from_label_centroid_map(lab)
    assert got.dtype == np.float32 and got.shape == ref.shape
    assert np.allclose(got, ref, rtol=RTOL, atol=1e-6)
    assert np.all(got[lab == 0] == 0)


@pytest.mark.parametrize("device_int32", [False, True])
def test_euclidean_distance_negative_labels(cle, oracle, device_int32):
    """int32 labels below 0: the label read clamps to the point list's column 0,
    so such a pixel gets its distance to the background's centroid (label-0
    pixels stay 0) -- the same rule in the kernel and the oracle."""
    rng = np.random.default_rng(5)
    lab = rng.integers(-3, 7, (5, 21, 34)).astype(np.int32)
    arg = cle.B200Array(torch.from_numpy(lab).cuda()) if device_int32 else lab
    got = cle.pull(cle.euclidean_distance_from_label_centroid_map(arg))
    ref = oracle.euclidean_distance_from_label_centroid_map(lab)
    assert np.allclose(got, ref, rtol=RTOL, atol=1e-5)
    assert np.all(got[lab == 0] == 0) and np.all(got[lab < 0] > 0)


def test_centroids_of_labels_point_lists(cle, oracle):
    rng = np.random.default_rng(4)
    lab = rng.integers(0, 6, (5, 20, 30)).astype(np.uint32)
    lab[lab == 2] = 0
    st = oracle.statistics_of_labelled_pixels(np.zeros(lab.shape, np.float32), lab)
    ref = np.stack([st["centroid_x"], st["centroid_y"], st["centroid_z"]])
    with_bg = cle.pull(cle.centroids_of_background_and_labels(lab))
    without = cle.pull(cle.centroids_of_labels(lab))
    assert with_bg.shape == (3, 6) and without.shape == (3, 5)
    assert _close(without, ref, RTOL)
    assert _close(with_bg[:, 1:], ref, RTOL)
    bg = np.argwhere(lab == 0)
    assert np.allclose(with_bg[:, 0], bg[:, ::-1].mean(axis=0), rtol=RTOL)


@pytest.mark.parametrize("shape", [(40, 100), (6, 33, 70)])
def test_centroids_of_labels_device_runs(cle, oracle, shape):
    # uint32 labels on the device with runs longer than a warp's 32 voxels and
    # an absent label (NaN column): one pass of per-run coordinate sums
    import torch
    rng = np.random.default_rng(6)
    lab = np.repeat(rng.integers(0, 7, size=shape[:-1] + (shape[-1] // 9 + 1,)), 9, axis=-1)[..., :shape[-1]]
    lab = np.ascontiguousarray(lab).astype(np.uint32)
    lab[lab == 3] = 0
    st = oracle.statistics_of_labelled_pixels(np.zeros(lab.shape, np.float32), lab)
    keys = ["centroid_x", "centroid_y", "centroid_z"][:len(shape)]
    ref = np.stack([st[k] for k in keys])
    got = cle.pull(cle.centroids_of_labels(cle.B200Array(torch.from_numpy(lab).cuda())))
    assert got.shape == ref.shape
    assert _close(got, ref, RTOL)
    assert np.all(np.isnan(got[:, 2]))   # label 3 is absent


# ---- neighbour-distance maps and their matrices ---------------------------
QUAD = np.asarray([[1, 1, 1, 3, 3, 3], [1, 1, 1, 3, 3, 3], [1, 1, 1, 3, 3, 3],
                   [0, 0, 0, 2, 2, 2], [0, 0, 0, 2, 2, 2], [0, 0, 0, 2, 2, 2]])
SPA = np.asarray([[1, 0, 0, 0, 0, 3], [0] * 6, [0] * 6, [0] * 6, [0] * 6, [0, 0, 0, 0, 0, 2]])
SPB = np.asarray([[0, 2, 0, 0, 0, 3], [1, 0, 0, 0, 0, 0], [0] * 6, [0] * 6, [0, 0, 0, 0, 0, 4],
                  [0, 0, 0, 0, 5, 0]])


def test_neighbor_maps_reference_tests(cle):
    # tests/test_average_distance_of_n_nearest_neighbors.py,
    # tests/test_average_neighbor_distance_map.py,
    # tests/test_average_distance_to_n_nearest_other_labels_map.py (rtol 0.01)
    got = cle.pull(cle.average_distance_of_n_nearest_neighbors_map(cle.push(QUAD), n=2))
    assert np.allclose(got, [[3.62] * 3 + [3] * 3] * 3 + [[0] * 3 + [3.62] * 3] * 3, 0.01)
    got = cle.pull(cle.average_neighbor_distance_map(cle.push(QUAD)))
    assert np.allclose(got, [[3] * 6] * 3 + [[0] * 3 + [3] * 3] * 3, 0.01)
    got = cle.pull(cle.average_distance_to_n_nearest_other_labels_map(cle.push(SPA), cle.push(SPB), n=1))
    ref = np.zeros((6, 6))
    ref[0, 0] = ref[5, 5] = 1
    assert np.allclose(got, ref, 0.01)


def test_neighbor_matrices_reference_tests(cle):
    # tests/test_generate_touch_matrix.py, test_average_distance_of_n_shortest_distances.py,
    # test_average_distance_of_touching_neighbors.py, test_average_distance_of_n_nearest_distances.py
    lab = np.asarray([[1, 1, 0, 0, 0], [1, 1, 0, 3, 0], [0, 2, 2, 3, 0], [0, 2, 2, 0, 0], [0, 0, 0, 0, 4]])
    ref = np.asarray([[0, 1, 1, 1, 1], [1, 0, 1, 0, 0], [1, 1, 0, 1, 0], [1, 0, 1, 0, 0], [1, 0, 0, 0, 0]]).T
    assert np.array_equal(cle.pull(cle.generate_touch_matrix(cle.push(lab))), ref)
    c = cle.centroids_of_labels(cle.push(QUAD))
    D = cle.generate_distance_matrix(c, c)
    assert np.allclose(cle.pull(cle.average_distance_of_n_shortest_distances(D, n=1)), [[0, 3, 3, 3]], 0.01)
    T = cle.generate_touch_matrix(cle.push(QUAD))
    assert np.allclose(cle.pull(cle.average_distance_of_touching_neighbors(D, T)), [[0, 3, 3, 3]], 0.01)
    D2 = cle.generate_distance_matrix(cle.centroids_of_labels(cle.push(SPA)), cle.centroids_of_labels(cle.push(SPB)))
    assert np.allclose(cle.pull(cle.average_distance_of_n_nearest_distances(D2, n=1)), [[0, 1, 1, 0]], 0.01)


def _voronoi_labels(shape, n, seed, gaps=False):
    # touching labels: every voxel to its nearest of n random points (1..n),
    # optionally with some labels dropped (absent labels: NaN centroids)
    r = np.random.default_rng(seed)
    pts = np.stack([r.integers(0, s, n) for s in shape], 1)
    grid = np.stack(np.indices(shape), -1).reshape(-1, len(shape))
    d2 = ((grid[:, None, :] - pts[None, :, :]) ** 2).sum(-1)
    lab = (np.argmin(d2, 1) + 1).reshape(shape).astype(np.uint32)
    lab[r.uniform(size=shape) < 0.15] = 0
    if gaps:
        for k in r.choice(np.arange(1, n + 1), n // 5, replace=False):
            lab[lab == k] = 0
    return lab


@pytest.mark.parametrize("shape,n,gaps", [((60, 70), 40, False), ((60, 70), 40, True),
                                          ((12, 30, 34), 60, False), ((12, 30, 34), 60, True)])
def test_neighbor_matrices_match_oracle(cle, oracle, shape, n, gaps):
    lab = _voronoi_labels(shape, n, 21, gaps).astype(np.float32)
    c = oracle.centroids_of_labels(lab)
    got_c = cle.pull(cle.centroids_of_labels(cle.push(lab)))
    assert _close(got_c, c, 1e-6)
    D = oracle.generate_distance_matrix(c, c)
    Dg = cle.generate_distance_matrix(cle.push(c), cle.push(c))
    assert np.array_equal(np.isnan(cle.pull(Dg)), np.isnan(D))
    assert np.array_equal(cle.pull(Dg)[~np.isnan(D)], D[~np.isnan(D)])       # bit for bit
    T = oracle.generate_touch_matrix(lab)
    Tg = cle.generate_touch_matrix(cle.push(lab))
    assert np.array_equal(cle.pull(Tg), T)
    for k in (1, 3, 7):
        assert _close(cle.pull(cle.average_distance_of_n_shortest_distances(Dg, n=k)),
                      oracle.average_distance_of_n_shortest_distances(D, k), 1e-6)
        assert _close(cle.pull(cle.average_distance_of_n_nearest_distances(Dg, n=k)),
                      oracle.average_distance_of_n_nearest_distances(D, k), 1e-6)
    assert _close(cle.pull(cle.average_distance_of_touching_neighbors(Dg, Tg)),
                  oracle.average_distance_of_touching_neighbors(D, T), 1e-6)


@pytest.mark.parametrize("shape,n,gaps", [((60, 70), 40, False), ((60, 70), 40, True),
                                          ((12, 30, 34), 60, False), ((12, 30, 34), 60, True)])
@pytest.mark.parametrize("k", [1, 4])
def test_neighbor_maps_match_oracle(cle, oracle, shape, n, gaps, k):
    lab = _voronoi_labels(shape, n, 22, gaps)
    other = _voronoi_labels(shape, n // 2, 23, False)
    src = cle.push(lab.astype(np.float32))
    assert _close(cle.pull(cle.average_distance_of_n_nearest_neighbors_map(src, n=k)),
                  oracle.average_distance_of_n_nearest_neighbors_map(lab, k), 1e-6)
    assert _close(cle.pull(cle.average_distance_to_n_nearest_other_labels_map(src, cle.push(other.astype(np.float32)), n=k)),
                  oracle.average_distance_to_n_nearest_other_labels_map(lab, other, k), 1e-6)
    assert _close(cle.pull(cle.average_neighbor_distance_map(src)),
                  oracle.average_neighbor_distance_map(lab), 1e-6)


def test_neighbor_maps_on_device_uint32_labels(cle, oracle):
    # uint32 device labels (the output of voronoi_otsu_labeling): the map is
    # replace_intensities' destination, made by create_like -- float32 whatever
    # the labels' type, as _tier0/_create.py create_like makes it
    lab = _voronoi_labels((40, 50), 30, 24)
    t = cle.B200Array(torch.from_numpy(lab).cuda())
    out = cle.average_neighbor_distance_map(t)
    assert out.dtype == np.float32
    assert _close(cle.pull(out), oracle.average_neighbor_distance_map(lab), 1e-6)
    out = cle.average_distance_of_n_nearest_neighbors_map(t, n=3)
    assert _close(cle.pull(out), oracle.average_distance_of_n_nearest_neighbors_map(lab, 3), 1e-6)


def test_n_distances_rejects_large_n(cle):
    c = cle.centroids_of_labels(cle.push(QUAD))
    D = cle.generate_distance_matrix(c, c)
    with pytest.raises(ValueError):
        cle.average_distance_of_n_shortest_distances(D, n=1001)


def test_neighbor_maps_without_labels(cle, oracle):
    # an image without labels (empty point lists): the reference kernels'
    # means over no rows are NaN, a label touching nothing gets 0
    zero = np.zeros((6, 7), np.float32)
    some = np.zeros((6, 7), np.float32)
    some[1:3, 2:4] = 1
    some[4, 5] = 2
    for lab, other in ((zero, zero), (zero, some), (some, zero)):
        got = cle.pull(cle.average_distance_of_n_nearest_neighbors_map(cle.push(lab), n=2))
        assert _close(got, oracle.average_distance_of_n_nearest_neighbors_map(lab, 2))
        got = cle.pull(cle.average_distance_to_n_nearest_other_labels_map(cle.push(lab), cle.push(other), n=1))
        assert _close(got, oracle.average_distance_to_n_nearest_other_labels_map(lab, other, 1))
        got = cle.pull(cle.average_neighbor_distance_map(cle.push(lab)))
        assert _close(got, oracle.average_neighbor_distance_map(lab))
