"""The oracle against every golden vector the reference's own tests hold for
this path, and against the demo-notebook known answers on blobs.tif
(tests/golden/, generated by tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_voronoi_otsu_labeling_golden(oracle):
    # tests/test_voronoi_otsu_labeling.py:4-39
    img = np.array([[0, 0, 1, 1, 0, 0], [0, 1, 8, 9, 1, 0], [0, 1, 7, 6, 1, 0], [0, 0, 1, 1, 1, 0],
                    [0, 0, 1, 1, 1, 0], [0, 0, 1, 8, 7, 1], [0, 0, 1, 1, 1, 0]])
    ref = np.array([[0, 0, 1, 1, 0, 0], [0, 1, 1, 1, 1, 0], [0, 1, 1, 1, 1, 0], [0, 0, 1, 2, 2, 0],
                    [0, 0, 0, 2, 2, 0], [0, 0, 2, 2, 2, 0], [0, 0, 0, 2, 2, 0]])
    assert np.array_equal(oracle.voronoi_otsu_labeling(img, 1, 1), ref)


def test_gaussian_blur_golden(oracle):
    # tests/test_gaussian_blur.py:4-22
    t = np.zeros((5, 5))
    t[2, 2] = 100
    a = oracle.gaussian_blur(t, 1, 1, 0)
    assert a.min() > 0 and 15.9 < a.max() < 16


def test_kernel_sizes(oracle):
    # _tier0/_sigma_to_kernel_size.py:1-4
    assert [oracle.sigma_to_kernel_size(s) for s in (1, 2, 3.5, 0.1, 1.125, 3.2)] == [9, 17, 29, 1, 9, 25]
    w = oracle.gauss_weights(2.0)
    assert w.dtype == np.float32 and abs(float(w.astype(np.float64).sum()) - 1) < 1e-6
    assert np.array_equal(w, w[::-1])


@pytest.mark.parametrize("img", [
    [[1, 2, 4, 4, 2, 3], [3, 3, 4, 4, 5, 5]],
    [[[1, 2, 4, 4, 2, 3]], [[3, 3, 4, 4, 5, 5]]],
    [[[1, 2, 4], [4, 2, 3]], [[3, 3, 4], [4, 5, 5]]],
])
def test_histogram_golden(oracle, img):
    # tests/test_histogram.py:4-56
    assert np.allclose(oracle.histogram(np.asarray(img), 5), [1, 2, 3, 4, 2])


def test_detect_maxima_golden(oracle):
    # tests/test_detect_maxima_box.py:4-35
    a = np.array([[0, 0, 0, 0, 0], [1, 0, 0, 2, 0], [1, 2, 1, 3, 2], [0, 1, 0, 2, 0], [0, 0, 0, 0, 0]])
    r = np.zeros((5, 5), np.uint8)
    r[2, 1] = r[2, 3] = 1
    assert np.array_equal(oracle.detect_maxima(a), r)


def test_ccl_golden(oracle):
    # tests/test_connected_components_labeling_box.py:6-32
    a = np.array([[[1, 0, 1], [1, 0, 0], [0, 0, 1]]])
    r = np.array([[[1, 0, 2], [1, 0, 0], [0, 0, 3]]])
    assert np.array_equal(oracle.connected_components_labeling_box(a), r)


def test_pixel_index_key_order(oracle):
    # tests/test_set_nonzero_pixels_to_pixelindex.py:4-26: key = x*H + y + 1,
    # so isolated pixels are numbered column by column
    a = np.array([[0, 0, 0, 1], [0, 0, 1, 0], [0, 0, 0, 0], [1, 0, 1, 0]])
    lab = oracle.connected_components_labeling_box(a)
    # components: {(0,3),(1,2)} connected diagonally, (3,0), (3,2)
    assert lab[3, 0] == 1 and lab[1, 2] == 2 and lab[0, 3] == 2 and lab[3, 2] == 3


def test_masked_voronoi_golden(oracle):
    # tests/test_masked_voronoi_labeling.py:4-46
    seeds = np.zeros((1, 6, 6), int)
    seeds[0, 0, 0] = seeds[0, 0, 5] = seeds[0, 5, 0] = seeds[0, 5, 5] = 1
    mask = np.array([[[1, 1, 1, 1, 0, 1], [1, 0, 0, 1, 0, 1], [1, 0, 1, 1, 0, 1], [1, 0, 1, 1, 0, 1],
                      [1, 0, 0, 0, 0, 1], [1, 1, 1, 1, 1, 1]]])
    ref = np.array([[[1, 1, 1, 1, 0, 3], [1, 0, 0, 1, 0, 3], [1, 0, 1, 1, 0, 3], [2, 0, 1, 1, 0, 4],
                     [2, 0, 0, 0, 0, 4], [2, 2, 2, 4, 4, 4]]])
    assert np.array_equal(oracle.masked_voronoi_labeling(seeds, mask), ref)


def test_relabel_golden(oracle):
    # tests/test_relabel_sequential.py:4-32
    a = np.array([[[1, 2, 3], [1, 6, 6], [7, 8, 9]]])
    r = np.array([[[1, 2, 3], [1, 4, 4], [5, 6, 7]]])
    assert np.array_equal(oracle.relabel_sequential(a), r)


_STATS_REF_2D = {  # tests/test_statistics_of_labelled_pixels.py:5-110 (push_regionprops rows)
    "bbox_min_x": [0, 1, 0], "bbox_min_y": [0, 0, 2], "bbox_min_z": [0, 0, 0],
    "bbox_max_x": [1, 2, 2], "bbox_max_y": [1, 1, 2], "bbox_max_z": [0, 0, 0],
    "bbox_width": [2, 2, 3], "bbox_height": [2, 2, 1], "bbox_depth": [1, 1, 1],
    "min_intensity": [0, 2, 2], "max_intensity": [1, 3, 4],
    "mean_intensity": [0.6666667, 2.3333333, 3.], "sum_intensity": [2, 7, 9],
    "standard_deviation_intensity": [0.47140452, 0.4714045, 0.8164966], "area": [3, 3, 3],
    "sum_intensity_times_x": [1, 12, 11], "sum_intensity_times_y": [1, 5, 18],
    "sum_intensity_times_z": [0, 0, 0], "mass_center_x": [0.5, 1.7142857, 1.2222222],
    "mass_center_y": [0.5, 0.71428573, 2.], "mass_center_z": [0, 0, 0],
    "sum_x": [1, 5, 3], "sum_y": [1, 2, 6], "sum_z": [0, 0, 0],
    "centroid_x": [0.33333334, 1.6666666, 1.], "centroid_y": [0.33333334, 0.6666667, 2.],
    "centroid_z": [0, 0, 0],
    "sum_distance_to_mass_center": [2.1213202, 1.9426796, 2.2222223],
    "mean_distance_to_mass_center": [0.70710677, 0.6475599, 0.7407408],
    "max_distance_to_mass_center": [0.70710677, 0.7693094, 1.2222222],
    "mean_max_distance_to_mass_center_ratio": [1., 1.1880127, 1.6499999],
    "sum_distance_to_centroid": [1.9621165, 1.9621165, 2.],
    "mean_distance_to_centroid": [0.65403885, 0.65403885, 0.6666667],
    "max_distance_to_centroid": [0.74535596, 0.745356, 1.],
    "mean_max_distance_to_centroid_ratio": [1.1396203, 1.1396204, 1.5],
}


def _swap_yz(d):
    out = dict(d)
    for a, b in (("bbox_min_y", "bbox_min_z"), ("bbox_max_y", "bbox_max_z"), ("bbox_height", "bbox_depth"),
                 ("sum_intensity_times_y", "sum_intensity_times_z"), ("mass_center_y", "mass_center_z"),
                 ("sum_y", "sum_z"), ("centroid_y", "centroid_z")):
        out[a], out[b] = d[b], d[a]
    return out


@pytest.mark.parametrize("three_d", [False, True])
def test_statistics_golden(oracle, three_d):
    inten = np.array([[0, 1, 2], [1, 2, 3], [2, 3, 4]])
    lab = np.array([[1, 1, 2], [1, 2, 2], [3, 3, 3]])
    ref = _STATS_REF_2D
    if three_d:  # tests/test_statistics_of_labelled_pixels.py:112-230 (rows become z)
        inten, lab, ref = inten[:, None, :], lab[:, None, :], _swap_yz(_STATS_REF_2D)
    s = oracle.statistics_of_labelled_pixels(inten, lab)
    assert list(s["label"]) == [1, 2, 3]
    for k, v in ref.items():
        assert np.allclose(s[k], v, rtol=1e-4), k


def _known():
    with open(os.path.join(HERE, "golden", "known_answers.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def blobs():
    return np.load(os.path.join(HERE, "golden", "blobs.npz"))["blobs"].astype(np.float32)


def _corners(lab):
    return {"top_left": lab[:3, :3].tolist(), "top_right": lab[:3, -3:].tolist(),
            "bottom_left": lab[-3:, :3].tolist(), "bottom_right": lab[-3:, -3:].tolist()}


def test_blobs_ccl_count(oracle, blobs):
    ka = _known()
    b = oracle.gaussian_blur(blobs, 1, 1)
    seg, _ = oracle.threshold_otsu(b)
    assert oracle.connected_components_labeling_box(seg).max() == ka["blur1_otsu_ccl_num_labels"]["value"]
    c = oracle.connected_components_labeling_box(blobs > 100)
    assert c.max() == ka["ccl_box_raw_gt_100"]["max"]
    assert _corners(c) == ka["ccl_box_raw_gt_100"]["corners"]


@pytest.mark.parametrize("key,sigma", [("gauss_otsu_1", 1), ("gauss_otsu_5", 5)])
def test_blobs_gauss_otsu(oracle, blobs, key, sigma):
    b = oracle.gaussian_blur(blobs, sigma, sigma)
    seg, _ = oracle.threshold_otsu(b)
    assert _corners(oracle.connected_components_labeling_box(seg)) == _known()[key]["corners"]


@pytest.mark.parametrize("key,spot,outline", [("vol_spot1_outline1", 1, 1),
                                              ("vol_spot3.2_outline1", 3.2, 1),
                                              ("vol_spot3.5_outline2", 3.5, 2)])
def test_blobs_voronoi_otsu(oracle, blobs, key, spot, outline):
    lab = oracle.voronoi_otsu_labeling(blobs, spot, outline)
    assert _corners(lab) == _known()[key]["corners"]


def test_blobs_statistics_table(oracle, blobs):
    ka = _known()["vol_spot3.5_outline2"]
    lab = oracle.voronoi_otsu_labeling(blobs, 3.5, 2)
    assert lab.max() == ka["num_labels"]
    s = oracle.statistics_of_labelled_pixels(blobs, lab)
    for k, row in ka["table_rows"].items():
        for col, val in row.items():
            assert s[col][int(k) - 1] == val, (k, col)
    for col, d in ka["describe"].items():
        if col in s and "mean" in d:
            assert np.isclose(np.float32(s[col].mean()), d["mean"], rtol=1e-5), col
            assert np.isclose(s[col].min(), d["min"], rtol=1e-5), col
            assert np.isclose(s[col].max(), d["max"], rtol=1e-5), col


# ---- gauss_otsu_labeling / eroded_otsu_labeling / erode_box --------------
def test_erode_box_golden(oracle):
    # tests/test_erode_box.py:5-29
    t = np.array([[0, 0, 0, 0, 0], [0, 1, 1, 1, 0], [0, 1, 1, 1, 0], [0, 1, 1, 1, 0], [0, 0, 0, 0, 0]])
    ref = np.zeros((5, 5), np.uint8)
    ref[2, 2] = 1
    assert np.array_equal(oracle.erode_box(t), ref)


def test_erode_box_clamps_at_the_edge(oracle):
    # a full image stays full: out-of-range neighbours read the edge voxel
    assert oracle.erode_box(np.ones((4, 5, 6))).all()
    assert oracle.erode_box(np.ones((3, 7))).all()


def test_gauss_otsu_labeling_golden(oracle):
    # tests/test_gauss_otsu_labeling.py:4-41
    src = np.array([[0, 0, 1, 1, 0, 0], [0, 1, 8, 9, 1, 0], [0, 1, 1, 0, 0, 0], [0, 0, 0, 0, 0, 0],
                    [0, 0, 0, 1, 1, 0], [0, 0, 1, 8, 7, 1], [0, 0, 1, 1, 1, 0]])
    ref = np.array([[0, 0, 1, 1, 0, 0], [0, 1, 1, 1, 1, 0], [0, 1, 1, 1, 0, 0], [0, 0, 0, 0, 0, 0],
                    [0, 0, 0, 2, 2, 0], [0, 0, 2, 2, 2, 2], [0, 0, 2, 2, 2, 0]])
    assert np.array_equal(oracle.gauss_otsu_labeling(src, 1), ref)


def test_eroded_otsu_labeling_golden(oracle):
    # tests/test_eroded_otsu_labeling.py:4-41 (number_of_erosions given as 1.0)
    src = np.array([[0, 0, 5, 5, 0, 0], [0, 5, 8, 9, 1, 0], [0, 5, 7, 6, 1, 1], [0, 0, 0, 5, 5, 1],
                    [0, 0, 0, 5, 5, 1], [0, 0, 5, 5, 5, 1], [0, 0, 5, 5, 5, 0]])
    ref = np.array([[0, 0, 1, 1, 0, 0], [0, 1, 1, 1, 1, 0], [0, 1, 1, 1, 1, 0], [0, 0, 1, 1, 1, 0],
                    [0, 0, 0, 2, 2, 0], [0, 0, 2, 2, 2, 0], [0, 0, 2, 2, 2, 0]])
    assert np.array_equal(oracle.eroded_otsu_labeling(src, 1.0, 1), ref)


@pytest.mark.parametrize("key,sigma", [("gauss_otsu_1", 1), ("gauss_otsu_5", 5)])
def test_blobs_gauss_otsu_labeling(oracle, blobs, key, sigma):
    # demo/segmentation/labeling.ipynb cells 13-14 through the composed oracle
    assert _corners(oracle.gauss_otsu_labeling(blobs, sigma)) == _known()[key]["corners"]


# ---- diamond CCL, extend_labeling_via_voronoi, voronoi_labeling ----------
def test_ccl_diamond_golden(oracle):
    # tests/test_connected_components_labeling_diamond.py:4-27
    src = np.array([[[0, 1, 0, 1], [0, 1, 0, 0], [1, 0, 0, 1]]])
    ref = np.array([[[0, 2, 0, 3], [0, 2, 0, 0], [1, 0, 0, 4]]])
    assert np.array_equal(oracle.connected_components_labeling_diamond(src), ref)


def test_extend_labeling_via_voronoi_golden(oracle):
    # tests/test_extend_labeling_via_voronoi.py:4-37
    src = np.array([[[0, 0, 0, 0, 3, 3], [0, 4, 0, 0, 3, 3], [0, 0, 0, 0, 0, 0], [0, 0, 0, 0, 0, 0],
                     [0, 2, 0, 0, 1, 0], [0, 0, 0, 0, 0, 0]]])
    ref = np.array([[[4, 4, 4, 3, 3, 3], [4, 4, 4, 3, 3, 3], [4, 4, 4, 3, 3, 3], [2, 2, 2, 1, 1, 1],
                     [2, 2, 2, 1, 1, 1], [2, 2, 2, 1, 1, 1]]])
    assert np.array_equal(oracle.extend_labeling_via_voronoi(src), ref)


def test_voronoi_labeling_golden(oracle):
    # tests/test_voronoi_labeling.py:4-37
    src = np.zeros((1, 6, 6))
    src[0, 1, 1] = src[0, 1, 4] = src[0, 4, 1] = src[0, 4, 4] = 1
    ref = np.array([[[1, 1, 1, 3, 3, 3]] * 3 + [[2, 2, 2, 4, 4, 4]] * 3])
    assert np.array_equal(oracle.voronoi_labeling(src), ref)


# ---- minimum_box / maximum_box / top_hat_box -----------------------------
def test_minimum_maximum_box_golden(oracle):
    # tests/test_minimum_box.py:4-31, tests/test_maximum_box.py:4-31
    t = np.zeros((5, 5), np.float32)
    t[1:4, 1:4] = 1
    ref = np.zeros((5, 5))
    ref[2, 2] = 1
    assert np.array_equal(oracle.minimum_box(t, 1, 1, 0), ref)
    assert np.array_equal(oracle.maximum_box(ref, 1, 1, 0), t)


def test_top_hat_box_golden(oracle):
    # tests/test_top_hat_box.py:4-22 (min 0, max 50)
    t = np.array([[0, 0, 0, 0, 0], [0, 50, 50, 50, 0], [0, 50, 100, 50, 0], [0, 50, 50, 50, 0],
                  [0, 0, 0, 0, 0]], np.float32)
    r = oracle.top_hat_box(t, 1, 1, 0)
    assert r.min() == 0 and r.max() == 50


# ---- euclidean_distance_from_label_centroid_map ---------------------------
CENTROID_DIST_LABELS = np.asarray([[1, 1, 1, 2], [1, 1, 1, 2], [1, 1, 1, 2], [2, 2, 2, 2]])
CENTROID_DIST_REF = np.asarray([[1.4142135, 1, 1.4142135, 2.3079278], [1, 0, 1, 1.4285713],
                                [1.4142135, 1, 1.4142135, 0.86896616],
                                [2.3079278, 1.4285713, 0.86896616, 1.2121831]])


def test_euclidean_distance_from_label_centroid_map_golden(oracle):
    # tests/test_euclidean_distance_from_label_centroid_map.py:4-34 (rtol 1e-3)
    got = oracle.euclidean_distance_from_label_centroid_map(CENTROID_DIST_LABELS)
    assert np.allclose(got, CENTROID_DIST_REF, 0.001)


# ---- neighbour-distance maps: the reference's own fixtures ------------------
QUADRANT_LABELS = np.asarray([[1, 1, 1, 3, 3, 3], [1, 1, 1, 3, 3, 3], [1, 1, 1, 3, 3, 3],
                              [0, 0, 0, 2, 2, 2], [0, 0, 0, 2, 2, 2], [0, 0, 0, 2, 2, 2]])
SPARSE_A = np.asarray([[1, 0, 0, 0, 0, 3], [0] * 6, [0] * 6, [0] * 6, [0] * 6, [0, 0, 0, 0, 0, 2]])
SPARSE_B = np.asarray([[0, 2, 0, 0, 0, 3], [1, 0, 0, 0, 0, 0], [0] * 6, [0] * 6, [0, 0, 0, 0, 0, 4],
                       [0, 0, 0, 0, 5, 0]])


def test_average_distance_of_n_nearest_neighbors_map_golden(oracle):
    # tests/test_average_distance_of_n_nearest_neighbors.py:4-35 (n = 2, rtol 0.01)
    ref = np.asarray([[3.62] * 3 + [3] * 3] * 3 + [[0] * 3 + [3.62] * 3] * 3)
    assert np.allclose(oracle.average_distance_of_n_nearest_neighbors_map(QUADRANT_LABELS, 2), ref, 0.01)


def test_average_neighbor_distance_map_golden(oracle):
    # tests/test_average_neighbor_distance_map.py:4-35
    ref = np.asarray([[3] * 6] * 3 + [[0] * 3 + [3] * 3] * 3)
    assert np.allclose(oracle.average_neighbor_distance_map(QUADRANT_LABELS), ref, 0.01)


def test_average_distance_to_n_nearest_other_labels_map_golden(oracle):
    # tests/test_average_distance_to_n_nearest_other_labels_map.py:4-45
    ref = np.zeros((6, 6))
    ref[0, 0] = ref[5, 5] = 1
    got = oracle.average_distance_to_n_nearest_other_labels_map(SPARSE_A, SPARSE_B, 1)
    assert np.allclose(got, ref, 0.01)


def test_neighbor_vectors_golden(oracle):
    # tests/test_average_distance_of_n_shortest_distances.py,
    # tests/test_average_distance_of_touching_neighbors.py,
    # tests/test_average_distance_of_n_nearest_distances.py
    c = oracle.centroids_of_labels(QUADRANT_LABELS)
    D = oracle.generate_distance_matrix(c, c)
    assert np.allclose(oracle.average_distance_of_n_shortest_distances(D, 1), [[0, 3, 3, 3]], 0.01)
    T = oracle.generate_touch_matrix(QUADRANT_LABELS)
    assert np.allclose(oracle.average_distance_of_touching_neighbors(D, T), [[0, 3, 3, 3]], 0.01)
    D2 = oracle.generate_distance_matrix(oracle.centroids_of_labels(SPARSE_A), oracle.centroids_of_labels(SPARSE_B))
    assert np.allclose(oracle.average_distance_of_n_nearest_distances(D2, 1), [[0, 1, 1, 0]], 0.01)


def test_generate_touch_matrix_golden(oracle):
    # tests/test_generate_touch_matrix.py:4-35
    lab = np.asarray([[1, 1, 0, 0, 0], [1, 1, 0, 3, 0], [0, 2, 2, 3, 0], [0, 2, 2, 0, 0], [0, 0, 0, 0, 4]])
    ref = np.asarray([[0, 1, 1, 1, 1], [1, 0, 1, 0, 0], [1, 1, 0, 1, 0], [1, 0, 1, 0, 0], [1, 0, 0, 0, 0]]).T
    assert np.array_equal(oracle.generate_touch_matrix(lab), ref)


def test_n_nearest_selection_keeps_nan_in_place(oracle):
    # the kernel's insertion pass never moves a NaN (absent label) and never
    # lets a value pass it: with n = 2 the NaN held first stays in the mean
    assert np.isnan(oracle._held_mean([np.nan, 3.0, 1.0], 2))
    assert oracle._held_mean([4.0, 3.0, 1.0, 2.0], 2) == np.float32(1.5)
    assert np.isnan(oracle._held_mean([], 3))
