"""CPU oracle for the voronoi_otsu_labeling + statistics path.

TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA library and the
timed CPU baseline.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py`` (its ``cpu_baseline`` leg and ``--impl reference``) import this
package; the product package never does.

The arithmetic lives in ``cle_oracle.c`` (a C restatement of the reference's
algorithm, citing the reference file:line for each step); this module is a
thin numpy/ctypes wrapper.  ``build()`` compiles it with the committed
Makefile.

Parity status: pinned against every golden vector the reference's own tests
hold for this path (tests/test_oracle_golden.py) and the demo known answers on
``blobs.tif`` (tests/golden/).  Unpinned by any reference fixture: the z term
of the 3D CCL key (x-major ``(x*H + y)*D + z`` assumed), the choice between
histogram bin rules (``floor((v-min)*255/range + 0.5)`` used), the float32
operation order inside a Gaussian pass (fused multiply-add chain used).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libcle_oracle.so")
_lib = None

NCOLS = 35
STAT_KEYS = [
    "bbox_min_x", "bbox_min_y", "bbox_min_z", "bbox_max_x", "bbox_max_y", "bbox_max_z",
    "bbox_width", "bbox_height", "bbox_depth", "min_intensity", "max_intensity",
    "sum_intensity", "area", "mean_intensity",
    "sum_intensity_times_x", "mass_center_x", "sum_intensity_times_y", "mass_center_y",
    "sum_intensity_times_z", "mass_center_z",
    "sum_x", "centroid_x", "sum_y", "centroid_y", "sum_z", "centroid_z",
    "sum_distance_to_centroid", "mean_distance_to_centroid",
    "sum_distance_to_mass_center", "mean_distance_to_mass_center",
    "standard_deviation_intensity", "max_distance_to_centroid", "max_distance_to_mass_center",
    "mean_max_distance_to_centroid_ratio", "mean_max_distance_to_mass_center_ratio",
]


def build() -> str:
    """Compile libcle_oracle.so in place (idempotent)."""
    src = os.path.join(_HERE, "cle_oracle.c")
    if (not os.path.exists(_LIB_PATH)) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        I64 = ctypes.c_int64
        D = ctypes.c_double
        I = ctypes.c_int
        F = ctypes.c_float
        L.orc_num_threads.restype = I
        L.orc_set_num_threads.argtypes = [I]
        L.orc_sigma_to_kernel_size.argtypes = [D]
        L.orc_sigma_to_kernel_size.restype = I
        L.orc_gauss_weights.argtypes = [D, I, P]
        L.orc_gaussian_blur.argtypes = [P, P, I64, I64, I64, I, D, D, D]
        L.orc_detect_maxima.argtypes = [P, P, I64, I64, I64, I]
        L.orc_minmax.argtypes = [P, I64, P, P]
        L.orc_histogram.argtypes = [P, I64, I64, I64, I, F, F, P]
        L.orc_otsu_threshold.argtypes = [P, I, F, F]
        L.orc_otsu_threshold.restype = D
        L.orc_greater_constant.argtypes = [P, P, I64, F]
        L.orc_binary_and.argtypes = [P, P, P, I64]
        L.orc_threshold_otsu.argtypes = [P, P, I64, I64, I64]
        L.orc_threshold_otsu.restype = D
        L.orc_ccl_box.argtypes = [P, P, I64, I64, I64]
        L.orc_ccl_box.restype = I64
        L.orc_relabel_sequential.argtypes = [P, P, I64]
        L.orc_masked_voronoi.argtypes = [P, P, P, P, I64, I64, I64, I]
        L.orc_masked_voronoi.restype = I64
        L.orc_voronoi_otsu_labeling.argtypes = [P, P, I64, I64, I64, I, D, D, P, P, P]
        L.orc_ccl_diamond.argtypes = [P, P, I64, I64, I64]
        L.orc_ccl_diamond.restype = I64
        L.orc_extend_labeling_via_voronoi.argtypes = [P, P, I64, I64, I64, I]
        L.orc_extend_labeling_via_voronoi.restype = I64
        L.orc_voronoi_labeling.argtypes = [P, P, I64, I64, I64, I]
        L.orc_voronoi_labeling.restype = I64
        L.orc_erode_box.argtypes = [P, P, I64, I64, I64, I]
        L.orc_minmax_box.argtypes = [P, P, I64, I64, I64, I, D, D, D, I]
        L.orc_top_hat_box.argtypes = [P, P, I64, I64, I64, I, D, D, D]
        L.orc_gauss_otsu_labeling.argtypes = [P, P, I64, I64, I64, I, D]
        L.orc_gauss_otsu_labeling.restype = I64
        L.orc_eroded_otsu_labeling.argtypes = [P, P, I64, I64, I64, I, I, D]
        L.orc_eroded_otsu_labeling.restype = I64
        L.orc_voronoi_otsu_labeling.restype = I64
        L.orc_statistics.argtypes = [P, P, I64, I64, I64, I64, P]
        L.orc_stats_ncols.restype = I
        assert L.orc_stats_ncols() == NCOLS
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _dhw(shape):
    if len(shape) == 2:
        return 1, shape[0], shape[1]
    if len(shape) == 3:
        return shape
    raise ValueError(f"2D or 3D image expected, got shape {shape}")


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a), dtype=np.float32)


def _u8(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a) != 0, dtype=np.uint8)


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return lib().orc_num_threads()


def sigma_to_kernel_size(sigma: float) -> int:
    return lib().orc_sigma_to_kernel_size(float(sigma))


def gauss_weights(sigma: float) -> np.ndarray:
    n = sigma_to_kernel_size(sigma)
    w = np.empty(n, np.float32)
    lib().orc_gauss_weights(float(sigma), n, _p(w))
    return w


def gaussian_blur(img, sigma_x=0.0, sigma_y=0.0, sigma_z=0.0) -> np.ndarray:
    a = _f32(img)
    out = np.empty_like(a)
    D, H, W = _dhw(a.shape)
    lib().orc_gaussian_blur(_p(a), _p(out), D, H, W, a.ndim, float(sigma_x), float(sigma_y),
                            float(sigma_z))
    return out


def detect_maxima(img) -> np.ndarray:
    a = _f32(img)
    out = np.empty(a.shape, np.uint8)
    D, H, W = _dhw(a.shape)
    lib().orc_detect_maxima(_p(a), _p(out), D, H, W, a.ndim)
    return out


def minmax(img):
    a = _f32(img)
    mn = np.zeros(1, np.float32)
    mx = np.zeros(1, np.float32)
    lib().orc_minmax(_p(a), a.size, _p(mn), _p(mx))
    return mn[0], mx[0]


def histogram(img, num_bins=256, minimum_intensity=None, maximum_intensity=None) -> np.ndarray:
    a = _f32(img)
    if minimum_intensity is None or maximum_intensity is None:
        minimum_intensity, maximum_intensity = minmax(a)
    out = np.empty(num_bins, np.float32)
    D, H, W = _dhw(a.shape)
    lib().orc_histogram(_p(a), D, H, W, int(num_bins), float(minimum_intensity),
                        float(maximum_intensity), _p(out))
    return out


def otsu_threshold_from_histogram(hist, mn, mx) -> float:
    h = _f32(hist)
    return lib().orc_otsu_threshold(_p(h), h.size, float(mn), float(mx))


def threshold_otsu(img):
    """Returns (binary u8, float64 threshold)."""
    a = _f32(img)
    out = np.empty(a.shape, np.uint8)
    D, H, W = _dhw(a.shape)
    t = lib().orc_threshold_otsu(_p(a), _p(out), D, H, W)
    return out, t


def greater_constant(img, constant) -> np.ndarray:
    a = _f32(img)
    out = np.empty(a.shape, np.uint8)
    lib().orc_greater_constant(_p(a), _p(out), a.size, float(constant))
    return out


def binary_and(a, b) -> np.ndarray:
    x, y = _u8(a), _u8(b)
    out = np.empty(x.shape, np.uint8)
    lib().orc_binary_and(_p(x), _p(y), _p(out), x.size)
    return out


def connected_components_labeling_box(binary) -> np.ndarray:
    fg = _u8(binary)
    out = np.empty(fg.shape, np.uint32)
    D, H, W = _dhw(fg.shape)
    lib().orc_ccl_box(_p(fg), _p(out), D, H, W)
    return out


def relabel_sequential(labels) -> np.ndarray:
    a = np.asarray(labels)
    if a.dtype.kind == "f":
        a = a.astype(np.int64)
    a = np.ascontiguousarray(np.clip(a, 0, None), dtype=np.uint32)
    out = np.empty_like(a)
    lib().orc_relabel_sequential(_p(a), _p(out), a.size)
    return out


def masked_voronoi_labeling(seeds, mask, return_steps=False):
    s = _u8(seeds)
    m = _f32(mask)
    out = np.empty(s.shape, np.uint32)
    D, H, W = _dhw(s.shape)
    steps = lib().orc_masked_voronoi(_p(s), _p(m), None, _p(out), D, H, W, s.ndim)
    return (out, steps) if return_steps else out


def voronoi_otsu_labeling(img, spot_sigma=2.0, outline_sigma=2.0, debug=False):
    a = _f32(img)
    out = np.empty(a.shape, np.uint32)
    D, H, W = _dhw(a.shape)
    spots = np.empty(a.shape, np.uint8)
    seg = np.empty(a.shape, np.uint8)
    thr = np.zeros(1, np.float64)
    steps = lib().orc_voronoi_otsu_labeling(_p(a), _p(out), D, H, W, a.ndim, float(spot_sigma),
                                            float(outline_sigma), _p(spots), _p(seg), _p(thr))
    if debug:
        return out, dict(seeds=spots, segmentation=seg, threshold=float(thr[0]), steps=steps)
    return out


def connected_components_labeling_diamond(binary) -> np.ndarray:
    fg = _u8(binary)
    out = np.empty(fg.shape, np.uint32)
    D, H, W = _dhw(fg.shape)
    lib().orc_ccl_diamond(_p(fg), _p(out), D, H, W)
    return out


def _labels_u32(a) -> np.ndarray:
    """uint32 labels as the reference's copy into a uint32 image makes them
    (float values: saturating conversion, fractions dropped)."""
    a = np.asarray(a)
    if a.dtype.kind == "f":
        a = np.where(np.isnan(a), 0, np.clip(a, 0, 4294967295.0))
        return np.ascontiguousarray(a.astype(np.uint64).astype(np.uint32))
    return np.ascontiguousarray(np.clip(a.astype(np.int64), 0, 4294967295).astype(np.uint32))


def extend_labeling_via_voronoi(labels) -> np.ndarray:
    a = _labels_u32(labels)
    out = np.empty(a.shape, np.uint32)
    D, H, W = _dhw(a.shape)
    lib().orc_extend_labeling_via_voronoi(_p(a), _p(out), D, H, W, a.ndim)
    return out


def voronoi_labeling(binary) -> np.ndarray:
    fg = _u8(binary)
    out = np.empty(fg.shape, np.uint32)
    D, H, W = _dhw(fg.shape)
    lib().orc_voronoi_labeling(_p(fg), _p(out), D, H, W, fg.ndim)
    return out


def minimum_box(img, radius_x=0.0, radius_y=0.0, radius_z=0.0, _max=0) -> np.ndarray:
    a = _f32(img)
    out = np.empty_like(a)
    D, H, W = _dhw(a.shape)
    lib().orc_minmax_box(_p(a), _p(out), D, H, W, a.ndim, float(radius_x), float(radius_y),
                         float(radius_z), int(_max))
    return out


def maximum_box(img, radius_x=0.0, radius_y=0.0, radius_z=0.0) -> np.ndarray:
    return minimum_box(img, radius_x, radius_y, radius_z, _max=1)


def top_hat_box(img, radius_x=1.0, radius_y=1.0, radius_z=1.0) -> np.ndarray:
    a = _f32(img)
    out = np.empty_like(a)
    D, H, W = _dhw(a.shape)
    lib().orc_top_hat_box(_p(a), _p(out), D, H, W, a.ndim, float(radius_x), float(radius_y),
                          float(radius_z))
    return out


def erode_box(img) -> np.ndarray:
    a = _f32(img)
    out = np.empty(a.shape, np.uint8)
    D, H, W = _dhw(a.shape)
    lib().orc_erode_box(_p(a), _p(out), D, H, W, a.ndim)
    return out


def gauss_otsu_labeling(img, outline_sigma=2.0) -> np.ndarray:
    a = _f32(img)
    out = np.empty(a.shape, np.uint32)
    D, H, W = _dhw(a.shape)
    lib().orc_gauss_otsu_labeling(_p(a), _p(out), D, H, W, a.ndim, float(outline_sigma))
    return out


def eroded_otsu_labeling(img, number_of_erosions=5, outline_sigma=2.0) -> np.ndarray:
    a = _f32(img)
    out = np.empty(a.shape, np.uint32)
    D, H, W = _dhw(a.shape)
    lib().orc_eroded_otsu_labeling(_p(a), _p(out), D, H, W, a.ndim, max(0, int(number_of_erosions)),
                                   float(outline_sigma))
    return out


def statistics_of_labelled_pixels(intensity, labels) -> dict:
    lab = np.asarray(labels)
    if lab.dtype.kind == "f":
        lab = lab.astype(np.int64)
    lab = np.ascontiguousarray(np.clip(lab, 0, None), dtype=np.uint32)
    inten = _f32(intensity)
    L = int(lab.max()) if lab.size else 0
    table = np.empty((NCOLS, max(L, 1)), np.float32)
    D, H, W = _dhw(lab.shape)
    if L > 0:
        lib().orc_statistics(_p(inten), _p(lab), D, H, W, L, _p(table))
    table = table[:, :L]
    out = {"label": np.arange(1, L + 1), "original_label": np.arange(1, L + 1)}
    for i, k in enumerate(STAT_KEYS):
        out[k] = table[i].copy()
    return out


def euclidean_distance_from_label_centroid_map(labels) -> np.ndarray:
    """Each labelled pixel's distance to its label's point in the centroid list
    of _tier9/_centroids_of_background_and_labels.py (column 0 the background's
    centroid, column k label k's: coordinate sums / pixel count, float32),
    label-0 pixels 0 (_tier9/_euclidean_distance_from_label_centroid_map.py).
    The label is read like an image read of the list: (int) of the value,
    clamped to the list's columns, so a negative label reads column 0 (the
    background centroid) and gets its distance to it.  Distances in float64,
    returned as float32."""
    lab = np.asarray(labels)
    if lab.dtype.kind == "f":
        lab = np.nan_to_num(lab, nan=0.0).astype(np.int64)
    lab = lab.astype(np.int64)
    # the point list: statistics of labels + 1 (label 1 = the background);
    # negative labels (+1 <= 0) are in no column's sums
    lab1 = np.where(lab >= 0, lab + 1, 0)
    st = statistics_of_labelled_pixels(np.zeros(lab.shape, np.float32), lab1)
    m = len(st["label"])                          # columns 0 .. m-1 = labels 0 .. m-1
    out = np.zeros(lab.shape, np.float64)
    if m == 0:
        return out.astype(np.float32)
    keys = ("centroid_x", "centroid_y", "centroid_z")[:lab.ndim if lab.ndim == 3 else 2]
    cen = [st[k].astype(np.float32) for k in keys]
    col = np.clip(lab, 0, m - 1)
    coords = np.indices(lab.shape)[::-1]          # x, y(, z) grids
    d2 = np.zeros(lab.shape, np.float64)
    for c, grid in zip(cen, coords):
        d2 += (grid - c[col].astype(np.float64)) ** 2
    out = np.where(lab != 0, np.sqrt(d2), 0.0)
    return out.astype(np.float32)


# ---- neighbour-distance maps ------------------------------------------------
# _tier1/_generate_distance_matrix.py, _tier1/_generate_touch_matrix.py with
# generate_touch_matrix_{2,3}d_x.cl, _tier1/_average_distance_of_n_nearest_distances.py
# with average_distance_of_n_nearest_distances_x.cl,
# _tier1/_average_distance_of_n_shortest_distances.py,
# _tier1/_average_distance_of_touching_neighbors.py and the three maps of _tier9
# built from them.  float32 throughout, as the reference's kernels compute.

def centroids_of_labels(labels) -> np.ndarray:
    """[d, L] float32 point list of labels 1..L (L = the largest label): per
    dimension float32(coordinate sum) / float32(voxel count), NaN for a label
    without voxels (_tier9/_centroids_of_labels.py)."""
    lab = np.asarray(labels)
    if lab.dtype.kind == "f":
        lab = np.nan_to_num(lab, nan=0.0)
    lab = np.clip(lab.astype(np.int64), 0, None)
    L = int(lab.max()) if lab.size else 0
    coords = np.indices(lab.shape)[::-1]          # x, y(, z)
    flat = lab.ravel()
    cnt = np.bincount(flat, minlength=L + 1)[1:L + 1]
    out = np.empty((lab.ndim, L), np.float32)
    with np.errstate(invalid="ignore", divide="ignore"):
        for k, g in enumerate(coords):
            s = np.bincount(flat, weights=g.ravel().astype(np.float64), minlength=L + 1)[1:L + 1]
            out[k] = np.float32(s) / np.float32(cnt)
    return out


def generate_distance_matrix(p1, p2) -> np.ndarray:
    """[m+1, n+1] float32: [j+1, i+1] = sqrt of the float32 sum, in the order
    x, y(, z), of the squared float32 differences of point i of p1 and point j
    of p2; row and column 0 zero."""
    p1 = np.asarray(p1, np.float32)
    p2 = np.asarray(p2, np.float32)
    n, m = p1.shape[1], p2.shape[1]
    out = np.zeros((m + 1, n + 1), np.float32)
    s = np.zeros((m, n), np.float32)
    with np.errstate(invalid="ignore"):
        for k in range(p1.shape[0]):
            t = (p1[k][None, :] - p2[k][:, None]).astype(np.float32)
            s = (s + (t * t).astype(np.float32)).astype(np.float32)
        out[1:, 1:] = np.sqrt(s)
    return out


def generate_touch_matrix(labels) -> np.ndarray:
    """[L+1, L+1] float32: 1 at (a, b) and (b, a) where a voxel of label a has
    its +x, +y (or +z) neighbour in label b != a."""
    lab = np.asarray(labels)
    lab = lab.astype(np.float32).astype(np.int64) if lab.dtype.kind == "f" else lab.astype(np.int64)
    L = int(lab.max()) if lab.size else 0
    T = np.zeros((L + 1, L + 1), np.float32)
    for ax in range(lab.ndim):
        a = np.moveaxis(lab, ax, 0)
        x, y = a[:-1].ravel(), a[1:].ravel()
        d = (x != y) & (x >= 0) & (y >= 0)
        T[y[d], x[d]] = 1.0
        T[x[d], y[d]] = 1.0
    return T


def _held_mean(values, n):
    """average_distance_of_n_nearest_distances_x.cl's selection: values are
    appended while fewer than n are held, then one insertion pass from the end
    moves a smaller value down; the mean is the float32 sum in buffer order over
    the count (NaN when none)."""
    buf = []
    for v in values:
        v = np.float32(v)
        if len(buf) < n:
            buf.append(v)
        for i in range(len(buf) - 1, -1, -1):
            if v > buf[i]:
                break
            if v < buf[i] and (i == 0 or v >= buf[i - 1]):
                for j in range(len(buf) - 1, i, -1):
                    buf[j] = buf[j - 1]
                buf[i] = v
                break
    s = np.float32(0.0)
    for b in buf:
        s = np.float32(s + b)
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.float32(s / np.float32(len(buf)))


def _n_distance_vector(D, n, exclude_self):
    D = np.asarray(D, np.float32)
    H, W = D.shape
    out = np.zeros((1, W), np.float32)
    for x in range(W):
        rows = [y for y in range(1, H) if not (exclude_self and y == x)]
        col = D[rows, x]
        if not np.isnan(col).any():
            # no NaN: the selection keeps the n smallest in ascending order
            col = np.sort(col)[:n]
        out[0, x] = _held_mean(col, n)
    return out


def average_distance_of_n_nearest_distances(D, n=1) -> np.ndarray:
    """[1, columns]: per column the mean of the n smallest of rows 1.."""
    return _n_distance_vector(D, int(n), False)


def average_distance_of_n_shortest_distances(D, n=1) -> np.ndarray:
    """[1, rows]: as above with the column's own row left out (the distance of a
    label to itself)."""
    return _n_distance_vector(D, int(n), True)


def average_distance_of_touching_neighbors(D, T) -> np.ndarray:
    """[1, rows]: per column the float32 mean (sum in row order) of the
    distances in rows >= 1 whose touch entry is set; 0 when none."""
    D = np.asarray(D, np.float32)
    T = np.asarray(T, np.float32)
    H, W = D.shape
    out = np.zeros((1, W), np.float32)
    for x in range(W):
        s, c = np.float32(0.0), 0
        for y in range(1, H):
            if T[y, x] > 0:
                s = np.float32(s + D[y, x])
                c += 1
        out[0, x] = np.float32(s / np.float32(c)) if c else np.float32(0.0)
    return out


def replace_intensities(labels, vec) -> np.ndarray:
    lab = np.asarray(labels)
    idx = lab.astype(np.float32).astype(np.int64) if lab.dtype.kind == "f" else lab.astype(np.int64)
    v = np.asarray(vec, np.float32).ravel()
    return v[np.clip(idx, 0, len(v) - 1)]


def average_distance_of_n_nearest_neighbors_map(labels, n=1) -> np.ndarray:
    c = centroids_of_labels(labels)
    D = generate_distance_matrix(c, c)
    return replace_intensities(labels, average_distance_of_n_shortest_distances(D, n))


def average_distance_to_n_nearest_other_labels_map(labels, other_labels, n=1) -> np.ndarray:
    D = generate_distance_matrix(centroids_of_labels(labels), centroids_of_labels(other_labels))
    return replace_intensities(labels, average_distance_of_n_nearest_distances(D, n))


def average_neighbor_distance_map(labels) -> np.ndarray:
    c = centroids_of_labels(labels)
    D = generate_distance_matrix(c, c)
    return replace_intensities(labels, average_distance_of_touching_neighbors(D, generate_touch_matrix(labels)))
