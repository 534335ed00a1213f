"""cle.* operations of the voronoi_otsu_labeling + statistics path.

Each function keeps the reference's name, parameter names, defaults, output
creator and return value; the work is one call into libcle_b200.so on the
current torch CUDA stream.  Reference citations are on each function.
"""
import contextlib
import threading
import warnings
from enum import Enum

import numpy as np
import torch

from . import _lib
from ._tier0 import (B200Array, Image, create, create_binary_like, create_labels_like, create_like,
                     create_none, plugin_function, push, push_native)

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
assert len(STAT_KEYS) == _lib.STATS_NCOLS


def _T(a: B200Array):
    return _lib.tensor_desc(a.tensor)


_tls = threading.local()


@contextlib.contextmanager
def call_options(max_loop_steps: int = 0, loop_time_limit_ms: int = 0, barrier_time_limit_ms: int = 0,
                 cooperative_ctas: int = 0):
    """Limits of the device loops (the Voronoi growth) for the cle.* calls this
    thread makes inside the block; 0 keeps a field's default.  A loop that
    reaches a limit raises RuntimeError from the call.  The setting belongs to
    the calling thread only; each call passes it to the library as an
    argument (nothing is stored in the library).

        with cle.call_options(max_loop_steps=1000):
            labels = cle.voronoi_otsu_labeling(image)
    """
    prev = getattr(_tls, "options", None)
    _tls.options = _lib.call_options(max_loop_steps, loop_time_limit_ms, barrier_time_limit_ms,
                                     cooperative_ctas)
    try:
        yield _tls.options
    finally:
        _tls.options = prev


def _opts():
    o = getattr(_tls, "options", None)
    return _lib.ref(o) if o is not None else None


def _call(name, *args):
    lib = _lib.load()
    _lib.check(getattr(lib, name)(*args), name[4:])


def _ws(query, *args, device=None):
    lib = _lib.load()
    n = getattr(lib, query)(*args)
    return _lib.workspace(n, device or torch.device("cuda", torch.cuda.current_device()))


def _ptr(t: torch.Tensor):
    return t.data_ptr() if t.numel() else None


def sigma_to_kernel_size(sigma):
    """_tier0/_sigma_to_kernel_size.py:1-4"""
    n = int(float(sigma) * 8.0)
    if n % 2 == 0:
        n = n + 1
    return n


def radius_to_kernel_size(radius):
    """_tier0/_radius_to_kernel_size.py:1-2."""
    return int(radius * 2 + 1)


# ---------------------------------------------------------------------------
@plugin_function(categories=['filter', 'denoise', 'in assistant', 'bia-bob-suggestion'], priority=1,
                 native_inputs=("source",))
def gaussian_blur(source: Image, destination: Image = None, sigma_x: float = 0, sigma_y: float = 0,
                  sigma_z: float = 0) -> Image:
    """Gaussian blur, separable along x, y, z (_tier1/_gaussian_blur.py:6-58)."""
    s, d = _T(source), _T(destination)
    ws = _ws("cle_gaussian_blur_workspace_bytes", _lib.ref(s))
    _call("cle_gaussian_blur", _lib.ref(s), _lib.ref(d), float(sigma_x), float(sigma_y),
          float(sigma_z), _ptr(ws), ws.numel(), _lib.stream_ptr())
    return destination


def _minmax(source: B200Array):
    s = _T(source)
    out = torch.empty(2, dtype=torch.float32, device=source.tensor.device)
    ws = _ws("cle_minimum_maximum_workspace_bytes", _lib.ref(s))
    _call("cle_minimum_maximum", _lib.ref(s), out.data_ptr(), _ptr(ws), ws.numel(), _lib.stream_ptr())
    return out


@plugin_function
def minimum_of_all_pixels(source: Image) -> float:
    """_tier2/_minimum_of_all_pixels.py:7-60"""
    return np.float32(_minmax(source)[0].item())


@plugin_function
def maximum_of_all_pixels(source: Image) -> float:
    """_tier2/_maximum_of_all_pixels.py:7-60"""
    return np.float32(_minmax(source)[1].item())


@plugin_function(output_creator=create_none)
def histogram(source: Image, destination: Image = None, num_bins: int = 256,
              minimum_intensity: float = None, maximum_intensity: float = None,
              determine_min_max: bool = True) -> Image:
    """Per-row partial histograms summed in float32 (_tier3/_histogram.py:26-130)."""
    if destination is None:
        destination = create([int(num_bins)])
    determine = bool(determine_min_max) or minimum_intensity is None or maximum_intensity is None
    s, d = _T(source), _T(destination)
    ws = _ws("cle_histogram_workspace_bytes", _lib.ref(s), int(num_bins))
    _call("cle_histogram", _lib.ref(s), _lib.ref(d), int(num_bins),
          float(minimum_intensity) if not determine else 0.0,
          float(maximum_intensity) if not determine else 0.0, int(determine), _ptr(ws),
          ws.numel(), _lib.stream_ptr())
    return destination


@plugin_function(categories=['binarize', 'in assistant', 'bia-bob-suggestion'], priority=1,
                 output_creator=create_binary_like)
def threshold_otsu(source: Image, destination: Image = None) -> Image:
    """Otsu threshold, histogram and Otsu both on the device
    (_tier9/_threshold_otsu.py:11-54)."""
    s, d = _T(source), _T(destination)
    ws = _ws("cle_threshold_otsu_workspace_bytes", _lib.ref(s))
    _call("cle_threshold_otsu", _lib.ref(s), _lib.ref(d), None, _ptr(ws), ws.numel(), _lib.stream_ptr())
    return destination


def scikit_image_threshold_otsu(image=None, nbins=256, *, hist=None):
    """Host Otsu on a given (counts, bin_centers) histogram, as the reference
    keeps it (_tier9/_threshold_otsu.py:64-106)."""
    if image is None and hist is None:
        raise Exception("Either name or hist must be provided.")
    if hist is not None:
        if isinstance(hist, (tuple, list)):
            counts, bin_centers = hist
        else:
            counts = hist
            bin_centers = np.arange(counts.size)
    else:
        image = np.asarray(image)
        first_pixel = image.ravel()[0]
        if np.all(image == first_pixel):
            return first_pixel
        counts, edges = np.histogram(image.ravel(), nbins)
        bin_centers = (edges[:-1] + edges[1:]) / 2
    counts = np.asarray(counts).astype(float)
    weight1 = np.cumsum(counts)
    weight2 = np.cumsum(counts[::-1])[::-1]
    with np.errstate(divide="ignore", invalid="ignore"):
        mean1 = np.cumsum(counts * bin_centers) / weight1
        mean2 = (np.cumsum((counts * bin_centers)[::-1]) / weight2[::-1])[::-1]
        variance12 = weight1[:-1] * weight2[1:] * (mean1[:-1] - mean2[1:]) ** 2
    idx = np.argmax(variance12)
    return bin_centers[:-1][idx]


@plugin_function(categories=['binarize', 'in assistant'], output_creator=create_binary_like)
def greater_constant(source: Image, destination: Image = None, constant: float = 0) -> Image:
    """_tier1/_greater_constant.py:6-40 (constant passed as float32)."""
    _call("cle_greater_constant", _lib.ref(_T(source)), _lib.ref(_T(destination)), float(constant),
          _lib.stream_ptr())
    return destination


@plugin_function(categories=['combine', 'binary processing', 'in assistant'],
                 output_creator=create_binary_like)
def binary_and(operand1: Image, operand2: Image, destination: Image = None) -> Image:
    """_tier1/_binary_and.py:6-47"""
    _call("cle_binary_and", _lib.ref(_T(operand1)), _lib.ref(_T(operand2)), _lib.ref(_T(destination)),
          _lib.stream_ptr())
    return destination


@plugin_function(categories=['combine', 'in assistant'])
def mask(source: Image, mask: Image, destination: Image = None) -> Image:
    """_tier1/_mask.py:6-44"""
    _call("cle_mask", _lib.ref(_T(source)), _lib.ref(_T(mask)), _lib.ref(_T(destination)),
          _lib.stream_ptr())
    return destination


@plugin_function(categories=['binarize', 'in assistant'], output_creator=create_binary_like)
def detect_maxima_box(source: Image, destination: Image = None, radius_x: int = 0,
                      radius_y: int = 0, radius_z: int = 0) -> Image:
    """_tier1/_detect_maxima_box.py:5-48 (+ detect_maxima_{2,3}d_x.cl)."""
    s, d = _T(source), _T(destination)
    ws = _ws("cle_detect_maxima_box_workspace_bytes", _lib.ref(s), int(radius_x), int(radius_y),
             int(radius_z))
    _call("cle_detect_maxima_box", _lib.ref(s), _lib.ref(d), int(radius_x), int(radius_y),
          int(radius_z), _ptr(ws), ws.numel(), _lib.stream_ptr())
    return destination


@plugin_function(categories=['label', 'in assistant', 'bia-bob-suggestion'], priority=1,
                 output_creator=create_labels_like)
def connected_components_labeling_box(binary_input: Image, labeling_destination: Image = None,
                                      flagged_nonzero_minimum_filter: callable = None) -> Image:
    """_tier4/_connected_components_labeling_box.py:15-66.  The reference's
    filter hook selects the Jacobi filter it iterates; the union-find here
    computes the fixed point of the box filter directly, so the hook is
    accepted for signature compatibility and ignored."""
    b, d = _T(binary_input), _T(labeling_destination)
    ws = _ws("cle_connected_components_labeling_box_workspace_bytes", _lib.ref(b))
    _call("cle_connected_components_labeling_box", _lib.ref(b), _lib.ref(d), _ptr(ws), ws.numel(),
          _lib.stream_ptr())
    return labeling_destination


def _label_max(labels: B200Array) -> int:
    s = _T(labels)
    out = torch.zeros(1, dtype=torch.int32, device=labels.tensor.device)
    _call("cle_label_maximum", _lib.ref(s), out.data_ptr(), None, 0, _lib.stream_ptr())
    return int(out.item()) & 0xFFFFFFFF


@plugin_function(output_creator=create_labels_like,
                 categories=['label processing', 'in assistant', 'bia-bob-suggestion'])
def relabel_sequential(source: Image, output: Image = None, blocksize: int = 4096) -> Image:
    """_tier3/_relabel_sequential.py:12-58 (blocksize kept for signature
    compatibility; the device ranks all values in one pass)."""
    mx = _label_max(source)
    s, d = _T(source), _T(output)
    ws = _ws("cle_relabel_sequential_workspace_bytes", _lib.ref(s), mx)
    _call("cle_relabel_sequential", _lib.ref(s), _lib.ref(d), mx, _ptr(ws), ws.numel(),
          _lib.stream_ptr())
    return output


@plugin_function(categories=['label'], output_creator=create_labels_like)
def masked_voronoi_labeling(binary_source: Image, mask_image: Image,
                            labeling_destination: Image = None) -> Image:
    """_tier5/_masked_voronoi_labeling.py:7-76 (general form: any mask values,
    seeds anywhere)."""
    b, m, d = _T(binary_source), _T(mask_image), _T(labeling_destination)
    ws = _ws("cle_masked_voronoi_labeling_workspace_bytes", _lib.ref(b))
    stream = _lib.stream_ptr()
    _call("cle_masked_voronoi_labeling", _lib.ref(b), _lib.ref(m), _lib.ref(d), _opts(), _ptr(ws),
          ws.numel(), stream)
    _lib.check(_lib.load().cle_workspace_status(ws.data_ptr(), ws.numel(), stream),
               "masked_voronoi_labeling")
    return labeling_destination


def masked_voronoi_labeling_binary(binary_source, mask_image, labeling_destination=None):
    """masked_voronoi_labeling for a 0/1 mask with every seed inside it (the
    case inside voronoi_otsu_labeling), on the active-front growth kernel.
    Same result as masked_voronoi_labeling for such inputs."""
    from ._tier0 import push_native
    b = push_native(binary_source) if not isinstance(binary_source, B200Array) else binary_source
    m = push_native(mask_image) if not isinstance(mask_image, B200Array) else mask_image
    if labeling_destination is None:
        labeling_destination = create_labels_like(b)
    bd, md, dd = _T(b), _T(m), _T(labeling_destination)
    ws = _ws("cle_masked_voronoi_labeling_binary_workspace_bytes", _lib.ref(bd))
    stream = _lib.stream_ptr()
    _call("cle_masked_voronoi_labeling_binary", _lib.ref(bd), _lib.ref(md), _lib.ref(dd), _opts(),
          _ptr(ws), ws.numel(), stream)
    _lib.check(_lib.load().cle_workspace_status(ws.data_ptr(), ws.numel(), stream),
               "masked_voronoi_labeling")
    return labeling_destination


@plugin_function(categories=['label', 'in assistant'], output_creator=create_labels_like)
def connected_components_labeling_diamond(binary_input: Image, labeling_destination: Image = None) -> Image:
    """Connected components with face connectivity (4 neighbours in 2D, 6 in 3D),
    labels as in connected_components_labeling_box
    (_tier5/_connected_components_labeling_diamond.py:6-40)."""
    b, d = _T(binary_input), _T(labeling_destination)
    ws = _ws("cle_connected_components_labeling_diamond_workspace_bytes", _lib.ref(b))
    _call("cle_connected_components_labeling_diamond", _lib.ref(b), _lib.ref(d), _ptr(ws), ws.numel(),
          _lib.stream_ptr())
    return labeling_destination


def _grow_call(name, src: B200Array, dst: B200Array):
    s, d = _T(src), _T(dst)
    ws = _ws(name + "_workspace_bytes", _lib.ref(s))
    stream = _lib.stream_ptr()
    _call(name, _lib.ref(s), _lib.ref(d), _opts(), _ptr(ws), ws.numel(), stream)
    _lib.check(_lib.load().cle_workspace_status(ws.data_ptr(), ws.numel(), stream), name[4:])
    return dst


@plugin_function(categories=['label processing', 'in assistant'], output_creator=create_labels_like)
def extend_labeling_via_voronoi(labeling_source: Image, labeling_destination: Image = None) -> Image:
    """Grows every label into the zero voxels around it, box and diamond steps
    alternating, until the labels touch (_tier4/_extend_labeling_via_voronoi.py:13-60)."""
    return _grow_call("cle_extend_labeling_via_voronoi", labeling_source, labeling_destination)


@plugin_function(categories=['label', 'in assistant', 'bia-bob-suggestion'], output_creator=create_labels_like)
def voronoi_labeling(binary_source: Image, labeling_destination: Image = None) -> Image:
    """Connected components (box) of the binary image, then their Voronoi
    extension over the whole image (_tier5/_voronoi_labeling.py:8-40)."""
    return _grow_call("cle_voronoi_labeling", binary_source, labeling_destination)


# ---- measurement tables and parametric label maps ------------------------
class STATISTICS_ENTRY(Enum):
    """Column index of each measurement in the pushed statistics table; the
    same names and values as the reference's enum (_tier9/_statistics_entry.py),
    which code indexing such tables relies on."""
    IDENTIFIER = 0
    BOUNDING_BOX_X = 1
    BOUNDING_BOX_Y = 2
    BOUNDING_BOX_Z = 3
    BOUNDING_BOX_END_X = 4
    BOUNDING_BOX_END_Y = 5
    BOUNDING_BOX_END_Z = 6
    BOUNDING_BOX_WIDTH = 7
    BOUNDING_BOX_HEIGHT = 8
    BOUNDING_BOX_DEPTH = 9
    MINIMUM_INTENSITY = 10
    MAXIMUM_INTENSITY = 11
    MEAN_INTENSITY = 12
    SUM_INTENSITY = 13
    STANDARD_DEVIATION_INTENSITY = 14
    PIXEL_COUNT = 15
    SUM_INTENSITY_TIMES_X = 16
    SUM_INTENSITY_TIMES_Y = 17
    SUM_INTENSITY_TIMES_Z = 18
    MASS_CENTER_X = 19
    MASS_CENTER_Y = 20
    MASS_CENTER_Z = 21
    SUM_X = 22
    SUM_Y = 23
    SUM_Z = 24
    CENTROID_X = 25
    CENTROID_Y = 26
    CENTROID_Z = 27
    SUM_DISTANCE_TO_MASS_CENTER = 28
    MEAN_DISTANCE_TO_MASS_CENTER = 29
    MAX_DISTANCE_TO_MASS_CENTER = 30
    MAX_MEAN_DISTANCE_TO_MASS_CENTER_RATIO = 31
    SUM_DISTANCE_TO_CENTROID = 32
    MEAN_DISTANCE_TO_CENTROID = 33
    MAX_DISTANCE_TO_CENTROID = 34
    MAX_MEAN_DISTANCE_TO_CENTROID_RATIO = 35
    NUMBER_OF_ENTRIES = 36


# statistics dict key of each table row, in STATISTICS_ENTRY order
_ENTRY_KEYS = [
    "original_label", "bbox_min_x", "bbox_min_y", "bbox_min_z", "bbox_max_x", "bbox_max_y",
    "bbox_max_z", "bbox_width", "bbox_height", "bbox_depth", "min_intensity", "max_intensity",
    "mean_intensity", "sum_intensity", "standard_deviation_intensity", "area",
    "sum_intensity_times_x", "sum_intensity_times_y", "sum_intensity_times_z", "mass_center_x",
    "mass_center_y", "mass_center_z", "sum_x", "sum_y", "sum_z", "centroid_x", "centroid_y",
    "centroid_z", "sum_distance_to_mass_center", "mean_distance_to_mass_center",
    "max_distance_to_mass_center", "mean_max_distance_to_mass_center_ratio",
    "sum_distance_to_centroid", "mean_distance_to_centroid", "max_distance_to_centroid",
    "mean_max_distance_to_centroid_ratio",
]


@plugin_function(categories=['filter', 'in assistant'])
def add_image_and_scalar(source: Image, destination: Image = None, scalar: float = 1) -> Image:
    """destination = source + scalar in float32 (_tier1/_add_image_and_scalar.py)."""
    _call("cle_add_image_and_scalar", _lib.ref(_T(source)), _lib.ref(_T(destination)), float(scalar),
          _lib.stream_ptr())
    return destination


@plugin_function(categories=['bia-bob-suggestion'])
def replace_intensities(source: Image, new_values_vector: Image, destination: Image = None) -> Image:
    """destination = new_values_vector[(int) source], the index clamped to the
    vector (_tier1/_replace_intensities.py)."""
    _call("cle_replace_intensities", _lib.ref(_T(source)), _lib.ref(_T(new_values_vector)),
          _lib.ref(_T(destination)), _lib.stream_ptr())
    return destination


def statistics_of_background_and_labelled_pixels(source: Image = None, labelmap: Image = None):
    """Statistics of the background (original_label 0) and every label
    (_tier9/_statistics_of_background_and_labelled_pixels.py:9-45): the
    statistics of labelmap + 1."""
    from ._tier0 import push as _push
    temp = add_image_and_scalar(_push(labelmap), scalar=1)
    props = statistics_of_labelled_pixels(source, temp)
    props["original_label"] = props["label"] - 1
    return props


def push_regionprops(props, first_row_index: int = 0) -> B200Array:
    """The statistics as a 36-row table image, one column per label, rows in
    STATISTICS_ENTRY order (_tier9/_push_regionprops.py:8-135).  Accepts the
    statistics dict; the reference's scikit-image RegionProperties input is not
    supported here."""
    from ._tier0 import push as _push
    if not isinstance(props, dict):
        raise TypeError("push_regionprops: pass the dict returned by statistics_of_labelled_pixels")
    return _push(np.asarray([np.asarray(props[k], np.float64) for k in _ENTRY_KEYS]))


def push_regionprops_column(regionprops, column: str) -> B200Array:
    """One measurement as a 1-row image (_tier9/_push_regionprops_column.py): for
    the statistics dict its column as is; for a list of objects with `label`
    (or `original_label`) the values placed at their labels."""
    from ._tier0 import push as _push
    if isinstance(regionprops, dict):
        return _push(np.asarray([regionprops[column]]))
    labels = [getattr(r, "original_label", None) if hasattr(r, "original_label") else r.label for r in regionprops]
    values = np.zeros([int(np.max(labels)) + 1])
    for lab, r in zip(labels, regionprops):
        values[int(lab)] = getattr(r, column)
    return _push(np.asarray([values]))


def _label_map(intensity, labels, key, destination):
    """replace_intensities(labels, column `key` of the statistics of labels + 1
    with entry 0 set to 0): the label_*_map functions of _tier9, on the device
    (no host round trip of the statistics)."""
    from ._tier0 import push as _push
    labels = _push(labels)
    temp = add_image_and_scalar(labels, scalar=1)
    n = _label_max(temp)
    inten = temp if intensity is None else push_native(intensity)
    table = statistics_table(inten, temp, n)          # [35, n]: column j = original label j
    vec = table[STAT_KEYS.index(key)].reshape(1, n).clone()
    vec[0, 0] = 0
    if destination is None:
        destination = create_like(labels)
    return replace_intensities(labels, B200Array(vec), destination)


@plugin_function(categories=['label measurement', 'map', 'in assistant'])
def label_pixel_count_map(source: Image, destination: Image = None) -> Image:
    """Every label replaced by its voxel count (_tier9/_label_pixel_count_map.py)."""
    return _label_map(None, source, "area", destination)


@plugin_function(categories=['combine', 'label measurement', 'map', 'in assistant'], priority=-1)
def label_mean_intensity_map(source: Image, label_map: Image, destination: Image = None) -> Image:
    """Every label replaced by its mean intensity (_tier9/_label_mean_intensity_map.py)."""
    return _label_map(source, label_map, "mean_intensity", destination)


@plugin_function(categories=['combine', 'label measurement', 'map', 'in assistant'], priority=-1)
def label_minimum_intensity_map(intensity_image: Image, labels: Image, minimum_intensity_map: Image = None) -> Image:
    """Every label replaced by its minimum intensity (_tier9/_label_minimum_intensity_map.py)."""
    return _label_map(intensity_image, labels, "min_intensity", minimum_intensity_map)


@plugin_function(categories=['combine', 'label measurement', 'map', 'in assistant'], priority=-1)
def label_maximum_intensity_map(intensity_image: Image, labels: Image, maximum_intensity_map: Image = None) -> Image:
    """Every label replaced by its maximum intensity (_tier9/_label_maximum_intensity_map.py)."""
    return _label_map(intensity_image, labels, "max_intensity", maximum_intensity_map)


@plugin_function(categories=['combine', 'label measurement', 'map', 'in assistant'], priority=-1)
def label_standard_deviation_intensity_map(intensity_image: Image, labels: Image,
                                           standard_deviation_intensity_map: Image = None) -> Image:
    """Every label replaced by the standard deviation of its intensity
    (_tier9/_label_standard_deviation_intensity_map.py)."""
    return _label_map(intensity_image, labels, "standard_deviation_intensity", standard_deviation_intensity_map)


@plugin_function(categories=['label measurement', 'map', 'in assistant'])
def label_mean_extension_map(labels: Image, destination: Image = None) -> Image:
    """Every label replaced by the mean distance of its voxels to its centroid
    (_tier9/_label_mean_extension_map.py)."""
    return _label_map(None, labels, "mean_distance_to_centroid", destination)


@plugin_function(categories=['label measurement', 'map', 'in assistant'])
def label_maximum_extension_map(labels: Image, destination: Image = None) -> Image:
    """Every label replaced by the largest distance of its voxels to its
    centroid (_tier9/_label_maximum_extension_map.py)."""
    return _label_map(None, labels, "max_distance_to_centroid", destination)


@plugin_function(categories=['label measurement', 'map', 'in assistant'])
def label_maximum_extension_ratio_map(labels: Image, destination: Image = None) -> Image:
    """Every label replaced by its maximum over mean distance to the centroid
    (_tier9/_label_maximum_extension_ratio_map.py)."""
    return _label_map(None, labels, "mean_max_distance_to_centroid_ratio", destination)


@plugin_function(output_creator=create_none, categories=['bia-bob-suggestion'])
def centroids_of_labels(labels: Image, pointlist_destination: Image = None,
                        include_background: bool = False) -> Image:
    """Centroids of the labels as a float32 [d, n] point list: row 0 x, row 1 y
    (row 2 z in 3D), column = label (from label 0 with include_background,
    else from label 1); labels absent from the image get NaN
    (_tier9/_centroids_of_labels.py).  The coordinate sums are the statistics'
    exact integer sums, divided by the voxel count in float32, from one pass
    over the labels (cle_label_centroids)."""
    from ._tier0 import push as _push
    labels = _push(labels)
    temp = add_image_and_scalar(labels, scalar=1)
    n = _label_max(temp)                                # labels 0 .. n-1
    dims = 3 if len(labels.shape) == 3 else 2
    pts = torch.empty((dims, max(n, 0)), dtype=torch.float32, device=labels.tensor.device)
    if n > 0:
        t = _T(temp)
        ws = _ws("cle_label_centroids_workspace_bytes", _lib.ref(t), int(n), device=labels.tensor.device)
        _call("cle_label_centroids", _lib.ref(t), int(n), pts.data_ptr(), _ptr(ws), ws.numel(),
              _lib.stream_ptr())                        # column j = original label j
    if not include_background:
        pts = pts[:, 1:]
    pts = pts.contiguous()
    if pointlist_destination is None:
        return B200Array(pts)
    pointlist_destination.tensor[:, :pts.shape[1]].copy_(pts)
    return pointlist_destination


@plugin_function(output_creator=create_none)
def centroids_of_background_and_labels(source: Image, pointlist_destination: Image = None) -> Image:
    """centroids_of_labels with the background as column 0
    (_tier9/_centroids_of_background_and_labels.py)."""
    return centroids_of_labels(source, pointlist_destination, True)


@plugin_function(output_creator=create_none)
def euclidean_distance_from_label_centroid_map(labels: Image, centroids_pointlist: Image = None,
                                               distance_map_destination: Image = None) -> Image:
    """Every labelled voxel replaced by its distance to its label's centroid,
    background 0 (_tier9/_euclidean_distance_from_label_centroid_map.py); the
    centroids come from centroids_of_background_and_labels unless given."""
    if centroids_pointlist is None:
        centroids_pointlist = centroids_of_background_and_labels(labels)
    if distance_map_destination is None:
        distance_map_destination = create_like(labels)
    _call("cle_euclidean_distance_from_label_centroid_map", _lib.ref(_T(labels)),
          _lib.ref(_T(centroids_pointlist)), _lib.ref(_T(distance_map_destination)), _lib.stream_ptr())
    return distance_map_destination


# ---- distance / touch matrices and the neighbour-distance maps -------------
def _create_matrix_from_pointlists(pointlist1, pointlist2):
    """_tier0/_create.py create_matrix_from_pointlists: [m + 1, n + 1] float32."""
    return create([pointlist2.shape[1] + 1, pointlist1.shape[1] + 1])


def _create_square_matrix_from_labelmap(labelmap):
    """_tier0/_create.py create_square_matrix_from_labelmap: [L + 1, L + 1]."""
    n = _label_max(push(labelmap)) + 1
    return create([n, n])


def _create_vector_from_square_matrix(square_matrix, *args):
    """_tier0/_create.py create_vector_from_square_matrix: [1, rows]."""
    return create([1, square_matrix.shape[0]])


@plugin_function(output_creator=_create_matrix_from_pointlists)
def generate_distance_matrix(coordinate_list1: Image, coordinate_list2: Image,
                             distance_matrix_destination: Image = None) -> Image:
    """Distances between all points of two [d, n] point lists as an
    [m + 1, n + 1] float32 matrix, row and column 0 zero
    (_tier1/_generate_distance_matrix.py)."""
    _call("cle_generate_distance_matrix", _lib.ref(_T(coordinate_list1)), _lib.ref(_T(coordinate_list2)),
          _lib.ref(_T(distance_matrix_destination)), _lib.stream_ptr())
    return distance_matrix_destination


@plugin_function(output_creator=_create_square_matrix_from_labelmap)
def generate_touch_matrix(label_map: Image, touch_matrix_destination: Image = None) -> Image:
    """[L + 1, L + 1] matrix with 1 where two labels (the background 0
    included) meet across a face, both (a, b) and (b, a)
    (_tier1/_generate_touch_matrix.py, generate_touch_matrix_{2,3}d_x.cl)."""
    _call("cle_generate_touch_matrix", _lib.ref(_T(label_map)), _lib.ref(_T(touch_matrix_destination)),
          _lib.stream_ptr())
    return touch_matrix_destination


@plugin_function(output_creator=_create_vector_from_square_matrix)
def average_distance_of_n_shortest_distances(distance_matrix: Image, distance_vector_destination: Image = None,
                                             n: int = 1) -> Image:
    """Per column the mean of the n smallest distances in rows 1.., the
    column's own row left out (_tier1/_average_distance_of_n_shortest_distances.py)."""
    _call("cle_average_distance_of_n_distances", _lib.ref(_T(distance_matrix)), int(n), 1,
          _lib.ref(_T(distance_vector_destination)), _lib.stream_ptr())
    return distance_vector_destination


@plugin_function(output_creator=create_none)
def average_distance_of_n_nearest_distances(distance_matrix: Image, distance_vector_destination: Image = None,
                                            n: int = 1) -> Image:
    """Per column the mean of the n smallest distances in rows 1.., the
    column's own row included (_tier1/_average_distance_of_n_nearest_distances.py,
    average_distance_of_n_nearest_distances_x.cl); a [1, columns] vector."""
    if distance_vector_destination is None:
        distance_vector_destination = create([1, distance_matrix.shape[1]])
    _call("cle_average_distance_of_n_distances", _lib.ref(_T(distance_matrix)), int(n), 0,
          _lib.ref(_T(distance_vector_destination)), _lib.stream_ptr())
    return distance_vector_destination


@plugin_function(output_creator=_create_vector_from_square_matrix)
def average_distance_of_touching_neighbors(distance_matrix: Image, touch_matrix: Image,
                                           average_distancelist_destination: Image = None) -> Image:
    """Per label the mean distance to the labels it touches, the background
    left out, 0 for a label touching none
    (_tier1/_average_distance_of_touching_neighbors.py)."""
    _call("cle_average_distance_of_touching_neighbors", _lib.ref(_T(distance_matrix)), _lib.ref(_T(touch_matrix)),
          _lib.ref(_T(average_distancelist_destination)), _lib.stream_ptr())
    return average_distancelist_destination


def _n_nearest_vector(pts_a, pts_b, n, exclude_self):
    na, nb = pts_a.shape[1], pts_b.shape[1]
    vec = create([1, na + 1])
    if na == 0 or nb == 0:
        # an empty point list (an image without labels): the kernel's means
        # over no rows are 0 / 0 = NaN; column 0 (the background) over nb
        # zero distances is 0 when n >= 1
        vec.tensor.fill_(float("nan"))
        if nb > 0 and int(n) >= 1:
            vec.tensor[0, 0] = 0.0
        return vec
    _call("cle_average_distance_of_n_nearest_points", _lib.ref(_T(pts_a)), _lib.ref(_T(pts_b)), int(n),
          1 if exclude_self else 0, _lib.ref(_T(vec)), _lib.stream_ptr())
    return vec


@plugin_function(categories=['label measurement', 'map', 'in assistant'])
def average_distance_of_n_nearest_neighbors_map(labels: Image, distance_map: Image = None, n: int = 1) -> Image:
    """Every label replaced by the mean centroid distance to its n nearest other
    labels (_tier9/_average_distance_of_n_nearest_neighbors_map.py): the vector
    of average_distance_of_n_shortest_distances on the centroids' distance
    matrix, computed from the centroids without building the matrix, then
    replace_intensities."""
    centroids = centroids_of_labels(labels)
    vec = _n_nearest_vector(centroids, centroids, n, True)
    return replace_intensities(labels, vec, distance_map)


@plugin_function(categories=['label measurement', 'map', 'in assistant'])
def average_distance_to_n_nearest_other_labels_map(labels: Image, other_labels: Image, distance_map: Image = None,
                                                   n: int = 1) -> Image:
    """Every label replaced by the mean distance from its centroid to the n
    nearest centroids of other_labels
    (_tier9/_average_distance_to_n_nearest_other_labels_map.py; the vector of
    average_distance_of_n_nearest_distances, without the matrix)."""
    centroids_a = centroids_of_labels(labels)
    centroids_b = centroids_of_labels(other_labels)
    vec = _n_nearest_vector(centroids_a, centroids_b, n, False)
    return replace_intensities(labels, vec, distance_map)


@plugin_function(categories=['label measurement', 'in assistant'])
def average_neighbor_distance_map(labels: Image, distance_map: Image = None) -> Image:
    """Every label replaced by the mean centroid distance to the labels it
    touches (_tier9/_average_neighbor_distance_map.py): the vector of
    average_distance_of_touching_neighbors, from a bitmap of touching label
    pairs and the centroids instead of the two [L + 1, L + 1] matrices."""
    centroids = centroids_of_labels(labels)
    L = centroids.shape[1]
    vec = create([1, L + 1])
    if L == 0:
        vec.tensor.zero_()                      # no labels: nothing touches
        return replace_intensities(labels, vec, distance_map)
    ws = _ws("cle_average_distance_of_touching_labels_workspace_bytes", int(L), device=labels.tensor.device)
    _call("cle_average_distance_of_touching_labels", _lib.ref(_T(labels)), _lib.ref(_T(centroids)),
          _lib.ref(_T(vec)), _ptr(ws), ws.numel(), _lib.stream_ptr())
    return replace_intensities(labels, vec, distance_map)


def _box_call(name, source, destination, rx, ry, rz):
    s, d = _T(source), _T(destination)
    ws = _ws("cle_box_filter_workspace_bytes", _lib.ref(s))
    _call(name, _lib.ref(s), _lib.ref(d), float(rx), float(ry), float(rz), _ptr(ws), ws.numel(),
          _lib.stream_ptr())
    return destination


@plugin_function(categories=['filter', 'in assistant'], native_inputs=("source",))
def minimum_box(source: Image, destination: Image = None, radius_x: float = 0, radius_y: float = 0,
                radius_z: float = 0) -> Image:
    """Local minimum over a box of int(2*radius+1) voxels per axis, separable
    (_tier1/_minimum_box.py:6-55)."""
    return _box_call("cle_minimum_box", source, destination, radius_x, radius_y, radius_z)


@plugin_function(categories=['filter', 'in assistant'], native_inputs=("source",))
def maximum_box(source: Image, destination: Image = None, radius_x: float = 0, radius_y: float = 0,
                radius_z: float = 0) -> Image:
    """Local maximum over a box of int(2*radius+1) voxels per axis, separable
    (_tier1/_maximum_box.py)."""
    return _box_call("cle_maximum_box", source, destination, radius_x, radius_y, radius_z)


@plugin_function(categories=['filter', 'background removal', 'in assistant'], priority=1,
                 native_inputs=("source",))
def top_hat_box(source: Image, destination: Image = None, radius_x: float = 1, radius_y: float = 1,
                radius_z: float = 1) -> Image:
    """Background subtraction: source minus its opening (maximum_box of
    minimum_box), float32 (_tier2/_top_hat_box.py:6-43)."""
    return _box_call("cle_top_hat_box", source, destination, radius_x, radius_y, radius_z)


@plugin_function(categories=['binary processing'], output_creator=create_binary_like)
def erode_box(source: Image, destination: Image = None) -> Image:
    """Binary erosion over the Moore neighbourhood (_tier1/_erode_box.py:6-47):
    1 where the pixel and all of its 8 (2D) or 26 (3D) neighbours are nonzero,
    else 0; reads clamp to the image edge."""
    _call("cle_erode_box", _lib.ref(_T(source)), _lib.ref(_T(destination)), _lib.stream_ptr())
    return destination


@plugin_function(categories=['label', 'in assistant'], output_creator=create_labels_like,
                 native_inputs=("source",))
def gauss_otsu_labeling(source: Image, label_image_destination: Image = None,
                        outline_sigma: float = 2) -> Image:
    """Gaussian blur, Otsu threshold, connected components (box) of the binary
    image (_tier9/_gauss_otsu_labeling.py:6-45); every step a device kernel,
    no host round trip."""
    temp = create(source)                       # float32, like the reference's create(source)
    gaussian_blur(source, temp, outline_sigma, outline_sigma, outline_sigma)
    segmentation = threshold_otsu(temp)
    return connected_components_labeling_box(segmentation, label_image_destination)


@plugin_function(categories=['label', 'in assistant'], output_creator=create_labels_like,
                 native_inputs=("image",))
def eroded_otsu_labeling(image: Image, labels_destination: Image = None, number_of_erosions: int = 5,
                         outline_sigma: float = 2) -> Image:
    """Gaussian blur, Otsu threshold, int(number_of_erosions) box erosions, then
    the eroded objects' labels grown back inside the binary image by masked
    Voronoi labelling (_tier9/_eroded_otsu_labeling.py:4-62).  The eroded
    image lies inside the 0/1 binary image, so the growth runs on the
    active-front kernel."""
    blurred = create(image)
    gaussian_blur(image, blurred, outline_sigma, outline_sigma, outline_sigma)
    binary = threshold_otsu(blurred)
    eroded = B200Array(binary.tensor.clone())
    eroded1 = create_binary_like(binary)
    for _ in range(int(number_of_erosions)):
        erode_box(eroded, eroded1)
        eroded, eroded1 = eroded1, eroded
    return masked_voronoi_labeling_binary(eroded, binary, labels_destination)


class Workspaces:
    """Per-shape cache of voronoi_otsu_labeling workspaces (device memory is
    reused across calls on one stream; calls on different streams must not
    share one)."""

    def __init__(self):
        self._cache = {}

    def get(self, src: B200Array) -> torch.Tensor:
        key = (src.shape, src.tensor.dtype, src.tensor.device, torch.cuda.current_stream().cuda_stream)
        ws = self._cache.get(key)
        if ws is None:
            s = _T(src)
            n = _lib.load().cle_voronoi_otsu_labeling_workspace_bytes(_lib.ref(s))
            ws = _lib.workspace(n, src.tensor.device)
            self._cache[key] = ws
        return ws

    def clear(self):
        self._cache.clear()


workspaces = Workspaces()


def _vol(source: B200Array, dest: B200Array, spot_sigma, outline_sigma, check=True):
    ws = workspaces.get(source)
    s, d = _T(source), _T(dest)
    stream = _lib.stream_ptr()
    _call("cle_voronoi_otsu_labeling", _lib.ref(s), _lib.ref(d), float(spot_sigma),
          float(outline_sigma), _opts(), ws.data_ptr(), ws.numel(), stream)
    if check:
        _lib.check(_lib.load().cle_workspace_status(ws.data_ptr(), ws.numel(), stream),
                   "voronoi_otsu_labeling")
    return dest


@plugin_function(categories=['label', 'in assistant', 'bia-bob-suggestion'], priority=1,
                 output_creator=create_labels_like, native_inputs=("source",))
def voronoi_otsu_labeling(source: Image, label_image_destination: Image = None,
                          spot_sigma: float = 2, outline_sigma: float = 2) -> Image:
    """Gaussian blurs, spot detection, Otsu threshold and masked Voronoi growth
    (_tier9/_voronoi_otsu_labeling.py:11-73), one device pipeline with no
    host round trip; the device loop status is checked after the call."""
    return _vol(source, label_image_destination, spot_sigma, outline_sigma)


@plugin_function(output_creator=create_none, categories=['bia-bob-suggestion'],
                 native_inputs=("intensity_image",))
def statistics_of_labelled_pixels(intensity_image: Image = None, label_image: Image = None):
    """Per-label statistics dict (_tier9/_statistics_of_labelled_pixels.py:7-293)."""
    if intensity_image is None and label_image is None:
        raise ValueError("Either intensity image or labels must be set")
    if label_image is None:
        warnings.warn("No label image provided. All pixels will be analysed in one group.")
        label_image = B200Array(torch.ones(intensity_image.shape, dtype=torch.uint32,
                                           device=intensity_image.tensor.device))
    if intensity_image is None:
        intensity_image = label_image
    L = _label_max(label_image)
    table = statistics_table(intensity_image, label_image, L)
    host = table.cpu().numpy() if L > 0 else np.zeros((len(STAT_KEYS), 0), np.float32)
    out = {"label": np.arange(1, L + 1), "original_label": np.arange(1, L + 1)}
    for i, k in enumerate(STAT_KEYS):
        out[k] = host[i].copy()
    return out


statistics_of_labeled_pixels = statistics_of_labelled_pixels


def statistics_table(intensity: B200Array, labels: B200Array, num_labels: int) -> torch.Tensor:
    """Device float32 table [35, num_labels] (rows in STAT_KEYS order)."""
    dev = labels.tensor.device
    table = torch.empty((len(STAT_KEYS), max(num_labels, 0)), dtype=torch.float32, device=dev)
    if num_labels <= 0:
        return table
    i, l = _T(intensity), _T(labels)
    ws = _ws("cle_statistics_workspace_bytes", _lib.ref(l), int(num_labels), device=dev)
    _call("cle_statistics_of_labelled_pixels", _lib.ref(i), _lib.ref(l), int(num_labels),
          table.data_ptr(), _ptr(ws), ws.numel(), _lib.stream_ptr())
    return table
