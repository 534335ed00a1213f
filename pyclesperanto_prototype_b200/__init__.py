"""pyclesperanto_prototype_b200 -- the voronoi_otsu_labeling +
statistics_of_labelled_pixels path of pyclesperanto_prototype, as hand-written
sm_100a CUDA kernels behind the reference's cle.* signatures.

    import pyclesperanto_prototype_b200 as cle
    labels = cle.voronoi_otsu_labeling(image, spot_sigma=2, outline_sigma=1)
    stats = cle.statistics_of_labelled_pixels(image, labels)

Device images are torch CUDA tensors wrapped in B200Array; the kernels live in
libcle_b200.so (C ABI, include/cle_b200.h), reached through ctypes.  Without
the library or a CUDA device the ops raise; there is no CPU fallback.
"""
from ._tier0 import (B200Array, B200Backend, Backend, Image, asarray, create, create_binary_like,
                     create_labels_like, create_like, create_none, create_zyx, is_image, nparray,
                     plugin_function, pull, pull_zyx, push, push_native, push_zyx)
from ._ops import (average_distance_of_n_nearest_distances, average_distance_of_n_nearest_neighbors_map,
                   average_distance_of_n_shortest_distances, average_distance_of_touching_neighbors,
                   average_distance_to_n_nearest_other_labels_map, average_neighbor_distance_map,
                   generate_distance_matrix, generate_touch_matrix)
from ._ops import (STATISTICS_ENTRY, add_image_and_scalar, centroids_of_background_and_labels,
                   centroids_of_labels, euclidean_distance_from_label_centroid_map,
                   label_maximum_extension_map,
                   label_maximum_extension_ratio_map, label_maximum_intensity_map,
                   label_mean_extension_map, label_mean_intensity_map, label_minimum_intensity_map,
                   label_pixel_count_map, label_standard_deviation_intensity_map, push_regionprops,
                   push_regionprops_column, replace_intensities,
                   statistics_of_background_and_labelled_pixels)
from ._ops import (binary_and, call_options, connected_components_labeling_box,
                   connected_components_labeling_diamond, detect_maxima_box,
                   erode_box, eroded_otsu_labeling, extend_labeling_via_voronoi, gauss_otsu_labeling,
                   voronoi_labeling,
                   gaussian_blur, greater_constant, histogram, mask, masked_voronoi_labeling,
                   maximum_box, minimum_box, top_hat_box,
                   masked_voronoi_labeling_binary,
                   maximum_of_all_pixels, minimum_of_all_pixels, radius_to_kernel_size,
                   relabel_sequential, scikit_image_threshold_otsu, sigma_to_kernel_size,
                   statistics_of_labeled_pixels, statistics_of_labelled_pixels, statistics_table,
                   threshold_otsu, voronoi_otsu_labeling, workspaces, STAT_KEYS)

__version__ = "0.1.0"
__common_alias__ = "cle"


def get_device():
    import torch
    from . import _lib
    _lib.load()
    return torch.cuda.get_device_name(torch.cuda.current_device())


def select_device(name: str = "", dev_type: str = "all", score_key=None, device_index: int = None):
    """Selects the CUDA device whose name contains `name` (or device_index),
    like the reference's select_device (_tier0/_device.py:48-84)."""
    import torch
    from . import _lib
    _lib.load()
    if device_index is not None:
        torch.cuda.set_device(int(device_index))
        return get_device()
    for i in range(torch.cuda.device_count()):
        if name.lower() in torch.cuda.get_device_name(i).lower():
            torch.cuda.set_device(i)
            return get_device()
    return get_device()


def available_device_names(dev_type: str = None, score_key=None):
    import torch
    return [torch.cuda.get_device_name(i) for i in range(torch.cuda.device_count())]


def set_wait_for_kernel_finish(wait: bool = None):
    """Kept for API compatibility: launches are stream-ordered; synchronise
    with torch.cuda.synchronize() when timing."""
    return None
