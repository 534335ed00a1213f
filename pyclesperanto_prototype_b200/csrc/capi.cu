// capi.cu -- the extern "C" entry points declared in include/cle_b200.h.
#include "common.cuh"
#include "kernels.cuh"

using namespace cle;

namespace {

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

int set_device_of(const Img &im, const cle_tensor *t) {
    (void)im;
    int cur = -1;
    CLE_CUDA(cudaGetDevice(&cur));
    if (t && t->device >= 0 && t->device != cur) CLE_CUDA(cudaSetDevice(t->device));
    return CLE_OK;
}

int ws_check(void *ws, size_t bytes, size_t need, const char *who) {
    if (need && (!ws || bytes < need)) {
        set_error("%s: workspace of %zu bytes needed, %zu given", who, need, ws ? bytes : (size_t)0);
        return CLE_ERR_WORKSPACE;
    }
    if (ws && (reinterpret_cast<uintptr_t>(ws) & 255)) {
        set_error("%s: workspace must be 256-byte aligned", who);
        return CLE_ERR_WORKSPACE;
    }
    return CLE_OK;
}

}  // namespace

extern "C" {

int cle_abi_version(void) { return CLE_B200_ABI_VERSION; }
const char *cle_version(void) { return "cle_b200 1.0 (sm_100a)"; }
const char *cle_last_error_message(void) { return last_error(); }
unsigned long long cle_kernel_launches(void) { return launches_issued(); }
int cle_profile_enable(int flags) { return profile_enable(flags); }
int cle_profile_stage_ms(float *out, int max) { return stage_ms(out, max); }
int cle_profile_trace(void *host, size_t bytes) { return profile_trace_read(host, bytes); }

// ---- gaussian_blur -------------------------------------------------------
size_t cle_gaussian_blur_workspace_bytes(const cle_tensor *src) {
    Img im;
    if (to_img(src, im, "source")) return 0;
    return separable_workspace_bytes(im);
}

int cle_gaussian_blur(const cle_tensor *src, const cle_tensor *dst, double sx, double sy, double sz,
                      void *ws, size_t ws_bytes, void *stream) {
    Img a, b;
    CLE_TRY(to_img(src, a, "source"));
    CLE_TRY(to_img(dst, b, "destination"));
    CLE_TRY(same_shape(a, b, "source", "destination"));
    if (b.dtype != CLE_F32) { set_error("gaussian_blur: destination must be float32"); return CLE_ERR_DTYPE; }
    CLE_TRY(ws_check(ws, ws_bytes, separable_workspace_bytes(a), "gaussian_blur"));
    CLE_TRY(set_device_of(a, src));
    // the fused path of a volume reports a staging wait that ran out in the
    // workspace's first word (cle_workspace_status); the three-pass path
    // uses the workspace for its intermediates instead
    int *status = nullptr;
    if (a.ndim == 3 && fused_blur_applies(a, sx, sy, sz) && ws && ws_bytes >= sizeof(int)) {
        status = static_cast<int *>(ws);
        CLE_CUDA(cudaMemsetAsync(status, 0, sizeof(int), S(stream)));
    }
    Arena ar(ws, ws_bytes);
    return gaussian_blur(a, (float *)b.data, sx, sy, sz, ar, S(stream), status);
}

// ---- min / max -------------------------------------------------------------
size_t cle_minimum_maximum_workspace_bytes(const cle_tensor *src) {
    Img im;
    if (to_img(src, im, "source")) return 0;
    return minmax_workspace_bytes(im);
}

int cle_minimum_maximum(const cle_tensor *src, float *d_minmax, void *ws, size_t ws_bytes,
                        void *stream) {
    Img a;
    CLE_TRY(to_img(src, a, "source"));
    if (!d_minmax) { set_error("minimum_maximum: null output"); return CLE_ERR_ARG; }
    CLE_TRY(ws_check(ws, ws_bytes, minmax_workspace_bytes(a), "minimum_maximum"));
    CLE_TRY(set_device_of(a, src));
    Arena ar(ws, ws_bytes);
    return minmax(a, d_minmax, ar, S(stream));
}

// ---- histogram -------------------------------------------------------------
size_t cle_histogram_workspace_bytes(const cle_tensor *src, int bins) {
    Img im;
    if (to_img(src, im, "source") || bins < 1) return 0;
    return 256 + minmax_workspace_bytes(im) + histogram_workspace_bytes(im, bins);
}

int cle_histogram(const cle_tensor *src, const cle_tensor *dst, int bins, float mn, float mx,
                  int determine, void *ws, size_t ws_bytes, void *stream) {
    Img a, h;
    CLE_TRY(to_img(src, a, "source"));
    CLE_TRY(to_img(dst, h, "destination"));
    if (bins < 1) { set_error("histogram: num_bins must be >= 1"); return CLE_ERR_ARG; }
    if (h.dtype != CLE_F32 || h.n() != bins) {
        set_error("histogram: destination must be float32 with num_bins=%d elements", bins);
        return CLE_ERR_SHAPE;
    }
    CLE_TRY(ws_check(ws, ws_bytes, cle_histogram_workspace_bytes(src, bins), "histogram"));
    CLE_TRY(set_device_of(a, src));
    Arena ar(ws, ws_bytes);
    float *mm = ar.take<float>(64);
    if (determine) {
        CLE_TRY(minmax(a, mm, ar, S(stream)));
    } else {
        float host[2] = {mn, mx};
        CLE_CUDA(cudaMemcpyAsync(mm, host, sizeof(host), cudaMemcpyHostToDevice, S(stream)));
    }
    return histogram(a, bins, mm, (float *)h.data, ar, S(stream));
}

// ---- threshold_otsu ---------------------------------------------------------
size_t cle_threshold_otsu_workspace_bytes(const cle_tensor *src) {
    Img im;
    if (to_img(src, im, "source")) return 0;
    return 2048 + minmax_workspace_bytes(im) + histogram_workspace_bytes(im, 256);
}

int cle_threshold_otsu(const cle_tensor *src, const cle_tensor *dst, double *d_thr, void *ws,
                       size_t ws_bytes, void *stream) {
    Img a, b;
    CLE_TRY(to_img(src, a, "source"));
    CLE_TRY(to_img(dst, b, "destination"));
    CLE_TRY(same_shape(a, b, "source", "destination"));
    CLE_TRY(ws_check(ws, ws_bytes, cle_threshold_otsu_workspace_bytes(src), "threshold_otsu"));
    CLE_TRY(set_device_of(a, src));
    Arena ar(ws, ws_bytes);
    float *mm = ar.take<float>(64);       // {min,max}, thr32 at [2]
    float *hist = ar.take<float>(256);
    double *thr = ar.take<double>(4);
    CLE_TRY(minmax(a, mm, ar, S(stream)));
    CLE_TRY(histogram(a, 256, mm, hist, ar, S(stream)));
    CLE_TRY(otsu(hist, mm, d_thr ? d_thr : thr, mm + 2, S(stream)));
    return greater_constant(a, b, 0.0f, mm + 2, S(stream));
}

int cle_threshold_otsu_noalloc(const cle_tensor *src, const cle_tensor *dst, void *stream) {
    Img a, b;
    CLE_TRY(to_img(src, a, "source"));
    CLE_TRY(to_img(dst, b, "destination"));
    CLE_TRY(set_device_of(a, src));
    return threshold_otsu_noalloc(a, b, S(stream));
}

size_t cle_threshold_otsu_noalloc_scratch_bytes(void) { return threshold_otsu_noalloc_capacity(); }

// ---- element-wise -----------------------------------------------------------
int cle_greater_constant(const cle_tensor *src, const cle_tensor *dst, float c, void *stream) {
    Img a, b;
    CLE_TRY(to_img(src, a, "source"));
    CLE_TRY(to_img(dst, b, "destination"));
    CLE_TRY(set_device_of(a, src));
    return greater_constant(a, b, c, nullptr, S(stream));
}

int cle_binary_and(const cle_tensor *x, const cle_tensor *y, const cle_tensor *dst, void *stream) {
    Img a, b, d;
    CLE_TRY(to_img(x, a, "operand1"));
    CLE_TRY(to_img(y, b, "operand2"));
    CLE_TRY(to_img(dst, d, "destination"));
    CLE_TRY(set_device_of(a, x));
    return binary_and(a, b, d, S(stream));
}

int cle_mask(const cle_tensor *src, const cle_tensor *msk, const cle_tensor *dst, void *stream) {
    Img a, m, d;
    CLE_TRY(to_img(src, a, "source"));
    CLE_TRY(to_img(msk, m, "mask"));
    CLE_TRY(to_img(dst, d, "destination"));
    CLE_TRY(set_device_of(a, src));
    return mask_op(a, m, d, S(stream));
}

int cle_erode_box(const cle_tensor *src, const cle_tensor *dst, void *stream) {
    Img a, d;
    CLE_TRY(to_img(src, a, "source"));
    CLE_TRY(to_img(dst, d, "destination"));
    CLE_TRY(set_device_of(a, src));
    return erode_box(a, d, S(stream));
}

int cle_add_image_and_scalar(const cle_tensor *src, const cle_tensor *dst, float scalar, void *stream) {
    Img a, d;
    CLE_TRY(to_img(src, a, "source"));
    CLE_TRY(to_img(dst, d, "destination"));
    CLE_TRY(set_device_of(a, src));
    return add_image_and_scalar(a, d, scalar, S(stream));
}

int cle_replace_intensities(const cle_tensor *src, const cle_tensor *map, const cle_tensor *dst, void *stream) {
    Img a, m, d;
    CLE_TRY(to_img(src, a, "source"));
    CLE_TRY(to_img(map, m, "new_values_vector"));
    CLE_TRY(to_img(dst, d, "destination"));
    CLE_TRY(set_device_of(a, src));
    return replace_intensities(a, m, d, S(stream));
}

int cle_euclidean_distance_from_label_centroid_map(const cle_tensor *labels, const cle_tensor *centroids,
                                                   const cle_tensor *dst, void *stream) {
    Img a, p, d;
    CLE_TRY(to_img(labels, a, "labels"));
    CLE_TRY(to_img(centroids, p, "centroids_pointlist"));
    CLE_TRY(to_img(dst, d, "distance_map_destination"));
    CLE_TRY(set_device_of(a, labels));
    return centroid_distance_map(a, p, d, S(stream));
}

int cle_generate_distance_matrix(const cle_tensor *list1, const cle_tensor *list2, const cle_tensor *dst,
                                 void *stream) {
    Img a, b, d;
    CLE_TRY(to_img(list1, a, "coordinate_list1"));
    CLE_TRY(to_img(list2, b, "coordinate_list2"));
    CLE_TRY(to_img(dst, d, "distance_matrix_destination"));
    CLE_TRY(set_device_of(a, list1));
    return generate_distance_matrix(a, b, d, S(stream));
}

int cle_generate_touch_matrix(const cle_tensor *labels, const cle_tensor *dst, void *stream) {
    Img a, d;
    CLE_TRY(to_img(labels, a, "label_map"));
    CLE_TRY(to_img(dst, d, "touch_matrix_destination"));
    CLE_TRY(set_device_of(a, labels));
    return generate_touch_matrix(a, d, S(stream));
}

int cle_average_distance_of_n_distances(const cle_tensor *distance_matrix, int n, int exclude_self,
                                        const cle_tensor *dst, void *stream) {
    Img m, d;
    CLE_TRY(to_img(distance_matrix, m, "distance_matrix"));
    CLE_TRY(to_img(dst, d, "distance_vector_destination"));
    CLE_TRY(set_device_of(m, distance_matrix));
    return average_distance_of_n_distances(m, n, exclude_self, d, S(stream));
}

int cle_average_distance_of_touching_neighbors(const cle_tensor *distance_matrix, const cle_tensor *touch_matrix,
                                               const cle_tensor *dst, void *stream) {
    Img m, t, d;
    CLE_TRY(to_img(distance_matrix, m, "distance_matrix"));
    CLE_TRY(to_img(touch_matrix, t, "touch_matrix"));
    CLE_TRY(to_img(dst, d, "average_distancelist_destination"));
    CLE_TRY(set_device_of(m, distance_matrix));
    return average_distance_of_touching_neighbors(m, t, d, S(stream));
}

int cle_average_distance_of_n_nearest_points(const cle_tensor *list1, const cle_tensor *list2, int n,
                                             int exclude_self, const cle_tensor *dst, void *stream) {
    Img a, b, d;
    CLE_TRY(to_img(list1, a, "pointlist1"));
    CLE_TRY(to_img(list2, b, "pointlist2"));
    CLE_TRY(to_img(dst, d, "distance_vector_destination"));
    CLE_TRY(set_device_of(a, list1));
    return average_distance_of_n_points(a, b, n, exclude_self, d, S(stream));
}

size_t cle_average_distance_of_touching_labels_workspace_bytes(int64_t num_labels) {
    return touching_labels_workspace_bytes(num_labels);
}

int cle_average_distance_of_touching_labels(const cle_tensor *labels, const cle_tensor *centroids,
                                            const cle_tensor *dst, void *ws, size_t ws_bytes, void *stream) {
    Img a, p, d;
    CLE_TRY(to_img(labels, a, "labels"));
    CLE_TRY(to_img(centroids, p, "centroids"));
    CLE_TRY(to_img(dst, d, "distance_vector_destination"));
    CLE_TRY(ws_check(ws, ws_bytes, touching_labels_workspace_bytes(p.W), "average_neighbor_distance_map"));
    CLE_TRY(set_device_of(a, labels));
    Arena ar(ws, ws_bytes);
    return average_distance_of_touching_labels(a, p, d, ar, S(stream));
}

size_t cle_box_filter_workspace_bytes(const cle_tensor *src) {
    Img im;
    if (to_img(src, im, "source")) return 0;
    return box_filter_workspace_bytes(im);
}

static int box_entry(const cle_tensor *src, const cle_tensor *dst, double rx, double ry, double rz, int kind,
                     void *ws, size_t ws_bytes, void *stream) {
    static const char *names[3] = {"minimum_box", "maximum_box", "top_hat_box"};
    Img a, d;
    CLE_TRY(to_img(src, a, "source"));
    CLE_TRY(to_img(dst, d, "destination"));
    CLE_TRY(ws_check(ws, ws_bytes, box_filter_workspace_bytes(a), names[kind]));
    CLE_TRY(set_device_of(a, src));
    Arena ar(ws, ws_bytes);
    if (kind == 2) return top_hat_box(a, d, rx, ry, rz, ar, S(stream));
    return box_filter(a, d, rx, ry, rz, kind == 1, ar, S(stream));
}

int cle_minimum_box(const cle_tensor *src, const cle_tensor *dst, double rx, double ry, double rz, void *ws,
                    size_t ws_bytes, void *stream) {
    return box_entry(src, dst, rx, ry, rz, 0, ws, ws_bytes, stream);
}

int cle_maximum_box(const cle_tensor *src, const cle_tensor *dst, double rx, double ry, double rz, void *ws,
                    size_t ws_bytes, void *stream) {
    return box_entry(src, dst, rx, ry, rz, 1, ws, ws_bytes, stream);
}

int cle_top_hat_box(const cle_tensor *src, const cle_tensor *dst, double rx, double ry, double rz, void *ws,
                    size_t ws_bytes, void *stream) {
    return box_entry(src, dst, rx, ry, rz, 2, ws, ws_bytes, stream);
}

// ---- detect_maxima_box -------------------------------------------------------
size_t cle_detect_maxima_box_workspace_bytes(const cle_tensor *src, int rx, int ry, int rz) {
    Img im;
    if (to_img(src, im, "source")) return 0;
    if (rx <= 0 && ry <= 0 && (rz <= 0 || im.ndim == 2)) return 0;
    return sizeof(float) * (size_t)im.n() + 256 + separable_workspace_bytes(im);
}

static void box_taps(int r, Taps &t) {
    // mean_box: N = 2r+1 uniform float32 weights (the missing mean_separable
    // kernel's op order is not pinned; the fused multiply-add chain is used)
    t.n = 2 * r + 1;
    for (int i = 0; i < t.n; ++i) t.w[i] = (float)(1.0 / (double)t.n);
}

int cle_detect_maxima_box(const cle_tensor *src, const cle_tensor *dst, int rx, int ry, int rz,
                          void *ws, size_t ws_bytes, void *stream) {
    Img a, d;
    CLE_TRY(to_img(src, a, "source"));
    CLE_TRY(to_img(dst, d, "destination"));
    CLE_TRY(same_shape(a, d, "source", "destination"));
    CLE_TRY(set_device_of(a, src));
    const size_t need = cle_detect_maxima_box_workspace_bytes(src, rx, ry, rz);
    if (need == 0) return detect_maxima(a, d, S(stream));
    CLE_TRY(ws_check(ws, ws_bytes, need, "detect_maxima_box"));
    if (2 * std::max(rx, std::max(ry, rz)) + 1 > kMaxTaps) { set_error("detect_maxima_box: radius too large"); return CLE_ERR_ARG; }
    Arena ar(ws, ws_bytes);
    float *mean = ar.take<float>(a.n());
    Taps tx, ty, tz;
    box_taps(rx > 0 ? rx : 0, tx);
    box_taps(ry > 0 ? ry : 0, ty);
    box_taps(rz > 0 ? rz : 0, tz);
    CLE_TRY(separable_filter(a, mean, rx > 0 ? &tx : nullptr, ry > 0 ? &ty : nullptr,
                             (a.ndim == 3 && rz > 0) ? &tz : nullptr, ar, S(stream)));
    Img mi = a;
    mi.data = mean;
    mi.dtype = CLE_F32;
    return detect_maxima(mi, d, S(stream));
}

// ---- CCL ---------------------------------------------------------------------
size_t cle_connected_components_labeling_box_workspace_bytes(const cle_tensor *bin) {
    Img im;
    if (to_img(bin, im, "binary_input")) return 0;
    return ccl_workspace_bytes(im);
}

int cle_connected_components_labeling_box(const cle_tensor *bin, const cle_tensor *dst, void *ws,
                                          size_t ws_bytes, void *stream) {
    Img a, d;
    CLE_TRY(to_img(bin, a, "binary_input"));
    CLE_TRY(to_img(dst, d, "labeling_destination"));
    CLE_TRY(same_shape(a, d, "binary_input", "labeling_destination"));
    if (d.dtype != CLE_U32 && d.dtype != CLE_F32) { set_error("connected_components_labeling_box: destination must be uint32 or float32"); return CLE_ERR_DTYPE; }
    CLE_TRY(ws_check(ws, ws_bytes, ccl_workspace_bytes(a), "connected_components_labeling_box"));
    CLE_TRY(set_device_of(a, bin));
    Arena ar(ws, ws_bytes);
    uint32_t *lab = ar.take<uint32_t>(a.n());
    if (d.dtype == CLE_U32) lab = (uint32_t *)d.data;
    CLE_TRY(ccl_dense(a, lab, ar, S(stream)));
    if (d.dtype == CLE_F32) return ccl_to_dst(lab, d, S(stream));
    return CLE_OK;
}

// ---- relabel_sequential ----------------------------------------------------------
size_t cle_relabel_sequential_workspace_bytes(const cle_tensor *src, uint32_t max_label) {
    Img im;
    if (to_img(src, im, "source")) return 0;
    return relabel_workspace_bytes(max_label);
}

int cle_relabel_sequential(const cle_tensor *src, const cle_tensor *dst, uint32_t max_label,
                           void *ws, size_t ws_bytes, void *stream) {
    Img a, d;
    CLE_TRY(to_img(src, a, "source"));
    CLE_TRY(to_img(dst, d, "output"));
    CLE_TRY(ws_check(ws, ws_bytes, relabel_workspace_bytes(max_label), "relabel_sequential"));
    CLE_TRY(set_device_of(a, src));
    Arena ar(ws, ws_bytes);
    return relabel_sequential(a, d, max_label, ar, S(stream));
}

// ---- masked_voronoi_labeling (general form) ---------------------------------------
size_t cle_masked_voronoi_labeling_workspace_bytes(const cle_tensor *bin) {
    Img im;
    if (to_img(bin, im, "binary_source")) return 0;
    return 256 + voronoi_dense_workspace_bytes(im);
}

int cle_masked_voronoi_labeling(const cle_tensor *bin, const cle_tensor *msk, const cle_tensor *dst,
                                const cle_call_options *opts, void *ws, size_t ws_bytes, void *stream) {
    Img a, m, d;
    Limits lim;
    CLE_TRY(limits_from(opts, lim));
    CLE_TRY(to_img(bin, a, "binary_source"));
    CLE_TRY(to_img(msk, m, "mask_image"));
    CLE_TRY(to_img(dst, d, "labeling_destination"));
    if (d.dtype != CLE_U32 && d.dtype != CLE_F32) { set_error("masked_voronoi_labeling: destination must be uint32 or float32"); return CLE_ERR_DTYPE; }
    CLE_TRY(ws_check(ws, ws_bytes, cle_masked_voronoi_labeling_workspace_bytes(bin), "masked_voronoi_labeling"));
    CLE_TRY(set_device_of(a, bin));
    Arena ar(ws, ws_bytes);
    int *status = ar.take<int>(64);
    CLE_CUDA(cudaMemsetAsync(status, 0, sizeof(int), S(stream)));
    return masked_voronoi_dense(a, m, d, status, ar, S(stream), lim);
}

size_t cle_connected_components_labeling_diamond_workspace_bytes(const cle_tensor *bin) {
    Img im;
    if (to_img(bin, im, "binary_input")) return 0;
    return ccl_workspace_bytes(im);
}

int cle_connected_components_labeling_diamond(const cle_tensor *bin, const cle_tensor *dst, void *ws,
                                              size_t ws_bytes, void *stream) {
    Img a, d;
    CLE_TRY(to_img(bin, a, "binary_input"));
    CLE_TRY(to_img(dst, d, "labeling_destination"));
    CLE_TRY(same_shape(a, d, "binary_input", "labeling_destination"));
    if (d.dtype != CLE_U32 && d.dtype != CLE_F32) { set_error("connected_components_labeling_diamond: destination must be uint32 or float32"); return CLE_ERR_DTYPE; }
    CLE_TRY(ws_check(ws, ws_bytes, ccl_workspace_bytes(a), "connected_components_labeling_diamond"));
    CLE_TRY(set_device_of(a, bin));
    Arena ar(ws, ws_bytes);
    uint32_t *lab = ar.take<uint32_t>(a.n());
    if (d.dtype == CLE_U32) lab = (uint32_t *)d.data;
    CLE_TRY(ccl_dense(a, lab, ar, S(stream), true));
    if (d.dtype == CLE_F32) return ccl_to_dst(lab, d, S(stream));
    return CLE_OK;
}

size_t cle_extend_labeling_via_voronoi_workspace_bytes(const cle_tensor *src) {
    Img im;
    if (to_img(src, im, "labeling_source")) return 0;
    return extend_voronoi_workspace_bytes(im);
}

int cle_extend_labeling_via_voronoi(const cle_tensor *src, const cle_tensor *dst,
                                    const cle_call_options *opts, void *ws, size_t ws_bytes, void *stream) {
    Img a, d;
    Limits lim;
    CLE_TRY(limits_from(opts, lim));
    CLE_TRY(to_img(src, a, "labeling_source"));
    CLE_TRY(to_img(dst, d, "labeling_destination"));
    CLE_TRY(ws_check(ws, ws_bytes, extend_voronoi_workspace_bytes(a), "extend_labeling_via_voronoi"));
    CLE_TRY(set_device_of(a, src));
    Arena ar(ws, ws_bytes);
    return extend_labeling_via_voronoi(a, d, ar, S(stream), lim);
}

size_t cle_voronoi_labeling_workspace_bytes(const cle_tensor *bin) {
    Img im;
    if (to_img(bin, im, "binary_source")) return 0;
    return extend_voronoi_workspace_bytes(im);
}

int cle_voronoi_labeling(const cle_tensor *bin, const cle_tensor *dst, const cle_call_options *opts,
                         void *ws, size_t ws_bytes, void *stream) {
    Img a, d;
    Limits lim;
    CLE_TRY(limits_from(opts, lim));
    CLE_TRY(to_img(bin, a, "binary_source"));
    CLE_TRY(to_img(dst, d, "labeling_destination"));
    CLE_TRY(ws_check(ws, ws_bytes, extend_voronoi_workspace_bytes(a), "voronoi_labeling"));
    CLE_TRY(set_device_of(a, bin));
    Arena ar(ws, ws_bytes);
    return voronoi_labeling(a, d, ar, S(stream), lim);
}

size_t cle_masked_voronoi_labeling_binary_workspace_bytes(const cle_tensor *bin) {
    Img im;
    if (to_img(bin, im, "binary_source")) return 0;
    return masked_voronoi_binary_workspace_bytes(im);
}

int cle_masked_voronoi_labeling_binary(const cle_tensor *bin, const cle_tensor *msk,
                                       const cle_tensor *dst, const cle_call_options *opts, void *ws,
                                       size_t ws_bytes, void *stream) {
    Img a, m, d;
    Limits lim;
    CLE_TRY(limits_from(opts, lim));
    CLE_TRY(to_img(bin, a, "binary_source"));
    CLE_TRY(to_img(msk, m, "mask_image"));
    CLE_TRY(to_img(dst, d, "labeling_destination"));
    CLE_TRY(ws_check(ws, ws_bytes, masked_voronoi_binary_workspace_bytes(a), "masked_voronoi_labeling"));
    CLE_TRY(set_device_of(a, bin));
    Arena ar(ws, ws_bytes);
    return masked_voronoi_binary(a, m, d, ar, S(stream), lim);
}

// ---- voronoi_otsu_labeling ----------------------------------------------------------
size_t cle_voronoi_otsu_labeling_workspace_bytes(const cle_tensor *src) {
    Img im;
    if (to_img(src, im, "source")) return 0;
    return vol_workspace_bytes(im);
}

int cle_voronoi_otsu_labeling(const cle_tensor *src, const cle_tensor *dst, double spot_sigma,
                              double outline_sigma, const cle_call_options *opts, void *ws,
                              size_t ws_bytes, void *stream) {
    Img a, d;
    Limits lim;
    CLE_TRY(limits_from(opts, lim));
    CLE_TRY(to_img(src, a, "source"));
    CLE_TRY(to_img(dst, d, "label_image_destination"));
    CLE_TRY(ws_check(ws, ws_bytes, vol_workspace_bytes(a), "voronoi_otsu_labeling"));
    CLE_TRY(set_device_of(a, src));
    Arena ar(ws, ws_bytes);
    return voronoi_otsu_labeling(a, d, spot_sigma, outline_sigma, ar, S(stream), lim);
}

const uint32_t *cle_workspace_label_count(const void *ws) {
    return ws ? workspace_label_count_ptr(const_cast<void *>(ws)) : nullptr;
}

int cle_workspace_status(const void *ws, size_t ws_bytes, void *stream) {
    if (!ws || ws_bytes < sizeof(int)) { set_error("workspace_status: no workspace"); return CLE_ERR_WORKSPACE; }
    int v = 0;
    CLE_CUDA(cudaMemcpyAsync(&v, workspace_status_ptr(const_cast<void *>(ws)), sizeof(int),
                             cudaMemcpyDeviceToHost, S(stream)));
    CLE_CUDA(cudaStreamSynchronize(S(stream)));
    if (v) set_error("device loop reported status %d (iteration or time limit)", v);
    return v;
}

// ---- label maximum / statistics -----------------------------------------------------
size_t cle_label_maximum_workspace_bytes(const cle_tensor *) { return 0; }

int cle_label_maximum(const cle_tensor *labels, uint32_t *d_max, void *ws, size_t ws_bytes,
                      void *stream) {
    Img a;
    CLE_TRY(to_img(labels, a, "label_image"));
    if (!d_max) { set_error("label_maximum: null output"); return CLE_ERR_ARG; }
    CLE_TRY(set_device_of(a, labels));
    Arena ar(ws, ws_bytes);
    return label_max(a, d_max, ar, S(stream));
}

size_t cle_statistics_workspace_bytes(const cle_tensor *labels, int64_t L) {
    Img im;
    if (to_img(labels, im, "label_image")) return 0;
    return stats_workspace_bytes(im, L);
}

int cle_statistics_of_labelled_pixels(const cle_tensor *inten, const cle_tensor *labels, int64_t L,
                                      float *d_table, void *ws, size_t ws_bytes, void *stream) {
    Img a, b;
    CLE_TRY(to_img(inten, a, "intensity_image"));
    CLE_TRY(to_img(labels, b, "label_image"));
    if (L > 0 && !d_table) { set_error("statistics: null table"); return CLE_ERR_ARG; }
    CLE_TRY(ws_check(ws, ws_bytes, L > 0 ? stats_workspace_bytes(b, L) : 0, "statistics_of_labelled_pixels"));
    CLE_TRY(set_device_of(a, inten));
    Arena ar(ws, ws_bytes);
    return statistics(a, b, L, d_table, ar, S(stream));
}

size_t cle_label_centroids_workspace_bytes(const cle_tensor *, int64_t num_labels) {
    return num_labels > 0 ? centroids_workspace_bytes(num_labels) : 0;
}

int cle_label_centroids(const cle_tensor *labels, int64_t num_labels, float *d_points, void *ws,
                        size_t ws_bytes, void *stream) {
    Img b;
    CLE_TRY(to_img(labels, b, "label_image"));
    if (num_labels > 0 && !d_points) { set_error("centroids: null point list"); return CLE_ERR_ARG; }
    CLE_TRY(ws_check(ws, ws_bytes, num_labels > 0 ? centroids_workspace_bytes(num_labels) : 0, "centroids_of_labels"));
    CLE_TRY(set_device_of(b, labels));
    Arena ar(ws, ws_bytes);
    return label_centroids(b, num_labels, d_points, ar, S(stream));
}

int cle_statistics_of_labelled_pixels_device_count(const cle_tensor *inten, const cle_tensor *labels,
                                                   const uint32_t *d_num_labels, int64_t capacity,
                                                   float *d_table, void *ws, size_t ws_bytes,
                                                   void *stream) {
    Img a, b;
    CLE_TRY(to_img(inten, a, "intensity_image"));
    CLE_TRY(to_img(labels, b, "label_image"));
    if (!d_num_labels || !d_table || capacity < 1) { set_error("statistics: null count/table or capacity < 1"); return CLE_ERR_ARG; }
    CLE_TRY(ws_check(ws, ws_bytes, stats_workspace_bytes(b, capacity), "statistics_of_labelled_pixels"));
    CLE_TRY(set_device_of(a, inten));
    Arena ar(ws, ws_bytes);
    return statistics(a, b, capacity, d_table, ar, S(stream), d_num_labels);
}

}  // extern "C"
