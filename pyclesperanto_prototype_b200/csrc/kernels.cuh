// kernels.cuh -- internal (C++) interface between the op files and the C ABI.
#pragma once

#include "common.cuh"

namespace cle {

// blur.cu
size_t separable_workspace_bytes(const Img &im);
int separable_filter(const Img &src, float *dst, const Taps *tx, const Taps *ty, const Taps *tz,
                     Arena &ws, cudaStream_t st);
// status (optional): a device status word; given it, the fused path of a
// volume may stage planes with TMA copies and reports a stage wait that ran
// out there (CLE_ERR_ITER_LIMIT)
int gaussian_blur(const Img &src, float *dst, double sx, double sy, double sz, Arena &ws,
                  cudaStream_t st, int *status = nullptr);

// blur_fused.cu (isotropic sigma, radius <= kMaxFusedR, one launch)
constexpr int kMaxFusedR = 14;
bool fused_blur_applies(const Img &src, double sx, double sy, double sz);
// mm (optional): 2 floats per CTA, the CTA's min / max of the result
int fused_blur(const Img &src, float *dst, double sigma, cudaStream_t st, float *mm = nullptr,
               int *status = nullptr);
// Isotropic blur whose {min, max} lands in d_minmax (device): the fused
// launch's CTA partials and a one-CTA finish, or blur + minmax otherwise.
size_t blur_minmax_workspace_bytes(const Img &src);
int blur_minmax(const Img &src, float *dst, double sigma, float *d_minmax, Arena &ws, cudaStream_t st,
                int *status = nullptr);

// reduce.cu
size_t minmax_workspace_bytes(const Img &im);
// Writes {min, max} to d_out (device) without host synchronisation.
int minmax(const Img &im, float *d_out, Arena &ws, cudaStream_t st);
// {min, max} of `blocks` partial pairs into d_out (one CTA).
int minmax_finish(const float *partial, int blocks, float *d_out, cudaStream_t st);
size_t histogram_workspace_bytes(const Img &im, int bins);
// Row-partial histogram + float32 row sum (reference order); d_minmax holds {min,max}.
int histogram(const Img &im, int bins, const float *d_minmax, float *d_hist, Arena &ws,
              cudaStream_t st);
// Otsu on a 256-bin float32 histogram, device float64.  Writes the float64
// threshold to d_thr (may be null) and its float32 cast to d_thr32.
int otsu(const float *d_hist, const float *d_minmax, double *d_thr, float *d_thr32,
         cudaStream_t st);
int greater_constant(const Img &src, const Img &dst, float c, const float *d_c, cudaStream_t st);
int binary_and(const Img &a, const Img &b, const Img &dst, cudaStream_t st);
int mask_op(const Img &src, const Img &mask, const Img &dst, cudaStream_t st);

// morph.cu
int erode_box(const Img &src, const Img &dst, cudaStream_t st);
// maps.cu
int add_image_and_scalar(const Img &src, const Img &dst, float c, cudaStream_t st);
int replace_intensities(const Img &src, const Img &map, const Img &dst, cudaStream_t st);
int centroid_distance_map(const Img &labels, const Img &pts, const Img &dst, cudaStream_t st);
// neighbors.cu: distance / touch matrices and the neighbour-distance vectors
int generate_distance_matrix(const Img &list1, const Img &list2, const Img &dst, cudaStream_t st);
int generate_touch_matrix(const Img &labels, const Img &dst, cudaStream_t st);
int average_distance_of_n_distances(const Img &dm, int n, int exclude_self, const Img &dst, cudaStream_t st);
int average_distance_of_touching_neighbors(const Img &dm, const Img &tm, const Img &dst, cudaStream_t st);
int average_distance_of_n_points(const Img &list1, const Img &list2, int n, int exclude_self, const Img &dst,
                                 cudaStream_t st);
size_t touching_labels_workspace_bytes(int64_t num_labels);
int average_distance_of_touching_labels(const Img &labels, const Img &pts, const Img &dst, Arena &ws,
                                        cudaStream_t st);

size_t box_filter_workspace_bytes(const Img &im);
int box_filter(const Img &src, const Img &dst, double rx, double ry, double rz, bool is_max, Arena &ws,
               cudaStream_t st);
int top_hat_box(const Img &src, const Img &dst, double rx, double ry, double rz, Arena &ws, cudaStream_t st);
int label_max(const Img &labels, uint32_t *d_max, Arena &ws, cudaStream_t st);
size_t label_max_workspace_bytes(const Img &im);

// maxima.cu
int detect_maxima(const Img &src, const Img &dst, cudaStream_t st);
// detect_maxima_box(T) & (T > *d_thr32) in one pass over the float32 image T:
// seg = T > t, lab = key + 1 on seeds (0 elsewhere), seeds listed (count in
// *d_count, which must start at 0)
int maxima_seeds(const Img &T, const float *d_thr32, uint8_t *seg, uint32_t *lab, uint32_t *seeds,
                 uint32_t *d_count, cudaStream_t st);

// ccl.cu
size_t ccl_workspace_bytes(const Img &im);
// Dense CCL of (binary != 0) into u32 labels (x-major float32 key ranks).
// diamond: face connectivity (4 in 2D, 6 in 3D) instead of the 3^d box
int ccl_dense(const Img &binary, uint32_t *labels, Arena &ws, cudaStream_t st, bool diamond = false);
// CCL restricted to a device list of voxel indices whose entries in `labels`
// already hold (own x-major key + 1); on return those entries hold labels.
// d_count: device count of list entries; cap: list capacity.
int ccl_list(const Geo &g, int64_t n, uint32_t *labels, const uint32_t *list,
             const uint32_t *d_count, int64_t cap, Arena &ws, cudaStream_t st,
             uint32_t *d_nlabels = nullptr);
int ccl_to_dst(const uint32_t *lab, const Img &dst, cudaStream_t st);
size_t relabel_workspace_bytes(uint32_t max_label);
int relabel_sequential(const Img &src, const Img &dst, uint32_t max_label, Arena &ws,
                       cudaStream_t st);
size_t rank_workspace_bytes(uint64_t bits);

// voronoi.cu
size_t voronoi_frontier_workspace_bytes(const Img &im);
// Frontier-queued Jacobi growth.  labels: u32 with seed labels, 0 elsewhere;
// seg: u8 mask (0/1); seeds: device list of seed memory indices (count in
// d_seed_count).  d_status receives 0 or an error.
// gate: when set, the launch returns at once unless *gate != 0 on the device.
int voronoi_frontier(const Img &shape, uint32_t *labels, const uint8_t *seg,
                     const uint32_t *seeds, const uint32_t *d_seed_count, int *d_status,
                     Arena &ws, cudaStream_t st, const Limits &lim, const int *gate = nullptr);
// The same growth by arrival keys (bricks relaxed to convergence per visit,
// rounds instead of steps), for labels up to 2^24 - 1 (d_max_label: the
// largest seed label on the device) and up to 120 steps; otherwise the labels
// are left as given and the frontier kernel above grows them.  seg: mask
// bytes as the seed passes write them (kMaskByte); the growth keeps each
// labelled voxel's arrival step in them.  Workspace includes the frontier
// kernel's.
size_t voronoi_grow_workspace_bytes(const Img &im);
int voronoi_grow(const Img &shape, uint32_t *labels, uint8_t *seg, const uint32_t *seeds,
                 const uint32_t *d_seed_count, const uint32_t *d_max_label, int *d_status, Arena &ws,
                 cudaStream_t st, const Limits &lim);
size_t voronoi_dense_workspace_bytes(const Img &im);
int masked_voronoi_dense(const Img &binary, const Img &mask, const Img &dst, int *d_status,
                         Arena &ws, cudaStream_t st, const Limits &lim);

// stats.cu
size_t stats_workspace_bytes(const Img &labels, int64_t L);
int statistics(const Img &inten, const Img &labels, int64_t L, float *d_table, Arena &ws,
               cudaStream_t st, const uint32_t *d_L = nullptr);
// centroid_x/y(/z) of labels 1..n as a float32 [dims][n] point list (pass 1 sums only)
size_t centroids_workspace_bytes(int64_t n);
int label_centroids(const Img &labels, int64_t n, float *pts, Arena &ws, cudaStream_t st);

// pipeline.cu
size_t vol_workspace_bytes(const Img &im);
int voronoi_otsu_labeling(const Img &src, const Img &dst, double spot_sigma,
                          double outline_sigma, Arena &ws, cudaStream_t st, const Limits &lim);

// masked_voronoi_labeling for a 0/1 mask with every seed inside it (the
// composite's case), on the active-brick growth.
size_t masked_voronoi_binary_workspace_bytes(const Img &im);
int masked_voronoi_binary(const Img &bin, const Img &mask, const Img &dst, Arena &ws, cudaStream_t st,
                          const Limits &lim);
// extend_labeling_via_voronoi / voronoi_labeling (status word at workspace offset 0)
size_t extend_voronoi_workspace_bytes(const Img &im);
int extend_labeling_via_voronoi(const Img &src, const Img &dst, Arena &ws, cudaStream_t st,
                                const Limits &lim);
int voronoi_labeling(const Img &bin, const Img &dst, Arena &ws, cudaStream_t st, const Limits &lim);

// noalloc.cu: threshold_otsu with a built-in scratch array
size_t threshold_otsu_noalloc_capacity();
int threshold_otsu_noalloc(const Img &src, const Img &dst, cudaStream_t st);

// Status word at a fixed offset of every composite workspace (first 256 B).
int *workspace_status_ptr(void *ws);
uint32_t *workspace_label_count_ptr(void *ws);

}  // namespace cle
