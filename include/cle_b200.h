/*
 * cle_b200.h -- C ABI of libcle_b200.so, the sm_100a implementation of
 * pyclesperanto_prototype's voronoi_otsu_labeling + statistics path.
 *
 * Conventions
 *   - Every image is a cle_tensor: a device pointer plus numpy-order shape
 *     (z, y, x) for 3D or (y, x) for 2D, C-contiguous (strides are element
 *     strides and are validated), dtype code and CUDA device ordinal.
 *   - Every compute entry point is asynchronous on the given CUDA stream
 *     (a cudaStream_t passed as void*; NULL = the legacy default stream) and
 *     returns a cle_status.  On failure cle_last_error_message() (thread
 *     local) holds a description.
 *   - Entry points never allocate device memory.  Scratch comes from a
 *     caller-provided workspace; its size is returned by the matching
 *     *_workspace_bytes() query (0 means none needed).  Workspaces must be
 *     256-byte aligned and must not be shared by calls that may overlap.
 *   - Output dtypes follow the reference's output creators
 *     (_tier0/_create.py:26-52): float32 (create_like), uint8
 *     (create_binary_like), uint32 (create_labels_like).  Where the
 *     reference also accepts a caller destination of another type the
 *     entry point converts the way the reference's WRITE_IMAGE does.
 *
 * The "replaces" line on each entry point names the reference function
 * (pyclesperanto_prototype/<file>:<line>) whose behaviour it implements.
 */
#ifndef CLE_B200_H
#define CLE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CLE_B200_ABI_VERSION 2

typedef enum cle_dtype {
    CLE_U8 = 1,
    CLE_U16 = 2,
    CLE_U32 = 3,
    CLE_I32 = 4,
    CLE_F32 = 5
} cle_dtype;

typedef enum cle_status {
    CLE_OK = 0,
    CLE_ERR_DTYPE = 1,      /* unsupported dtype              -> KeyError   */
    CLE_ERR_SHAPE = 2,      /* shapes disagree / not 2D or 3D -> ValueError */
    CLE_ERR_ARG = 3,        /* bad scalar argument            -> ValueError */
    CLE_ERR_WORKSPACE = 4,  /* workspace missing or too small -> RuntimeError */
    CLE_ERR_ITER_LIMIT = 5, /* device loop hit its step/time limit          */
    CLE_ERR_CUDA = 6,       /* CUDA runtime error             -> RuntimeError */
    CLE_ERR_TOO_LARGE = 7,  /* image exceeds the 2^31-2 voxel index range   */
    CLE_ERR_CANCELLED = 8   /* the caller's cancel word stopped a device loop */
} cle_status;

typedef struct cle_tensor {
    void *data;         /* device pointer                                   */
    int32_t ndim;       /* 1, 2 or 3                                        */
    int32_t dtype;      /* cle_dtype                                        */
    int64_t shape[3];   /* numpy order; unused trailing entries ignored     */
    int64_t strides[3]; /* element strides, must be C-contiguous            */
    int32_t device;     /* CUDA device ordinal                              */
} cle_tensor;

/* Per-call limits of the device loops (the Voronoi growth of the composite
 * ops runs until a step changes nothing; the reference's host loops,
 * _tier5/_masked_voronoi_labeling.py:62-69, have no bound).  Passed by the
 * entry points that run such a loop; NULL means every field at its default.
 * A loop that reaches a limit stops, and the call's status word (see
 * cle_workspace_status) reads CLE_ERR_ITER_LIMIT.  Nothing here is stored
 * between calls: two calls with different options may run at once. */
typedef struct cle_call_options {
    uint32_t struct_bytes;          /* sizeof(cle_call_options); 0 = this version's size */
    uint32_t max_loop_steps;        /* 0 = voxels + 16 (every step that does not stop
                                       the loop labels at least one voxel) */
    uint32_t loop_time_limit_ms;    /* 0 = 20000: wall-clock bound of one loop launch */
    uint32_t barrier_time_limit_ms; /* 0 = 4000: bound of one grid-barrier wait */
    int32_t cooperative_ctas;       /* 0 = one CTA per SM; n > 0 caps the loop's grid at n
                                       CTAs (several pipelines sharing the GPU) */
    int32_t reserved;               /* must be 0 */
    const volatile int32_t *cancel; /* NULL, or a word in page-locked host memory
                                       (cudaHostAlloc / cudaHostRegister): the loop reads it
                                       once per step and stops with CLE_ERR_CANCELLED once
                                       it is nonzero (per-request cancellation) */
} cle_call_options;

/* Number of float32 columns of the statistics table (see
 * cle_statistics_of_labelled_pixels). */
#define CLE_STATS_NCOLS 35

/* ---- library ---------------------------------------------------------- */
int cle_abi_version(void);
const char *cle_version(void);
const char *cle_last_error_message(void);
/* Number of kernel launches this library has issued in this process. */
unsigned long long cle_kernel_launches(void);
/* Profiling (off by default; the setting belongs to the calling host thread
 * and covers the calls that thread makes).  flags bit 0: the composite ops record a CUDA
 * event at each stage boundary on their stream; bit 1: the Voronoi loop also
 * writes a per-step trace to a buffer allocated here (not in the compute
 * calls).  0 turns profiling off.
 * cle_profile_stage_ms() waits for the last recorded event and writes the
 * elapsed milliseconds between consecutive events (returns how many).
 * Events 0-7 (voronoi_otsu_labeling): blur(spot) | detect_maxima |
 * blur(outline) | min/max+histogram+Otsu | threshold+seeds | seed CCL |
 * Voronoi growth; events 8-12 (statistics): pass 1 | finalise 1 | pass 2 |
 * finalise 2.  Interval 7 (between the two ops) is host time. */
int cle_profile_enable(int flags);
int cle_profile_stage_ms(float *out, int max);
/* Per-step trace of the last device loop (Voronoi growth) while profiling is
 * enabled: 4 uint64 per step (ns since the loop started at the end of the
 * step's compute phase, frontier size, voxels changed, ns at the end of its
 * write / queueing phase), zero after the last step.  Synchronous; returns
 * the bytes copied.  Profiling allocates its own trace buffer (outside any
 * workspace; bit 1 of cle_profile_enable). */
int cle_profile_trace(void *host, size_t bytes);

/* ---- gaussian_blur -----------------------------------------------------
 * replaces _tier1/_gaussian_blur.py:6-58 (+ _tier1/_execute_separable_kernel.py:7-76,
 * _tier0/_sigma_to_kernel_size.py:1-4).  src: u8/u16/f32; dst: f32.
 * Kernel size per axis int(8*sigma)|1; sigma <= 0 leaves that axis as is;
 * sigma_z is ignored for 2D images.  An isotropic blur of a volume stages
 * its planes with TMA copies; a copy wait that ran out (2 s) is reported by
 * cle_workspace_status on the same workspace as CLE_ERR_ITER_LIMIT. */
size_t cle_gaussian_blur_workspace_bytes(const cle_tensor *src);
int cle_gaussian_blur(const cle_tensor *src, const cle_tensor *dst, double sigma_x,
                      double sigma_y, double sigma_z, void *workspace, size_t workspace_bytes,
                      void *stream);

/* ---- minimum_of_all_pixels / maximum_of_all_pixels ----------------------
 * replaces _tier2/_minimum_of_all_pixels.py:7-60 and
 * _tier2/_maximum_of_all_pixels.py:7-60.  Writes {min, max} as two float32
 * to the device pointer d_minmax.  src: u8/u16/u32/f32. */
size_t cle_minimum_maximum_workspace_bytes(const cle_tensor *src);
int cle_minimum_maximum(const cle_tensor *src, float *d_minmax, void *workspace,
                        size_t workspace_bytes, void *stream);

/* ---- histogram -----------------------------------------------------------
 * replaces _tier3/_histogram.py:26-130.  dst: f32[num_bins].  With
 * determine_min_max != 0 the range is computed on the device (no host
 * round trip); otherwise [minimum, maximum] is used. */
size_t cle_histogram_workspace_bytes(const cle_tensor *src, int num_bins);
int cle_histogram(const cle_tensor *src, const cle_tensor *dst, int num_bins, float minimum,
                  float maximum, int determine_min_max, void *workspace,
                  size_t workspace_bytes, void *stream);

/* ---- threshold_otsu ----------------------------------------------------
 * replaces _tier9/_threshold_otsu.py:11-54 (and the host Otsu of
 * scikit_image_threshold_otsu, :64-106, now on the device in float64).
 * dst: u8 or f32 (1/0).  d_threshold (may be NULL) receives the float64
 * threshold. */
size_t cle_threshold_otsu_workspace_bytes(const cle_tensor *src);
int cle_threshold_otsu(const cle_tensor *src, const cle_tensor *dst, double *d_threshold,
                       void *workspace, size_t workspace_bytes, void *stream);

/* threshold_otsu without a workspace.  No counterpart in the reference: it
 * is for callers that can pass in the input and output buffers but cannot
 * allocate device memory themselves (a host that owns a fixed device-memory
 * budget and allows no allocation in its processing loop, a plugin that only
 * passes on the buffers its host gives it).  Same result as
 * cle_threshold_otsu; the scratch is an array built into the library
 * (cle_threshold_otsu_noalloc_scratch_bytes(), about 4 MiB, held on every
 * GPU that loads the library until the process exits), which limits the
 * image to 4096 rows (y); larger images return CLE_ERR_TOO_LARGE.  Every
 * call looks up the array's device address on its device (no cached pointer
 * survives a device reset); the first call on each device is its set-up and
 * loads the library's code there -- make that call before any stream
 * capture.  All calls share the array: calls that overlap
 * on the GPU (different streams or threads) race and must be serialised by
 * the caller.  Allocates nothing. */
int cle_threshold_otsu_noalloc(const cle_tensor *src, const cle_tensor *dst, void *stream);
size_t cle_threshold_otsu_noalloc_scratch_bytes(void);

/* ---- element-wise ops --------------------------------------------------
 * greater_constant replaces _tier1/_greater_constant.py:6-40 (constant as float32);
 * binary_and       replaces _tier1/_binary_and.py:6-47;
 * mask             replaces _tier1/_mask.py:6-44 (f32 -> u32 saturating like
 *                  clij_convert_uint_sat, _tier0/preamble.cl:548-556). */
int cle_greater_constant(const cle_tensor *src, const cle_tensor *dst, float constant,
                         void *stream);
int cle_binary_and(const cle_tensor *a, const cle_tensor *b, const cle_tensor *dst, void *stream);
int cle_mask(const cle_tensor *src, const cle_tensor *mask, const cle_tensor *dst, void *stream);

/* erode_box replaces _tier1/_erode_box.py:6-47 (erode_box_{2,3}d_x.cl): 1 where the
 * voxel and all of its 3x3(x3) box neighbours are nonzero, reads clamped to the
 * edge; source u8/u16/u32/i32/f32, destination u8/u16/u32/f32. */
int cle_erode_box(const cle_tensor *src, const cle_tensor *dst, void *stream);

/* ---- add_image_and_scalar / replace_intensities -------------------------
 * add_image_and_scalar replaces _tier1/_add_image_and_scalar.py (dst = src +
 * scalar in float32, saturating conversion to an integer destination);
 * replace_intensities replaces _tier1/_replace_intensities.py (dst = map[(int) src]
 * with the index clamped to the map, which is read along x of its first row,
 * float32).  Together with the statistics they make the label_*_map
 * functions of _tier9. */
int cle_add_image_and_scalar(const cle_tensor *src, const cle_tensor *dst, float scalar, void *stream);
int cle_replace_intensities(const cle_tensor *src, const cle_tensor *map, const cle_tensor *dst,
                            void *stream);

/* ---- euclidean_distance_from_label_centroid_map ---------------------------
 * replaces _tier9/_euclidean_distance_from_label_centroid_map.py: every
 * labelled voxel gets its float32 distance to its label's point in
 * `centroids` (a float32 [d, n] point list, one row per dimension x, y(, z),
 * column = label, as centroids_of_background_and_labels makes it); background
 * voxels get 0.  Any label / destination dtype of the path. */
int cle_euclidean_distance_from_label_centroid_map(const cle_tensor *labels, const cle_tensor *centroids,
                                                   const cle_tensor *dst, void *stream);

/* ---- distance / touch matrices and neighbour distances ------------------
 * Point lists are float32 [d, n] (one row per dimension x, y(, z), as
 * centroids_of_labels makes them).  Matrices are float32 [rows, columns] with
 * row y = item y - 1 of the second list (or label y), column x = item x - 1 of
 * the first (or label x), row and column 0 the background (zeros).
 * cle_generate_distance_matrix replaces _tier1/_generate_distance_matrix.py
 * (dst [m+1, n+1]: float32 Euclidean distances, squared differences summed x,
 * y, z in order).  cle_generate_touch_matrix replaces
 * _tier1/_generate_touch_matrix.py with generate_touch_matrix_{2,3}d_x.cl (dst
 * [L+1, L+1], cleared, then 1 at (a, b) and (b, a) for labels a != b meeting
 * across a face).  cle_average_distance_of_n_distances replaces
 * _tier1/_average_distance_of_n_nearest_distances.py (exclude_self 0, with
 * average_distance_of_n_nearest_distances_x.cl) and
 * _tier1/_average_distance_of_n_shortest_distances.py (exclude_self 1: row ==
 * column left out): per column the mean of the n smallest of rows 1.. (0 <= n
 * <= 1000; NaN when no row counts).  cle_average_distance_of_touching_neighbors
 * replaces _tier1/_average_distance_of_touching_neighbors.py: per column the
 * mean distance over rows >= 1 whose touch entry is set (0 if none).
 * cle_average_distance_of_n_nearest_points gives the n-distances vector of the
 * distance matrix of two point lists without building it, and
 * cle_average_distance_of_touching_labels the touching-neighbour vector of a
 * label image and its centroids (workspace: a bitmap of touching label pairs,
 * (L+1) x ceil((L+1)/32) words); these serve
 * _tier9/_average_distance_of_n_nearest_neighbors_map.py,
 * _tier9/_average_distance_to_n_nearest_other_labels_map.py and
 * _tier9/_average_neighbor_distance_map.py with replace_intensities. */
int cle_generate_distance_matrix(const cle_tensor *list1, const cle_tensor *list2, const cle_tensor *dst,
                                 void *stream);
int cle_generate_touch_matrix(const cle_tensor *labels, const cle_tensor *dst, void *stream);
int cle_average_distance_of_n_distances(const cle_tensor *distance_matrix, int n, int exclude_self,
                                        const cle_tensor *dst, void *stream);
int cle_average_distance_of_touching_neighbors(const cle_tensor *distance_matrix, const cle_tensor *touch_matrix,
                                               const cle_tensor *dst, void *stream);
int cle_average_distance_of_n_nearest_points(const cle_tensor *list1, const cle_tensor *list2, int n,
                                             int exclude_self, const cle_tensor *dst, void *stream);
size_t cle_average_distance_of_touching_labels_workspace_bytes(int64_t num_labels);
int cle_average_distance_of_touching_labels(const cle_tensor *labels, const cle_tensor *centroids,
                                            const cle_tensor *dst, void *workspace, size_t workspace_bytes,
                                            void *stream);

/* ---- minimum_box / maximum_box / top_hat_box ----------------------------
 * minimum_box replaces _tier1/_minimum_box.py:6-55, maximum_box
 * _tier1/_maximum_box.py, top_hat_box _tier2/_top_hat_box.py:6-43 (source minus
 * maximum_box(minimum_box(source)), in float32).  Separable passes over clamped
 * windows of int(2 * radius + 1) voxels; radius <= 0 leaves an axis alone;
 * radii above 700 are rejected.  src: u8/u16/f32; dst: f32.  One workspace
 * size (cle_box_filter_workspace_bytes) serves all three. */
size_t cle_box_filter_workspace_bytes(const cle_tensor *src);
int cle_minimum_box(const cle_tensor *src, const cle_tensor *dst, double radius_x, double radius_y,
                    double radius_z, void *workspace, size_t workspace_bytes, void *stream);
int cle_maximum_box(const cle_tensor *src, const cle_tensor *dst, double radius_x, double radius_y,
                    double radius_z, void *workspace, size_t workspace_bytes, void *stream);
int cle_top_hat_box(const cle_tensor *src, const cle_tensor *dst, double radius_x, double radius_y,
                    double radius_z, void *workspace, size_t workspace_bytes, void *stream);

/* ---- detect_maxima_box ---------------------------------------------------
 * replaces _tier1/_detect_maxima_box.py:5-48 with kernels
 * _tier1/detect_maxima_3d_x.cl:1-49, _tier1/detect_maxima_2d_x.cl:1-35.
 * Radii > 0 apply mean_box first (as the reference does); dst: u8 or f32. */
size_t cle_detect_maxima_box_workspace_bytes(const cle_tensor *src, int rx, int ry, int rz);
int cle_detect_maxima_box(const cle_tensor *src, const cle_tensor *dst, int rx, int ry, int rz,
                          void *workspace, size_t workspace_bytes, void *stream);

/* ---- connected_components_labeling_box ---------------------------------
 * replaces _tier4/_connected_components_labeling_box.py:15-66 (+ relabel,
 * _tier3/_relabel_sequential.py:12-58).  binary: u8/u32/f32 (nonzero =
 * foreground); dst: u32 or f32.  Labels are the ranks of each component's
 * float32 pixel-index key (x-major), as in the reference. */
size_t cle_connected_components_labeling_box_workspace_bytes(const cle_tensor *binary);
int cle_connected_components_labeling_box(const cle_tensor *binary, const cle_tensor *dst,
                                          void *workspace, size_t workspace_bytes,
                                          void *stream);

/* ---- connected_components_labeling_diamond -----------------------------
 * replaces _tier5/_connected_components_labeling_diamond.py:6-40: the same as
 * the box form with face connectivity (4 neighbours in 2D, 6 in 3D).  Same
 * workspace size as the box form. */
size_t cle_connected_components_labeling_diamond_workspace_bytes(const cle_tensor *binary);
int cle_connected_components_labeling_diamond(const cle_tensor *binary, const cle_tensor *dst,
                                              void *workspace, size_t workspace_bytes,
                                              void *stream);

/* ---- relabel_sequential --------------------------------------------------
 * replaces _tier3/_relabel_sequential.py:12-58.  src: u32 or f32 labels;
 * dst: u32 or f32.  max_label is the maximum of src (the reference also
 * reads it first, :42). */
size_t cle_relabel_sequential_workspace_bytes(const cle_tensor *src, uint32_t max_label);
int cle_relabel_sequential(const cle_tensor *src, const cle_tensor *dst, uint32_t max_label,
                           void *workspace, size_t workspace_bytes, void *stream);

/* ---- masked_voronoi_labeling -------------------------------------------
 * replaces _tier5/_masked_voronoi_labeling.py:7-76.  binary: seeds (u8/u32/f32,
 * nonzero); mask: u8/f32; dst: u32 or f32.  General form: any mask values,
 * seeds anywhere (dense Jacobi on the device, exact reference semantics). */
size_t cle_masked_voronoi_labeling_workspace_bytes(const cle_tensor *binary);
int cle_masked_voronoi_labeling(const cle_tensor *binary, const cle_tensor *mask,
                                const cle_tensor *dst, const cle_call_options *options,
                                void *workspace, size_t workspace_bytes, void *stream);

/* Fast form of masked_voronoi_labeling for the case voronoi_otsu_labeling
 * produces: mask values in {0, 1} and every seed inside the mask (then the
 * reference's -1/0/label state reduces to labels in the mask).  Growth visits
 * only the active part of the front (row bricks).  For other masks or seeds
 * outside the mask use cle_masked_voronoi_labeling.  The status word of the
 * workspace (cle_workspace_status) reports the loop outcome. */
size_t cle_masked_voronoi_labeling_binary_workspace_bytes(const cle_tensor *binary);
int cle_masked_voronoi_labeling_binary(const cle_tensor *binary, const cle_tensor *mask,
                                       const cle_tensor *dst, const cle_call_options *options,
                                       void *workspace, size_t workspace_bytes, void *stream);

/* ---- extend_labeling_via_voronoi / voronoi_labeling -------------------
 * extend_labeling_via_voronoi replaces _tier4/_extend_labeling_via_voronoi.py:13-60:
 * labels (u8/u16/u32/i32/f32, converted to uint32 like the reference's copy)
 * grow into every zero voxel, box and diamond steps alternating, until a
 * step changes nothing.  voronoi_labeling replaces _tier5/_voronoi_labeling.py:8-40
 * (connected_components_labeling_box, then that growth).  dst: u32 or f32.
 * The status word of the workspace (cle_workspace_status) reports the loop
 * outcome. */
size_t cle_extend_labeling_via_voronoi_workspace_bytes(const cle_tensor *src);
int cle_extend_labeling_via_voronoi(const cle_tensor *src, const cle_tensor *dst,
                                    const cle_call_options *options, void *workspace,
                                    size_t workspace_bytes, void *stream);
size_t cle_voronoi_labeling_workspace_bytes(const cle_tensor *binary);
int cle_voronoi_labeling(const cle_tensor *binary, const cle_tensor *dst,
                         const cle_call_options *options, void *workspace,
                         size_t workspace_bytes, void *stream);

/* ---- voronoi_otsu_labeling ---------------------------------------------
 * replaces _tier9/_voronoi_otsu_labeling.py:11-73.  src: u8/u16/f32 (u8 and
 * u16 are converted on the fly, exactly as push's float32 cast would);
 * dst: u32 (or f32).  No host synchronisation inside. */
size_t cle_voronoi_otsu_labeling_workspace_bytes(const cle_tensor *src);
int cle_voronoi_otsu_labeling(const cle_tensor *src, const cle_tensor *dst, double spot_sigma,
                              double outline_sigma, const cle_call_options *options,
                              void *workspace, size_t workspace_bytes, void *stream);

/* ---- batched voronoi_otsu_labeling --------------------------------------
 * The reference has no batched form: it runs every tile as the host-driven
 * sequence of _tier9/_voronoi_otsu_labeling.py:57-71.  A plan fixes a set of
 * tiles (shapes and dtypes u8/u16/f32, one device), the two sigmas and the
 * loop options; cle_vol_batch_launch then runs voronoi_otsu_labeling on every
 * tile (labels: uint32 or float32, the tile's shape), spread over the plan's
 * lanes -- CUDA streams forked from `stream` and joined back into it, so the
 * batch is stream-ordered on `stream` and the caller may capture it into a
 * CUDA graph.  lanes = 0 takes the lane count from the library's tuned table
 * (by mean tile size); with several lanes each lane's growth loop uses its
 * share of the SMs unless options set cooperative_ctas.  The plan owns host
 * objects (streams, events), not device memory: the one workspace
 * (cle_vol_batch_workspace_bytes) and the device status word (int32, receives
 * the maximum of every tile's loop status; 0 = all finished) come from the
 * caller.  A plan launches on one stream at a time. */
typedef struct cle_vol_batch cle_vol_batch;   /* opaque plan */
int cle_vol_batch_plan(const cle_tensor *tiles, int n_tiles, double spot_sigma, double outline_sigma,
                       int lanes, const cle_call_options *options, cle_vol_batch **plan);
size_t cle_vol_batch_workspace_bytes(const cle_vol_batch *plan);
int cle_vol_batch_lanes(const cle_vol_batch *plan);
int cle_vol_batch_launch(const cle_vol_batch *plan, const cle_tensor *tiles, const cle_tensor *labels,
                         void *workspace, size_t workspace_bytes, int32_t *d_status, void *stream);
void cle_vol_batch_free(cle_vol_batch *plan);

/* Device pointer to the label count (= maximum label) written by the last
 * voronoi_otsu_labeling / masked_voronoi_labeling_binary call that used this
 * workspace; for stream-ordered consumers such as
 * cle_statistics_of_labelled_pixels_device_count. */
const uint32_t *cle_workspace_label_count(const void *workspace);

/* Device status word of the last voronoi_otsu_labeling / masked Voronoi
 * call that used this workspace: 0 = finished, else a cle_status.  Reads
 * 4 bytes (synchronises the stream). */
int cle_workspace_status(const void *workspace, size_t workspace_bytes, void *stream);

/* ---- maximum label -------------------------------------------------------
 * Maximum value of a label image (u32 or f32 read as (int)), written as one
 * uint32 to d_max (device).  Used to size the statistics table
 * (_tier9/_statistics_of_labelled_pixels.py:56). */
size_t cle_label_maximum_workspace_bytes(const cle_tensor *labels);
int cle_label_maximum(const cle_tensor *labels, uint32_t *d_max, void *workspace,
                      size_t workspace_bytes, void *stream);

/* ---- statistics_of_labelled_pixels -------------------------------------
 * replaces _tier9/_statistics_of_labelled_pixels.py:7-293 (kernels
 * _tier9/statistics_per_label_x.cl, _tier9/standard_deviation_per_label_x.cl).
 * Writes a float32 table of CLE_STATS_NCOLS rows x num_labels columns
 * (row-major) to d_table, rows in the reference's dict order after 'label'
 * and 'original_label':
 *   bbox_min_x/y/z, bbox_max_x/y/z, bbox_width/height/depth, min_intensity,
 *   max_intensity, sum_intensity, area, mean_intensity,
 *   sum_intensity_times_x, mass_center_x, (y), (z), sum_x, centroid_x, (y),
 *   (z), sum_distance_to_centroid, mean_distance_to_centroid,
 *   sum_distance_to_mass_center, mean_distance_to_mass_center,
 *   standard_deviation_intensity, max_distance_to_centroid,
 *   max_distance_to_mass_center, mean_max_distance_to_centroid_ratio,
 *   mean_max_distance_to_mass_center_ratio.
 * Labels 1..num_labels; values above num_labels are ignored. */
size_t cle_statistics_workspace_bytes(const cle_tensor *labels, int64_t num_labels);
int cle_statistics_of_labelled_pixels(const cle_tensor *intensity, const cle_tensor *labels,
                                      int64_t num_labels, float *d_table, void *workspace,
                                      size_t workspace_bytes, void *stream);

/* Statistics with the label count in device memory (no host round trip):
 * d_num_labels points to the number of labels (e.g. from
 * cle_workspace_label_count); the table has `capacity` columns (row stride
 * capacity) and only the first min(count, capacity) are meaningful; labels
 * above capacity are ignored.  Workspace: cle_statistics_workspace_bytes(labels,
 * capacity).  Same results as cle_statistics_of_labelled_pixels. */
int cle_statistics_of_labelled_pixels_device_count(const cle_tensor *intensity,
                                                   const cle_tensor *labels,
                                                   const uint32_t *d_num_labels, int64_t capacity,
                                                   float *d_table, void *workspace,
                                                   size_t workspace_bytes, void *stream);

/* ---- centroids of labels -------------------------------------------------
 * replaces the centroid rows of _tier9/_statistics_of_labelled_pixels.py as
 * used by _tier9/_centroids_of_labels.py: for labels 1..num_labels of a u32 /
 * f32 label image, writes the float32 point list d_points[dim][num_labels]
 * (dim = x, y (, z)): float32(exact coordinate sum) / float32(voxel count),
 * the same values as the statistics table's centroid rows (NaN for a label
 * with no voxel).  One pass over the labels; labels above num_labels and 0
 * are ignored. */
size_t cle_label_centroids_workspace_bytes(const cle_tensor *labels, int64_t num_labels);
int cle_label_centroids(const cle_tensor *labels, int64_t num_labels, float *d_points,
                        void *workspace, size_t workspace_bytes, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CLE_B200_H */
