// neighbors.cu -- distance and touch matrices between labels and the
// neighbour-distance label maps:
//   generate_distance_matrix          _tier1/_generate_distance_matrix.py
//   generate_touch_matrix             _tier1/_generate_touch_matrix.py,
//                                     _tier1/generate_touch_matrix_{2,3}d_x.cl
//   average_distance_of_n_nearest_distances / _n_shortest_distances
//                                     _tier1/_average_distance_of_n_nearest_distances.py,
//                                     _tier1/average_distance_of_n_nearest_distances_x.cl,
//                                     _tier1/_average_distance_of_n_shortest_distances.py
//   average_distance_of_touching_neighbors
//                                     _tier1/_average_distance_of_touching_neighbors.py
//   and, for the maps of _tier9 (_average_distance_of_n_nearest_neighbors_map.py,
//   _average_neighbor_distance_map.py, _average_distance_to_n_nearest_other_labels_map.py),
//   the same value vectors straight from the centroid point lists, without the
//   (n+1) x (m+1) matrices: the n-nearest mean per point from a scan of the
//   other list, and the touching-neighbour mean from a bitmap of touching
//   label pairs.
//
// Matrices follow the reference's layout: float32, row y = point (or label)
// y - 1 of the second list, column x = point x - 1 of the first, row and
// column 0 (the background) zero.  Value vectors are [1, columns].
#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

// float32 distance between point i of list a ([d, na]) and point j of list b:
// squared differences summed in the order x, y(, z), every operation rounded
// to float32 (no contraction), then the correctly rounded square root.
__device__ __forceinline__ float point_distance(const float *a, int64_t na, int64_t i, const float *b, int64_t nb,
                                                int64_t j, int d) {
    float s = 0.0f;
    for (int k = 0; k < d; ++k) {
        const float t = __fsub_rn(a[k * na + i], b[k * nb + j]);
        s = __fadd_rn(s, __fmul_rn(t, t));
    }
    return __fsqrt_rn(s);
}

__global__ void distance_matrix_kernel(const float *__restrict__ a, int64_t na, const float *__restrict__ b,
                                       int64_t nb, int d, float *__restrict__ dst) {
    const int64_t W = na + 1, total = (nb + 1) * W;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t y = e / W, x = e - y * W;
        dst[e] = (x == 0 || y == 0) ? 0.0f : point_distance(a, na, x - 1, b, nb, y - 1, d);
    }
}

// label value as the reference reads it: the float value, truncated
template <typename T>
__device__ __forceinline__ int64_t label_index(T v) { return (int64_t)(float)v; }

// Touch matrix: a voxel and its +x, +y (, +z) neighbour with different labels
// mark both (a, b) and (b, a); the last voxel of a row compares with itself
// (clamp to edge).  Labels outside 0 .. L are skipped.
template <typename T>
__global__ void touch_matrix_kernel(const T *__restrict__ lab, int64_t D, int64_t H, int64_t W, int64_t L,
                                    float *__restrict__ dst) {
    const int64_t n = D * H * W, M = L + 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = i % W, zy = i / W, y = zy % H, z = zy / H;
        const int64_t a = label_index(lab[i]);
        int64_t nbr[3];
        nbr[0] = x + 1 < W ? label_index(lab[i + 1]) : a;
        nbr[1] = y + 1 < H ? label_index(lab[i + W]) : a;
        nbr[2] = z + 1 < D ? label_index(lab[i + H * W]) : a;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int64_t b = nbr[k];
            if (b != a && a >= 0 && b >= 0 && a <= L && b <= L) {
                dst[b * M + a] = 1.0f;
                dst[a * M + b] = 1.0f;
            }
        }
    }
}

// The n smallest values of a stream, kept the way
// average_distance_of_n_nearest_distances_x.cl keeps them: while fewer than n
// are held the value is appended, then one insertion pass from the end moves
// a smaller value down (a value equal to a held one, or NaN, stays where it
// is).  buf holds n values at a stride (one column of a shared-memory block).
__device__ __forceinline__ void keep_smallest(float *buf, int stride, int &filled, int n, float v) {
    if (filled < n) {
        ++filled;
        buf[(filled - 1) * stride] = v;
    }
    for (int i = filled - 1; i >= 0; --i) {
        const float bi = buf[i * stride];
        if (v > bi) break;
        if (v < bi && (i == 0 || v >= buf[(i - 1) * stride])) {
            for (int j = filled - 1; j > i; --j) buf[j * stride] = buf[(j - 1) * stride];
            buf[i * stride] = v;
            break;
        }
    }
}

// the mean of the held values: a float32 sum in buffer order over the count
// (0 / 0 = NaN when nothing is held, as in the reference)
__device__ __forceinline__ float held_mean(const float *buf, int stride, int filled) {
    float s = 0.0f;
    for (int i = 0; i < filled; ++i) s = __fadd_rn(s, buf[i * stride]);
    return __fdiv_rn(s, (float)filled);
}

// Per column x of a [H, W] distance matrix: the mean of the n smallest of
// rows 1 .. H-1 (row x left out when exclude_self).  One thread per column,
// its buffer a column of the block's shared memory.
__global__ void n_distances_matrix_kernel(const float *__restrict__ dm, int64_t H, int64_t W, int n,
                                          int exclude_self, float *__restrict__ out) {
    extern __shared__ float s_buf[];
    const int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (x >= W) return;
    float *buf = s_buf + threadIdx.x;
    int filled = 0;
    for (int64_t y = 1; y < H; ++y) {
        if (exclude_self && y == x) continue;
        keep_smallest(buf, blockDim.x, filled, n, dm[y * W + x]);
    }
    out[x] = held_mean(buf, blockDim.x, filled);
}

// The same vector straight from the two point lists (the matrix's entries
// computed on the fly; column 0 and row 0 are the background's zeros).
// Points of list b are staged through shared memory in tiles.
constexpr int kPtsTile = 256;
__global__ void n_distances_points_kernel(const float *__restrict__ a, int64_t na, const float *__restrict__ b,
                                          int64_t nb, int d, int n, int exclude_self, float *__restrict__ out) {
    extern __shared__ float s_buf[];
    float *s_pts = s_buf;                              // [d][kPtsTile]
    float *buf = s_buf + 3 * kPtsTile + threadIdx.x;   // column of the n-value buffers
    const int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;   // column: 0 background, i + 1 point i
    const bool live = x <= na;
    float ax[3] = {0.f, 0.f, 0.f};
    if (live && x > 0)
        for (int k = 0; k < d; ++k) ax[k] = a[k * na + (x - 1)];
    int filled = 0;
    for (int64_t t0 = 0; t0 < nb; t0 += kPtsTile) {
        const int cnt = (int)(nb - t0 < (int64_t)kPtsTile ? nb - t0 : (int64_t)kPtsTile);
        __syncthreads();
        for (int e = threadIdx.x; e < d * kPtsTile; e += blockDim.x) {
            const int k = e / kPtsTile, j = e - k * kPtsTile;
            if (j < cnt) s_pts[k * kPtsTile + j] = b[k * nb + t0 + j];
        }
        __syncthreads();
        if (!live) continue;
        for (int j = 0; j < cnt; ++j) {
            const int64_t y = t0 + j + 1;
            if (exclude_self && y == x) continue;
            float v = 0.0f;
            if (x > 0) {
                float s = 0.0f;
                for (int k = 0; k < d; ++k) {
                    const float t = __fsub_rn(ax[k], s_pts[k * kPtsTile + j]);
                    s = __fadd_rn(s, __fmul_rn(t, t));
                }
                v = __fsqrt_rn(s);
            }
            keep_smallest(buf, blockDim.x, filled, n, v);
        }
    }
    if (live) out[x] = held_mean(buf, blockDim.x, filled);
}

// Per column x: the mean of the distances in rows y >= 1 whose touch entry is
// set (0 when no label touches), the sum in row order.
__global__ void touching_matrix_kernel(const float *__restrict__ dm, const float *__restrict__ tm, int64_t H,
                                       int64_t W, int64_t TW, float *__restrict__ out) {
    const int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (x >= W) return;
    float s = 0.0f;
    int64_t c = 0;
    for (int64_t y = 1; y < H; ++y)
        if (tm[y * TW + x] > 0.0f) {
            s = __fadd_rn(s, dm[y * W + x]);
            ++c;
        }
    out[x] = c > 0 ? __fdiv_rn(s, (float)c) : 0.0f;
}

// Touching label pairs as a bitmap: row a holds bit b when labels a and b
// (both 1 .. L) touch across a face, as generate_touch_matrix defines it.
template <typename T>
__global__ void touch_bits_kernel(const T *__restrict__ lab, int64_t D, int64_t H, int64_t W, int64_t L,
                                  int64_t words, uint32_t *__restrict__ bits) {
    const int64_t n = D * H * W;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = i % W, zy = i / W, y = zy % H, z = zy / H;
        const int64_t a = label_index(lab[i]);
        if (a < 1 || a > L) continue;
        int64_t nbr[3];
        nbr[0] = x + 1 < W ? label_index(lab[i + 1]) : a;
        nbr[1] = y + 1 < H ? label_index(lab[i + W]) : a;
        nbr[2] = z + 1 < D ? label_index(lab[i + H * W]) : a;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int64_t b = nbr[k];
            if (b != a && b >= 1 && b <= L) {
                atomicOr(bits + a * words + (b >> 5), 1u << (b & 31));
                atomicOr(bits + b * words + (a >> 5), 1u << (a & 31));
            }
        }
    }
}

// Per label x (column x of the vector; 0 stays 0): the mean distance from
// point x - 1 to the points of the labels touching it, in label order.
__global__ void touching_points_kernel(const uint32_t *__restrict__ bits, int64_t words, const float *__restrict__ p,
                                       int64_t np, int d, int64_t L, float *__restrict__ out) {
    const int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (x > L) return;
    if (x == 0) { out[0] = 0.0f; return; }
    float s = 0.0f;
    int64_t c = 0;
    const uint32_t *row = bits + x * words;
    for (int64_t w = 0; w < words; ++w) {
        uint32_t v = row[w];
        while (v) {
            const int64_t y = w * 32 + (__ffs(v) - 1);
            v &= v - 1u;
            s = __fadd_rn(s, point_distance(p, np, x - 1, p, np, y - 1, d));
            ++c;
        }
    }
    out[x] = c > 0 ? __fdiv_rn(s, (float)c) : 0.0f;
}

int point_list(const Img &p, const char *name, int &d, int64_t &n) {
    if (p.dtype != CLE_F32 || p.D != 1 || p.H < 1 || p.H > 3) {
        set_error("%s: a float32 [d, n] point list with d = 1..3 is required", name);
        return CLE_ERR_ARG;
    }
    d = (int)p.H;
    n = p.W;
    return CLE_OK;
}

int vector_out(const Img &v, int64_t len, const char *name) {
    if (v.dtype != CLE_F32 || v.D != 1 || v.H != 1 || v.W < len) {
        set_error("%s: a float32 [1, >= %lld] vector is required", name, (long long)len);
        return CLE_ERR_ARG;
    }
    return CLE_OK;
}

// threads per block of the n-value buffers (one shared-memory column each)
int buffer_threads(int n, size_t extra, size_t &smem) {
    int t = 128;
    while (t > 32 && (size_t)t * n * sizeof(float) + extra > 200 * 1024) t >>= 1;
    smem = (size_t)t * n * sizeof(float) + extra;
    return t;
}

constexpr int kMaxN = 1000;   // the reference kernel's buffer (float distances[1000])

}  // namespace

int generate_distance_matrix(const Img &a, const Img &b, const Img &dst, cudaStream_t st) {
    int da = 0, db = 0;
    int64_t na = 0, nb = 0;
    CLE_TRY(point_list(a, "generate_distance_matrix: coordinate_list1", da, na));
    CLE_TRY(point_list(b, "generate_distance_matrix: coordinate_list2", db, nb));
    if (da != db) { set_error("generate_distance_matrix: point lists of different dimensionality"); return CLE_ERR_ARG; }
    if (dst.dtype != CLE_F32 || dst.D != 1 || dst.H != nb + 1 || dst.W != na + 1) {
        set_error("generate_distance_matrix: destination must be float32 [%lld, %lld]", (long long)(nb + 1),
                  (long long)(na + 1));
        return CLE_ERR_ARG;
    }
    const int64_t total = (nb + 1) * (na + 1);
    distance_matrix_kernel<<<launch_blocks(total, 256), 256, 0, st>>>((const float *)a.data, na, (const float *)b.data,
                                                                       nb, da, (float *)dst.data);
    CLE_LAUNCH_CHECK("distance matrix");
    return CLE_OK;
}

int generate_touch_matrix(const Img &lab, const Img &dst, cudaStream_t st) {
    if (dst.dtype != CLE_F32 || dst.D != 1 || dst.H != dst.W || dst.W < 1) {
        set_error("generate_touch_matrix: destination must be a square float32 matrix");
        return CLE_ERR_ARG;
    }
    const int64_t L = dst.W - 1;
    CLE_CUDA(cudaMemsetAsync(dst.data, 0, sizeof(float) * (size_t)(dst.W * dst.H), st));
    const int b = launch_blocks(lab.n(), 256);
    switch (lab.dtype) {
        case CLE_U8: touch_matrix_kernel<uint8_t><<<b, 256, 0, st>>>((const uint8_t *)lab.data, lab.D, lab.H, lab.W, L, (float *)dst.data); break;
        case CLE_U16: touch_matrix_kernel<uint16_t><<<b, 256, 0, st>>>((const uint16_t *)lab.data, lab.D, lab.H, lab.W, L, (float *)dst.data); break;
        case CLE_U32: touch_matrix_kernel<uint32_t><<<b, 256, 0, st>>>((const uint32_t *)lab.data, lab.D, lab.H, lab.W, L, (float *)dst.data); break;
        case CLE_I32: touch_matrix_kernel<int32_t><<<b, 256, 0, st>>>((const int32_t *)lab.data, lab.D, lab.H, lab.W, L, (float *)dst.data); break;
        case CLE_F32: touch_matrix_kernel<float><<<b, 256, 0, st>>>((const float *)lab.data, lab.D, lab.H, lab.W, L, (float *)dst.data); break;
        default: set_error("generate_touch_matrix: unsupported label dtype %d", lab.dtype); return CLE_ERR_DTYPE;
    }
    CLE_LAUNCH_CHECK("touch matrix");
    return CLE_OK;
}

int average_distance_of_n_distances(const Img &dm, int n, int exclude_self, const Img &dst, cudaStream_t st) {
    if (dm.dtype != CLE_F32 || dm.D != 1) { set_error("average distance: a float32 distance matrix is required"); return CLE_ERR_ARG; }
    if (n < 0 || n > kMaxN) { set_error("average distance: n must lie in 0..%d (got %d)", kMaxN, n); return CLE_ERR_ARG; }
    CLE_TRY(vector_out(dst, dm.W, "average distance"));
    if (dm.W == 0) return CLE_OK;
    size_t smem = 0;
    const int t = buffer_threads(std::max(n, 1), 0, smem);
    CLE_CUDA(cudaFuncSetAttribute(n_distances_matrix_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    n_distances_matrix_kernel<<<(unsigned)((dm.W + t - 1) / t), t, smem, st>>>((const float *)dm.data, dm.H, dm.W, n,
                                                                              exclude_self, (float *)dst.data);
    CLE_LAUNCH_CHECK("n distances");
    return CLE_OK;
}

int average_distance_of_touching_neighbors(const Img &dm, const Img &tm, const Img &dst, cudaStream_t st) {
    if (dm.dtype != CLE_F32 || tm.dtype != CLE_F32 || dm.D != 1 || tm.D != 1 || tm.H < dm.H || tm.W < dm.W) {
        set_error("average_distance_of_touching_neighbors: float32 distance and touch matrices of one size are required");
        return CLE_ERR_ARG;
    }
    CLE_TRY(vector_out(dst, dm.W, "average_distance_of_touching_neighbors"));
    if (dm.W == 0) return CLE_OK;
    touching_matrix_kernel<<<(unsigned)((dm.W + 127) / 128), 128, 0, st>>>((const float *)dm.data, (const float *)tm.data,
                                                                          dm.H, dm.W, tm.W, (float *)dst.data);
    CLE_LAUNCH_CHECK("touching neighbours");
    return CLE_OK;
}

int average_distance_of_n_points(const Img &a, const Img &b, int n, int exclude_self, const Img &dst, cudaStream_t st) {
    int da = 0, db = 0;
    int64_t na = 0, nb = 0;
    CLE_TRY(point_list(a, "average distance: list 1", da, na));
    CLE_TRY(point_list(b, "average distance: list 2", db, nb));
    if (da != db) { set_error("average distance: point lists of different dimensionality"); return CLE_ERR_ARG; }
    if (n < 0 || n > kMaxN) { set_error("average distance: n must lie in 0..%d (got %d)", kMaxN, n); return CLE_ERR_ARG; }
    CLE_TRY(vector_out(dst, na + 1, "average distance"));
    size_t smem = 0;
    const int t = buffer_threads(std::max(n, 1), sizeof(float) * 3 * kPtsTile, smem);
    CLE_CUDA(cudaFuncSetAttribute(n_distances_points_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    n_distances_points_kernel<<<(unsigned)((na + 1 + t - 1) / t), t, smem, st>>>(
        (const float *)a.data, na, (const float *)b.data, nb, da, n, exclude_self, (float *)dst.data);
    CLE_LAUNCH_CHECK("n nearest points");
    return CLE_OK;
}

size_t touching_labels_workspace_bytes(int64_t num_labels) {
    if (num_labels < 0) return 0;
    const int64_t words = (num_labels + 1 + 31) / 32;
    Arena a(nullptr, 0);
    a.take<uint32_t>((size_t)(num_labels + 1) * (size_t)words);
    return a.off;
}

int average_distance_of_touching_labels(const Img &lab, const Img &p, const Img &dst, Arena &ws, cudaStream_t st) {
    int d = 0;
    int64_t L = 0;
    CLE_TRY(point_list(p, "average_neighbor_distance_map: centroids", d, L));
    CLE_TRY(vector_out(dst, L + 1, "average_neighbor_distance_map"));
    const int64_t words = (L + 1 + 31) / 32;
    uint32_t *bits = ws.take<uint32_t>((size_t)(L + 1) * (size_t)words);
    if (!ws.ok()) { set_error("average_neighbor_distance_map: workspace too small"); return CLE_ERR_WORKSPACE; }
    CLE_CUDA(cudaMemsetAsync(bits, 0, sizeof(uint32_t) * (size_t)(L + 1) * (size_t)words, st));
    const int b = launch_blocks(lab.n(), 256);
    switch (lab.dtype) {
        case CLE_U8: touch_bits_kernel<uint8_t><<<b, 256, 0, st>>>((const uint8_t *)lab.data, lab.D, lab.H, lab.W, L, words, bits); break;
        case CLE_U16: touch_bits_kernel<uint16_t><<<b, 256, 0, st>>>((const uint16_t *)lab.data, lab.D, lab.H, lab.W, L, words, bits); break;
        case CLE_U32: touch_bits_kernel<uint32_t><<<b, 256, 0, st>>>((const uint32_t *)lab.data, lab.D, lab.H, lab.W, L, words, bits); break;
        case CLE_I32: touch_bits_kernel<int32_t><<<b, 256, 0, st>>>((const int32_t *)lab.data, lab.D, lab.H, lab.W, L, words, bits); break;
        case CLE_F32: touch_bits_kernel<float><<<b, 256, 0, st>>>((const float *)lab.data, lab.D, lab.H, lab.W, L, words, bits); break;
        default: set_error("average_neighbor_distance_map: unsupported label dtype %d", lab.dtype); return CLE_ERR_DTYPE;
    }
    CLE_LAUNCH_CHECK("touching pairs");
    touching_points_kernel<<<(unsigned)((L + 1 + 127) / 128), 128, 0, st>>>(bits, words, (const float *)p.data, L, d, L,
                                                                           (float *)dst.data);
    CLE_LAUNCH_CHECK("touching means");
    return CLE_OK;
}

}  // namespace cle
