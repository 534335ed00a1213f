// maps.cu -- the element-wise ops behind the parametric label maps:
//   add_image_and_scalar  (_tier1/_add_image_and_scalar.py): dst = src + scalar
//                         in float32, converted to the destination type;
//   replace_intensities   (_tier1/_replace_intensities.py): dst = map[(int) src],
//                         the index clamped to the map like the reference's
//                         clamped image read.
// The label_*_map functions (_tier9/_label_*_map.py) combine them with the
// statistics table on the device: statistics of labels + 1 (so the background
// gets a column), one row of the table as the map, entry 0 set to 0.
//   euclidean_distance_from_label_centroid_map
//                         (_tier9/_euclidean_distance_from_label_centroid_map.py):
//                         each labelled voxel's float32 distance to its label's
//                         point in a [d, n] centroid list; background stays 0.
#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

template <typename Td>
__device__ __forceinline__ Td from_f32(float v) {
    if constexpr (std::is_same<Td, float>::value) {
        return v;
    } else {   // clij_convert_*_sat (unsigned Td): NaN and negatives to 0, saturate, truncate
        const Td top = (Td)~Td(0);
        return !(v > 0.0f) ? Td(0) : (v >= (float)top ? top : (Td)v);
    }
}

template <typename Ts, typename Td>
__global__ void add_scalar_kernel(const Ts *__restrict__ src, Td *__restrict__ dst, float c, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = from_f32<Td>(__fadd_rn((float)src[i], c));
}

template <typename Ts, typename Td>
__global__ void replace_kernel(const Ts *__restrict__ src, const float *__restrict__ map, int64_t m,
                               Td *__restrict__ dst, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = (float)src[i];
        int64_t k = (v != v) ? 0 : (int64_t)fmaxf(fminf(v, 2147483647.0f), -2147483648.0f);   // (int) read
        k = k < 0 ? 0 : (k >= m ? m - 1 : k);
        dst[i] = from_f32<Td>(map[k]);
    }
}

// pts: row r (x, y, z) of the point list at pts[r * m + label]; label index
// read like replace_kernel's (clamped to the list)
// (x, y, z) of voxel i: 32-bit multiply-shift divisions while the image has
// under 2^32 voxels, 64-bit division otherwise
template <typename Ts, typename Td>
__global__ void centroid_distance_kernel(const Ts *__restrict__ src, const float *__restrict__ pts, int64_t m,
                                         int dims, int64_t W, int64_t H, FastDiv fW, FastDiv fH,
                                         Td *__restrict__ dst, int64_t n) {
    const bool small = n <= 0xFFFFFFFFll;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = (float)src[i];
        int64_t k = (v != v) ? 0 : (int64_t)fmaxf(fminf(v, 2147483647.0f), -2147483648.0f);
        float d = 0.0f;
        if (k != 0) {
            k = k < 0 ? 0 : (k >= m ? m - 1 : k);
            int64_t x, y, z;
            if (small) {
                const uint32_t r = fW.div((uint32_t)i), q = fH.div(r);
                x = (uint32_t)i - r * fW.d;
                y = r - q * fH.d;
                z = q;
            } else {
                const int64_t r = i / W;
                x = i % W;
                y = r % H;
                z = r / H;
            }
            const float dx = __fsub_rn((float)x, pts[k]);
            const float dy = __fsub_rn((float)y, pts[m + k]);
            float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
            if (dims > 2) {
                const float dz = __fsub_rn((float)z, pts[2 * m + k]);
                d2 = __fadd_rn(d2, __fmul_rn(dz, dz));
            }
            d = __fsqrt_rn(d2);
        }
        dst[i] = from_f32<Td>(d);
    }
}

template <typename Ts>
int centroid_distance_dst(const Img &s, const float *pts, int64_t m, int dims, const Img &d, cudaStream_t st) {
    const int64_t n = s.n();
    const int b = launch_blocks(n, 256);
    const FastDiv fW((uint32_t)std::min<int64_t>(s.W, 0xFFFFFFFFll)), fH((uint32_t)std::min<int64_t>(s.H, 0xFFFFFFFFll));
    switch (d.dtype) {
        case CLE_F32: centroid_distance_kernel<Ts, float><<<b, 256, 0, st>>>((const Ts *)s.data, pts, m, dims, s.W, s.H, fW, fH, (float *)d.data, n); break;
        case CLE_U32: centroid_distance_kernel<Ts, uint32_t><<<b, 256, 0, st>>>((const Ts *)s.data, pts, m, dims, s.W, s.H, fW, fH, (uint32_t *)d.data, n); break;
        case CLE_U16: centroid_distance_kernel<Ts, uint16_t><<<b, 256, 0, st>>>((const Ts *)s.data, pts, m, dims, s.W, s.H, fW, fH, (uint16_t *)d.data, n); break;
        case CLE_U8: centroid_distance_kernel<Ts, uint8_t><<<b, 256, 0, st>>>((const Ts *)s.data, pts, m, dims, s.W, s.H, fW, fH, (uint8_t *)d.data, n); break;
        default: set_error("euclidean_distance_from_label_centroid_map: unsupported destination dtype %d", d.dtype); return CLE_ERR_DTYPE;
    }
    CLE_LAUNCH_CHECK("euclidean_distance_from_label_centroid_map");
    return CLE_OK;
}

template <typename Ts>
int add_scalar_dst(const Img &s, const Img &d, float c, cudaStream_t st) {
    const int64_t n = s.n();
    const int b = launch_blocks(n, 256);
    switch (d.dtype) {
        case CLE_F32: add_scalar_kernel<Ts, float><<<b, 256, 0, st>>>((const Ts *)s.data, (float *)d.data, c, n); break;
        case CLE_U32: add_scalar_kernel<Ts, uint32_t><<<b, 256, 0, st>>>((const Ts *)s.data, (uint32_t *)d.data, c, n); break;
        case CLE_U16: add_scalar_kernel<Ts, uint16_t><<<b, 256, 0, st>>>((const Ts *)s.data, (uint16_t *)d.data, c, n); break;
        case CLE_U8: add_scalar_kernel<Ts, uint8_t><<<b, 256, 0, st>>>((const Ts *)s.data, (uint8_t *)d.data, c, n); break;
        default: set_error("add_image_and_scalar: unsupported destination dtype %d", d.dtype); return CLE_ERR_DTYPE;
    }
    CLE_LAUNCH_CHECK("add_image_and_scalar");
    return CLE_OK;
}

template <typename Ts>
int replace_dst(const Img &s, const float *map, int64_t m, const Img &d, cudaStream_t st) {
    const int64_t n = s.n();
    const int b = launch_blocks(n, 256);
    switch (d.dtype) {
        case CLE_F32: replace_kernel<Ts, float><<<b, 256, 0, st>>>((const Ts *)s.data, map, m, (float *)d.data, n); break;
        case CLE_U32: replace_kernel<Ts, uint32_t><<<b, 256, 0, st>>>((const Ts *)s.data, map, m, (uint32_t *)d.data, n); break;
        case CLE_U16: replace_kernel<Ts, uint16_t><<<b, 256, 0, st>>>((const Ts *)s.data, map, m, (uint16_t *)d.data, n); break;
        case CLE_U8: replace_kernel<Ts, uint8_t><<<b, 256, 0, st>>>((const Ts *)s.data, map, m, (uint8_t *)d.data, n); break;
        default: set_error("replace_intensities: unsupported destination dtype %d", d.dtype); return CLE_ERR_DTYPE;
    }
    CLE_LAUNCH_CHECK("replace_intensities");
    return CLE_OK;
}

}  // namespace

int add_image_and_scalar(const Img &src, const Img &dst, float c, cudaStream_t st) {
    CLE_TRY(same_shape(src, dst, "source", "destination"));
    if (src.n() == 0) return CLE_OK;
    switch (src.dtype) {
        case CLE_F32: return add_scalar_dst<float>(src, dst, c, st);
        case CLE_U32: return add_scalar_dst<uint32_t>(src, dst, c, st);
        case CLE_U16: return add_scalar_dst<uint16_t>(src, dst, c, st);
        case CLE_U8: return add_scalar_dst<uint8_t>(src, dst, c, st);
        case CLE_I32: return add_scalar_dst<int32_t>(src, dst, c, st);
        default: set_error("add_image_and_scalar: unsupported source dtype %d", src.dtype); return CLE_ERR_DTYPE;
    }
}

int replace_intensities(const Img &src, const Img &map, const Img &dst, cudaStream_t st) {
    CLE_TRY(same_shape(src, dst, "source", "destination"));
    if (map.dtype != CLE_F32) { set_error("replace_intensities: the values vector must be float32"); return CLE_ERR_DTYPE; }
    if (map.n() < 1) { set_error("replace_intensities: empty values vector"); return CLE_ERR_SHAPE; }
    if (src.n() == 0) return CLE_OK;
    // the vector is read along x of its first row, like the reference's (index, 0) read
    const int64_t m = map.W;
    switch (src.dtype) {
        case CLE_F32: return replace_dst<float>(src, (const float *)map.data, m, dst, st);
        case CLE_U32: return replace_dst<uint32_t>(src, (const float *)map.data, m, dst, st);
        case CLE_U16: return replace_dst<uint16_t>(src, (const float *)map.data, m, dst, st);
        case CLE_U8: return replace_dst<uint8_t>(src, (const float *)map.data, m, dst, st);
        case CLE_I32: return replace_dst<int32_t>(src, (const float *)map.data, m, dst, st);
        default: set_error("replace_intensities: unsupported source dtype %d", src.dtype); return CLE_ERR_DTYPE;
    }
}

int centroid_distance_map(const Img &labels, const Img &pts, const Img &dst, cudaStream_t st) {
    CLE_TRY(same_shape(labels, dst, "labels", "distance_map_destination"));
    if (pts.dtype != CLE_F32) { set_error("euclidean_distance_from_label_centroid_map: the point list must be float32"); return CLE_ERR_DTYPE; }
    const int dims = labels.ndim == 3 ? 3 : 2;
    // the point list is a [dims, n] image: n points along x, one row per dimension
    if (pts.D != 1 || pts.H < dims || pts.W < 1) {
        set_error("euclidean_distance_from_label_centroid_map: the point list must be %d x n", dims);
        return CLE_ERR_SHAPE;
    }
    if (labels.n() == 0) return CLE_OK;
    const int64_t m = pts.W;
    switch (labels.dtype) {
        case CLE_F32: return centroid_distance_dst<float>(labels, (const float *)pts.data, m, dims, dst, st);
        case CLE_U32: return centroid_distance_dst<uint32_t>(labels, (const float *)pts.data, m, dims, dst, st);
        case CLE_U16: return centroid_distance_dst<uint16_t>(labels, (const float *)pts.data, m, dims, dst, st);
        case CLE_U8: return centroid_distance_dst<uint8_t>(labels, (const float *)pts.data, m, dims, dst, st);
        case CLE_I32: return centroid_distance_dst<int32_t>(labels, (const float *)pts.data, m, dims, dst, st);
        default: set_error("euclidean_distance_from_label_centroid_map: unsupported label dtype %d", labels.dtype); return CLE_ERR_DTYPE;
    }
}

}  // namespace cle
