// morph.cu -- erode_box (_tier1/_erode_box.py:6-47): binary erosion over the
// 3x3 (2D) or 3x3x3 (3D) box.  A voxel of the output is 1 when it and every
// neighbour in its box are nonzero in the source, else 0.  Reads clamp to the
// image edge like every buffer read of the reference; a clamped read lands on
// a voxel of the same box, so only in-range neighbours decide.
//
// One launch: a CTA covers 32 x 8 (x, y) columns and marches a chunk of z.
// Per plane a thread ANDs rows y-1, y, y+1 of its column, takes the x
// neighbours' column results by warp shuffles (the two edge lanes load their
// outer column), and keeps the last three plane results in registers, so each
// source voxel is read about once per plane pass and each output written once.
#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

constexpr int kEX = 32;   // x columns per CTA (one warp per y row)
constexpr int kEY = 8;    // y rows per CTA

template <typename T>
__device__ __forceinline__ uint32_t nonzero(T v) { return v != T(0) ? 1u : 0u; }

template <typename Ts, typename Td, bool Z>
__global__ void __launch_bounds__(kEX * kEY)
erode_box_kernel(const Ts *__restrict__ src, Td *__restrict__ dst, int D, int H, int W, int zchunk) {
    const int lane = threadIdx.x;
    const int x = blockIdx.x * kEX + lane;
    const int y = blockIdx.y * kEY + threadIdx.y;
    // columns and rows beyond the image repeat the last one (clamp); they
    // take part in the shuffles but store nothing
    const int xc = min(x, W - 1), yc = min(y, H - 1);
    const int ym = max(yc - 1, 0), yp = min(yc + 1, H - 1);
    const int xe = (lane == 0) ? max(xc - 1, 0) : min(xc + 1, W - 1);   // edge lanes' outer column
    const bool edge = lane == 0 || lane == kEX - 1;
    const int64_t plane = (int64_t)H * W;

    auto plane_and = [&](int z) -> uint32_t {
        const Ts *p = src + (int64_t)z * plane;
        const uint32_t c = nonzero(__ldg(p + (int64_t)ym * W + xc)) & nonzero(__ldg(p + (int64_t)yc * W + xc)) &
                           nonzero(__ldg(p + (int64_t)yp * W + xc));
        uint32_t e = 1u;
        if (edge)
            e = nonzero(__ldg(p + (int64_t)ym * W + xe)) & nonzero(__ldg(p + (int64_t)yc * W + xe)) &
                nonzero(__ldg(p + (int64_t)yp * W + xe));
        const uint32_t l = __shfl_up_sync(0xffffffffu, c, 1);
        const uint32_t r = __shfl_down_sync(0xffffffffu, c, 1);
        return c & (lane == 0 ? e : l) & (lane == kEX - 1 ? e : r);
    };

    const bool store = x < W && y < H;
    if constexpr (!Z) {
        const uint32_t o = plane_and(0);
        if (store) dst[(int64_t)y * W + x] = (Td)o;
    } else {
        const int z0 = (int)blockIdx.z * zchunk;
        const int z1 = min(D, z0 + zchunk);
        uint32_t prev = plane_and(max(z0 - 1, 0));
        uint32_t cur = plane_and(z0);
        for (int z = z0; z < z1; ++z) {
            const uint32_t next = plane_and(min(z + 1, D - 1));
            if (store) dst[(int64_t)z * plane + (int64_t)y * W + x] = (Td)(prev & cur & next);
            prev = cur;
            cur = next;
        }
    }
}

template <typename Ts, typename Td>
int launch_erode(const Img &src, const Img &dst, cudaStream_t st) {
    const int64_t gx = (src.W + kEX - 1) / kEX, gy = (src.H + kEY - 1) / kEY;
    if (gy > 65535) { set_error("erode_box: image too large"); return CLE_ERR_TOO_LARGE; }
    const bool z = src.ndim == 3;
    int zchunk = 1;
    int64_t gz = 1;
    if (z) {
        int dev = 0;
        CLE_CUDA(cudaGetDevice(&dev));
        // enough CTAs for 4 waves of 2048-thread SMs, chunks of >= 8 planes
        const int64_t want = (int64_t)num_sms(dev) * 32;
        int64_t chunks = (want + gx * gy - 1) / (gx * gy);
        chunks = std::max<int64_t>(1, std::min<int64_t>(chunks, src.D / 8));
        zchunk = (int)((src.D + chunks - 1) / chunks);
        gz = (src.D + zchunk - 1) / zchunk;
        if (gz > 65535) { set_error("erode_box: image too large"); return CLE_ERR_TOO_LARGE; }
    }
    const dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)gz), block(kEX, kEY);
    if (z)
        erode_box_kernel<Ts, Td, true><<<grid, block, 0, st>>>((const Ts *)src.data, (Td *)dst.data, (int)src.D,
                                                              (int)src.H, (int)src.W, zchunk);
    else
        erode_box_kernel<Ts, Td, false><<<grid, block, 0, st>>>((const Ts *)src.data, (Td *)dst.data, 1,
                                                               (int)src.H, (int)src.W, 1);
    CLE_LAUNCH_CHECK("erode_box");
    return CLE_OK;
}

template <typename Ts>
int erode_dst(const Img &src, const Img &dst, cudaStream_t st) {
    switch (dst.dtype) {
        case CLE_U8: return launch_erode<Ts, uint8_t>(src, dst, st);
        case CLE_U16: return launch_erode<Ts, uint16_t>(src, dst, st);
        case CLE_U32: return launch_erode<Ts, uint32_t>(src, dst, st);
        case CLE_F32: return launch_erode<Ts, float>(src, dst, st);
        default: set_error("erode_box: unsupported destination dtype %d", dst.dtype); return CLE_ERR_DTYPE;
    }
}

// ---- minimum_box / maximum_box (separable, clamped windows) -------------
// _tier1/_minimum_box.py:6-55, _tier1/_maximum_box.py (minimum/maximum_separable_
// {2,3}d_x.cl, absent from the checkout): passes along x, then y, then z (3D), each
// the minimum (maximum) over v + i*e, i = -c..c, c = (N-1)/2 with
// N = int(2*radius + 1), reads clamped to the edge (so the window is the
// in-range part of it); a pass with radius <= 0 is a copy.  min/max are exact,
// so the float32 result does not depend on the order of the comparisons.
constexpr int kLX = 256;        // x pass: outputs per CTA
constexpr int kLT = 64;         // y/z passes: outputs per CTA along the axis
constexpr int kLC = 32;         // y/z passes: columns per CTA

template <bool MAX>
__device__ __forceinline__ float mm(float a, float b) { return MAX ? fmaxf(a, b) : fminf(a, b); }

template <bool MAX>
__global__ void __launch_bounds__(kLX)
minmax_x_kernel(const float *__restrict__ src, float *__restrict__ dst, int W, int r) {
    extern __shared__ float row[];                 // [kLX + 2r]
    const int64_t line = (int64_t)blockIdx.z * gridDim.y + blockIdx.y;
    const float *s = src + line * W;
    const int x0 = blockIdx.x * kLX;
    for (int i = threadIdx.x; i < kLX + 2 * r; i += kLX) row[i] = s[clampi(x0 - r + i, 0, W - 1)];
    __syncthreads();
    const int x = x0 + (int)threadIdx.x;
    if (x >= W) return;
    float m = row[threadIdx.x];
    for (int i = 1; i <= 2 * r; ++i) m = mm<MAX>(m, row[threadIdx.x + i]);
    dst[line * W + x] = m;
}

// Pass along an axis of length L and element stride S (y: S = W, z: S = H*W);
// blockIdx.z indexes the remaining coordinate with stride OS.
template <bool MAX>
__global__ void __launch_bounds__(kLC * 8)
minmax_axis_kernel(const float *__restrict__ src, float *__restrict__ dst, int W, int L, int64_t S,
                   int64_t OS, int r) {
    extern __shared__ float tile[];                // [kLT + 2r][kLC]
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x = blockIdx.x * kLC + tx;
    const int a0 = blockIdx.y * kLT;
    const int64_t base = (int64_t)blockIdx.z * OS + min(x, W - 1);
    for (int i = ty; i < kLT + 2 * r; i += 8) tile[i * kLC + tx] = src[base + (int64_t)clampi(a0 - r + i, 0, L - 1) * S];
    __syncthreads();
    if (x >= W) return;
    for (int o = ty; o < kLT; o += 8) {
        const int a = a0 + o;
        if (a >= L) break;
        float m = tile[o * kLC + tx];
        for (int i = 1; i <= 2 * r; ++i) m = mm<MAX>(m, tile[(o + i) * kLC + tx]);
        dst[(int64_t)blockIdx.z * OS + x + (int64_t)a * S] = m;
    }
}

constexpr int kMaxBoxRadius = 700;   // shared tile (kLT + 2r) x 32 floats <= 187 KB

template <bool MAX>
int minmax_pass(const float *src, float *dst, const Img &im, int axis, int r, cudaStream_t st) {
    const int64_t n = im.n();
    if (r <= 0) {
        if (dst != src) CLE_CUDA(cudaMemcpyAsync(dst, src, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
        return CLE_OK;
    }
    if (im.H > 65535 || im.D > 65535) { set_error("minimum/maximum box: image too large"); return CLE_ERR_TOO_LARGE; }
    if (axis == 0) {
        r = (int)std::min<int64_t>(r, im.W - 1);
        const size_t smem = sizeof(float) * (kLX + 2 * r);
        CLE_CUDA(cudaFuncSetAttribute(minmax_x_kernel<MAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        minmax_x_kernel<MAX><<<dim3((unsigned)((im.W + kLX - 1) / kLX), (unsigned)im.H, (unsigned)im.D), kLX, smem,
                               st>>>(src, dst, (int)im.W, r);
    } else {
        const int64_t L = axis == 1 ? im.H : im.D;
        r = (int)std::min<int64_t>(r, L - 1);
        if (r == 0) {
            CLE_CUDA(cudaMemcpyAsync(dst, src, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
            return CLE_OK;
        }
        const int64_t S = axis == 1 ? im.W : im.H * im.W;
        const int64_t other = axis == 1 ? im.D : im.H;
        const int64_t OS = axis == 1 ? im.H * im.W : im.W;
        const size_t smem = sizeof(float) * (size_t)(kLT + 2 * r) * kLC;
        CLE_CUDA(cudaFuncSetAttribute(minmax_axis_kernel<MAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        minmax_axis_kernel<MAX><<<dim3((unsigned)((im.W + kLC - 1) / kLC), (unsigned)((L + kLT - 1) / kLT),
                                       (unsigned)other), dim3(kLC, 8), smem, st>>>(src, dst, (int)im.W, (int)L, S, OS, r);
    }
    CLE_LAUNCH_CHECK("minimum/maximum box");
    return CLE_OK;
}

__global__ void to_f32_kernel_any_u8(const uint8_t *s, float *d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) d[i] = s[i];
}
__global__ void to_f32_kernel_any_u16(const uint16_t *s, float *d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) d[i] = s[i];
}

__global__ void top_hat_sub_kernel(const float *__restrict__ a, const float *__restrict__ b, float *__restrict__ d,
                                   int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = __fsub_rn(a[i], b[i]);            // add_images_weighted(a, b, 1, -1)
}

}  // namespace

size_t box_filter_workspace_bytes(const Img &im) {
    Arena a(nullptr, 0);
    a.take<float>(im.n());      // source as float32 (u8/u16 sources)
    a.take<float>(im.n());      // pass temporary
    a.take<float>(im.n());      // second temporary (top-hat opening)
    return a.off;
}

// min (MAX=false) or max box of `in` (float32) into `out` (not aliasing `in`);
// tmp: n floats
template <bool MAX>
static int box3(const float *in, float *out, float *tmp, const Img &im, const int r[3], cudaStream_t st) {
    if (im.ndim == 3) {                // x -> out, y -> tmp, z -> out
        CLE_TRY(minmax_pass<MAX>(in, out, im, 0, r[0], st));
        CLE_TRY(minmax_pass<MAX>(out, tmp, im, 1, r[1], st));
        return minmax_pass<MAX>(tmp, out, im, 2, r[2], st);
    }
    CLE_TRY(minmax_pass<MAX>(in, tmp, im, 0, r[0], st));   // x -> tmp, y -> out
    return minmax_pass<MAX>(tmp, out, im, 1, r[1], st);
}

static int radii(const Img &im, double rx, double ry, double rz, int r[3]) {
    const double rr[3] = {rx, ry, rz};
    for (int i = 0; i < 3; ++i) {
        if (!(rr[i] > 0)) { r[i] = 0; continue; }
        const int64_t n = (int64_t)(rr[i] * 2 + 1);     // radius_to_kernel_size
        r[i] = (int)std::min<int64_t>((n - 1) / 2, kMaxBoxRadius);
        if ((n - 1) / 2 > kMaxBoxRadius) {
            set_error("minimum/maximum box: radius above %d", kMaxBoxRadius);
            return CLE_ERR_ARG;
        }
    }
    if (im.ndim == 2) r[2] = 0;
    return CLE_OK;
}

// The source as float32: in place when it is float32 and not the destination,
// else converted / copied into the workspace.
static int float_source(const Img &src, const Img &dst, Arena &ws, const float **out, cudaStream_t st) {
    float *f = ws.take<float>(src.n());
    if (src.dtype == CLE_F32 && src.data != dst.data) { *out = (const float *)src.data; return CLE_OK; }
    if (src.dtype == CLE_F32) {
        if (f) CLE_CUDA(cudaMemcpyAsync(f, src.data, sizeof(float) * src.n(), cudaMemcpyDeviceToDevice, st));
        *out = f;
        return CLE_OK;
    }
    const int b = launch_blocks(src.n(), 256);
    if (src.dtype == CLE_U8) to_f32_kernel_any_u8<<<b, 256, 0, st>>>((const uint8_t *)src.data, f, src.n());
    else if (src.dtype == CLE_U16) to_f32_kernel_any_u16<<<b, 256, 0, st>>>((const uint16_t *)src.data, f, src.n());
    else { set_error("box filter: unsupported source dtype %d", src.dtype); return CLE_ERR_DTYPE; }
    CLE_LAUNCH_CHECK("to float32");
    *out = f;
    return CLE_OK;
}

int box_filter(const Img &src, const Img &dst, double rx, double ry, double rz, bool is_max, Arena &ws,
               cudaStream_t st) {
    CLE_TRY(same_shape(src, dst, "source", "destination"));
    if (dst.dtype != CLE_F32) { set_error("minimum/maximum box: destination must be float32"); return CLE_ERR_DTYPE; }
    int r[3];
    CLE_TRY(radii(src, rx, ry, rz, r));
    const float *in = nullptr;
    CLE_TRY(float_source(src, dst, ws, &in, st));
    float *tmp = ws.take<float>(src.n());
    if (!ws.ok()) { set_error("minimum/maximum box: workspace too small"); return CLE_ERR_WORKSPACE; }
    if (src.n() == 0) return CLE_OK;
    return is_max ? box3<true>(in, (float *)dst.data, tmp, src, r, st)
                  : box3<false>(in, (float *)dst.data, tmp, src, r, st);
}

// top_hat_box: _tier2/_top_hat_box.py:37-43
int top_hat_box(const Img &src, const Img &dst, double rx, double ry, double rz, Arena &ws, cudaStream_t st) {
    CLE_TRY(same_shape(src, dst, "source", "destination"));
    if (dst.dtype != CLE_F32) { set_error("top_hat_box: destination must be float32"); return CLE_ERR_DTYPE; }
    int r[3];
    CLE_TRY(radii(src, rx, ry, rz, r));
    const float *in = nullptr;
    CLE_TRY(float_source(src, dst, ws, &in, st));
    float *tmp = ws.take<float>(src.n());
    float *open_ = ws.take<float>(src.n());
    if (!ws.ok()) { set_error("top_hat_box: workspace too small"); return CLE_ERR_WORKSPACE; }
    const int64_t n = src.n();
    if (n == 0) return CLE_OK;
    float *d = (float *)dst.data;
    // opening: maximum_box(minimum_box(src)) into open_ (dst serves as a temporary)
    CLE_TRY(box3<false>(in, d, tmp, src, r, st));
    CLE_TRY(box3<true>(d, open_, tmp, src, r, st));
    top_hat_sub_kernel<<<launch_blocks(n, 256), 256, 0, st>>>(in, open_, d, n);
    CLE_LAUNCH_CHECK("top_hat_box");
    return CLE_OK;
}

int erode_box(const Img &src, const Img &dst, cudaStream_t st) {
    CLE_TRY(same_shape(src, dst, "source", "destination"));
    if (src.n() == 0) return CLE_OK;
    switch (src.dtype) {
        case CLE_U8: return erode_dst<uint8_t>(src, dst, st);
        case CLE_U16: return erode_dst<uint16_t>(src, dst, st);
        case CLE_U32: return erode_dst<uint32_t>(src, dst, st);
        case CLE_I32: return erode_dst<int32_t>(src, dst, st);
        case CLE_F32: return erode_dst<float>(src, dst, st);
        default: set_error("erode_box: unsupported source dtype %d", src.dtype); return CLE_ERR_DTYPE;
    }
}

}  // namespace cle
