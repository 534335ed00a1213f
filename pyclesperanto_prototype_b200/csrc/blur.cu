// blur.cu -- separable Gaussian blur (and the uniform-weight box mean used by
// detect_maxima_box with radius > 0).
//
// Semantics (_tier1/_gaussian_blur.py:39-56, _tier1/_execute_separable_kernel.py:7-76):
// passes along x, then y, then z (3D only), each with clamp-to-edge reads and
// float32 intermediates; a pass with sigma <= 0 is a copy.  Inside a pass
// the output is acc = fma(w_i, v_i, acc) for i = -r..r ascending from 0.
//
// Layout: the row pass stages a run of one x-row (+halo) in shared memory;
// the column passes (y and z) stage a (rows + 2r) x 32-column tile, so every
// global access is a coalesced 128-byte segment.
#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

constexpr int kRowTile = 1024;   // outputs per CTA along x
constexpr int kRowThreads = 256;
constexpr int kColW = 32;        // columns per CTA in the column pass
constexpr int kColRows = 64;     // outputs per CTA along the pass axis
constexpr int kColThreadsY = 8;

template <typename Tin>
__global__ void __launch_bounds__(kRowThreads)
blur_row_kernel(const Tin *__restrict__ src, float *__restrict__ dst, int64_t rows, int W,
                const __grid_constant__ Taps taps) {
    extern __shared__ float s[];
    const int r = (taps.n - 1) / 2;
    const int64_t row = blockIdx.y + (int64_t)blockIdx.z * gridDim.y;
    if (row >= rows) return;
    const int x0 = blockIdx.x * kRowTile;
    const Tin *in = src + row * (int64_t)W;
    const int span = kRowTile + 2 * r;
    for (int i = threadIdx.x; i < span; i += kRowThreads) {
        int x = clampi(x0 - r + i, 0, W - 1);
        s[i] = to_f32(in[x]);
    }
    __syncthreads();
    float *out = dst + row * (int64_t)W;
#pragma unroll 4
    for (int k = 0; k < kRowTile / kRowThreads; ++k) {
        int xo = threadIdx.x + k * kRowThreads;
        if (x0 + xo >= W) break;
        float acc = 0.0f;
        for (int i = 0; i < taps.n; ++i) acc = __fmaf_rn(taps.w[i], s[xo + i], acc);
        out[x0 + xo] = acc;
    }
}

// Pass along an axis of length L with element stride `inner`, for a volume
// viewed as [outer][L][inner].
template <typename Tin>
__global__ void __launch_bounds__(kColW *kColThreadsY)
blur_col_kernel(const Tin *__restrict__ src, float *__restrict__ dst, int64_t inner, int L,
                int64_t outer, const __grid_constant__ Taps taps) {
    extern __shared__ float s[];
    const int r = (taps.n - 1) / 2;
    const int64_t c = (int64_t)blockIdx.x * kColW + threadIdx.x;
    const int l0 = blockIdx.y * kColRows;
    const int64_t o = blockIdx.z;
    if (o >= outer) return;
    const int span = kColRows + 2 * r;
    const int64_t base = o * (int64_t)L * inner;
    for (int j = threadIdx.y; j < span; j += kColThreadsY) {
        int l = clampi(l0 - r + j, 0, L - 1);
        s[j * kColW + threadIdx.x] = (c < inner) ? to_f32(src[base + (int64_t)l * inner + c]) : 0.0f;
    }
    __syncthreads();
    if (c >= inner) return;
    for (int lo = threadIdx.y; lo < kColRows; lo += kColThreadsY) {
        int l = l0 + lo;
        if (l >= L) break;
        float acc = 0.0f;
        for (int i = 0; i < taps.n; ++i) acc = __fmaf_rn(taps.w[i], s[(lo + i) * kColW + threadIdx.x], acc);
        dst[base + (int64_t)l * inner + c] = acc;
    }
}

template <typename Tin>
__global__ void convert_kernel(const Tin *__restrict__ src, float *__restrict__ dst, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = to_f32(src[i]);
}

template <typename Tin>
int launch_pass(const Tin *src, float *dst, const Img &im, int axis, const Taps &t,
                cudaStream_t st) {
    const int r = (t.n - 1) / 2;
    if (axis == 2) {
        const int64_t rows = im.D * im.H;
        dim3 grid((unsigned)((im.W + kRowTile - 1) / kRowTile), (unsigned)std::min<int64_t>(rows, 65535),
                  (unsigned)((rows + 65534) / 65535));
        size_t smem = sizeof(float) * (kRowTile + 2 * r);
        if (smem > 48 * 1024)
            CLE_CUDA(cudaFuncSetAttribute(blur_row_kernel<Tin>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        blur_row_kernel<Tin><<<grid, kRowThreads, smem, st>>>(src, dst, rows, (int)im.W, t);
    } else {
        int64_t inner, outer;
        int L;
        if (axis == 1) { inner = im.W; L = (int)im.H; outer = im.D; }
        else { inner = im.W * im.H; L = (int)im.D; outer = 1; }
        dim3 grid((unsigned)((inner + kColW - 1) / kColW), (unsigned)((L + kColRows - 1) / kColRows),
                  (unsigned)outer);
        dim3 block(kColW, kColThreadsY);
        size_t smem = sizeof(float) * kColW * (kColRows + 2 * r);
        if (smem > 48 * 1024)
            CLE_CUDA(cudaFuncSetAttribute(blur_col_kernel<Tin>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        blur_col_kernel<Tin><<<grid, block, smem, st>>>(src, dst, inner, L, outer, t);
    }
    CLE_LAUNCH_CHECK("blur pass");
    return CLE_OK;
}

template <typename Tin>
int launch_convert(const Tin *src, float *dst, int64_t n, cudaStream_t st) {
    convert_kernel<Tin><<<launch_blocks(n, 256), 256, 0, st>>>(src, dst, n);
    CLE_LAUNCH_CHECK("convert");
    return CLE_OK;
}

template <typename Tin>
int separable_typed(const Img &src, float *dst, const Taps *taps[3], float *t1, float *t2,
                    cudaStream_t st) {
    // pass order x (axis 2), y (axis 1), z (axis 0, 3D only)
    const int passes = (src.ndim == 3) ? 3 : 2;
    const int64_t n = src.n();
    const void *cur = src.data;
    bool cur_is_src = true;
    float *bufs[2] = {t1, t2};
    int which = 0;
    for (int p = 0; p < passes; ++p) {
        float *o = (p == passes - 1) ? dst : bufs[which];
        const Taps *t = taps[p];
        if (cur_is_src) {
            if (t) CLE_TRY(launch_pass<Tin>((const Tin *)cur, o, src, 2 - p, *t, st));
            else CLE_TRY(launch_convert<Tin>((const Tin *)cur, o, n, st));
        } else {
            if (t) CLE_TRY(launch_pass<float>((const float *)cur, o, src, 2 - p, *t, st));
            else if (o != cur) CLE_CUDA(cudaMemcpyAsync(o, cur, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
        }
        cur = o;
        cur_is_src = false;
        which ^= 1;
    }
    return CLE_OK;
}

}  // namespace

size_t separable_workspace_bytes(const Img &im) {
    Arena a(nullptr, 0);
    a.take<float>(im.n());
    a.take<float>(im.n());
    return a.off;
}

int separable_filter(const Img &src, float *dst, const Taps *tx, const Taps *ty, const Taps *tz,
                     Arena &ws, cudaStream_t st) {
    float *t1 = ws.take<float>(src.n());
    float *t2 = ws.take<float>(src.n());
    if (!ws.ok()) {
        set_error("gaussian_blur: workspace too small");
        return CLE_ERR_WORKSPACE;
    }
    const Taps *taps[3] = {tx, ty, tz};
    switch (src.dtype) {
        case CLE_F32: return separable_typed<float>(src, dst, taps, t1, t2, st);
        case CLE_U16: return separable_typed<uint16_t>(src, dst, taps, t1, t2, st);
        case CLE_U8: return separable_typed<uint8_t>(src, dst, taps, t1, t2, st);
        default:
            set_error("gaussian_blur: source dtype %d not supported (u8/u16/f32)", src.dtype);
            return CLE_ERR_DTYPE;
    }
}

int gaussian_blur(const Img &src, float *dst, double sx, double sy, double sz, Arena &ws,
                  cudaStream_t st, int *status) {
    if (fused_blur_applies(src, sx, sy, sz))
        return fused_blur(src, dst, sx, st, nullptr, status);
    Taps tx, ty, tz;
    const Taps *px = nullptr, *py = nullptr, *pz = nullptr;
    if (sx > 0) { CLE_TRY(make_gauss_taps(sx, tx)); px = &tx; }
    if (sy > 0) { CLE_TRY(make_gauss_taps(sy, ty)); py = &ty; }
    if (src.ndim == 3 && sz > 0) { CLE_TRY(make_gauss_taps(sz, tz)); pz = &tz; }
    return separable_filter(src, dst, px, py, pz, ws, st);
}

}  // namespace cle
