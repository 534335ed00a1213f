// blur_fused.cu -- one-launch separable Gaussian blur for isotropic sigma.
//
// Same arithmetic as the three-pass path in blur.cu (x pass, then y, then z,
// float32 intermediates, clamp-to-edge, acc = fma(w_i, v_i, acc) for
// i = -R..R from 0), fused so the source is read once and the result written
// once:
//   * a CTA owns a kTX x kTY output tile in (x, y) and marches along z over a
//     chunk of planes (plus R halo planes at each end, clamped);
//   * per input plane it stages the clamped (kTY+2R) x (kTX+2R) tile in
//     shared memory -- the next plane's raw values are loaded into registers
//     while the current one is computed and converted to float32 only when
//     stored, so no instruction waits on them early;
//   * x pass: each item produces 8 consecutive x outputs of one row as four
//     packed pairs (fma.rn.f32x2: two independent round-to-nearest FMAs, the
//     same rounding as fmaf) from 128-bit shared loads; the operand pair of an
//     odd offset is formed from the loaded registers;
//   * y pass: each thread produces kRY rows of a pair of adjacent columns,
//     the pair packed, from a register window of 64-bit shared loads;
//   * z pass: a register ring of 2R+1 planes per owned column pair, shifted by one
//     slot per plane (the plane loop is not unrolled, which keeps the kernel's
//     code small enough for the instruction caches).
// Radius R (= sigma_to_kernel_size(sigma)/2) is a template parameter; radii
// above kMaxFusedR or anisotropic sigmas use the three-pass path.  Given a
// partial buffer, each CTA also reduces the exact min / max of the values it
// stores (the global min / max of the result in a one-CTA finish), which
// saves threshold_otsu's separate pass over the blurred image.
#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

constexpr int kTX = 32;          // output columns per CTA
constexpr int kTY = 32;          // output rows per CTA
constexpr int kRY = 2;           // output rows per thread (y and z passes)
constexpr int kCP = kTX / 2;     // column pairs per tile (y and z passes own a pair)
constexpr int kXO = 8;           // x outputs per x-pass item
constexpr int kThreads = kCP * (kTY / kRY);   // 256
constexpr int kWarps = kThreads / 32;

template <int R>
struct Geom {
    static constexpr int ROWS = kTY + 2 * R;                     // staged rows
    static constexpr int COLS = kTX + 2 * R;                     // staged columns
    static constexpr int QUADS = (kXO + 2 * R + 3) / 4;          // float4 per x-pass item
    static constexpr int STRIDE = ((COLS + 3) / 4) * 4 + 4;      // In row stride (floats)
    static constexpr int ROWS_PER_WARP = (ROWS + kWarps - 1) / kWarps;
    static constexpr int COL_LOADS = (COLS + 31) / 32;
    static constexpr int LOADS = ROWS_PER_WARP * COL_LOADS;
    static constexpr int XO_STRIDE = kTX;                        // Xo row stride
    static constexpr size_t SMEM = sizeof(float) * (ROWS * STRIDE + ROWS * kTX);
    static_assert(ROWS * (kTX / kXO) <= kThreads, "x pass: at most one item per thread");
};

// Two CTAs per SM (<= 128 registers, no spills) while the z ring is small.
template <int R>
constexpr int min_ctas() { return R <= 8 ? 2 : 1; }

template <typename Tin, int R, bool Z>
__global__ void __launch_bounds__(kThreads, min_ctas<R>())
blur_fused_kernel(const Tin *__restrict__ src, float *__restrict__ dst, int D, int H, int W,
                  int zchunk, const __grid_constant__ Taps taps, float *__restrict__ mm) {
    using G = Geom<R>;
    constexpr int WIN = 2 * R + 1;
    extern __shared__ __align__(16) float smem[];
    float *In = smem;                          // [ROWS][STRIDE]
    float *Xo = smem + G::ROWS * G::STRIDE;    // [ROWS][kTX]

    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * kTX;
    const int y0 = blockIdx.y * kTY;
    const int z0 = Z ? (int)blockIdx.z * zchunk : 0;
    const int z1 = Z ? min(D, z0 + zchunk) : 1;
    // virtual planes z0-R .. z1-1+R (clamped); 2D: the single plane
    const int nvirt = Z ? (z1 - z0) + 2 * R : 1;
    const int zbase = Z ? z0 - R : 0;
    const int64_t plane = (int64_t)H * W;

    // staging: warp w loads rows w, w+kWarps, ...; lane loads columns
    // lane, lane+32, ... (clamped to the image)
    const int lane = tid & 31, warp = tid >> 5;
    int gx[G::COL_LOADS];
#pragma unroll
    for (int c = 0; c < G::COL_LOADS; ++c) gx[c] = clampi(x0 - R + lane + 32 * c, 0, W - 1);
    // raw source values; converted when stored, so the loads of the next
    // plane stay in flight while the current plane is computed
    Tin pre[G::LOADS];
    auto load_plane = [&](int v) {
        const int zi = Z ? clampi(zbase + v, 0, D - 1) : 0;
        const Tin *p = src + (int64_t)zi * plane;
#pragma unroll
        for (int rr = 0; rr < G::ROWS_PER_WARP; ++rr) {
            const int r = warp + rr * kWarps;
            const Tin *row = p + (int64_t)clampi(y0 - R + r, 0, H - 1) * W;
#pragma unroll
            for (int c = 0; c < G::COL_LOADS; ++c) {
                const bool ok = r < G::ROWS && lane + 32 * c < G::COLS;
                pre[rr * G::COL_LOADS + c] = ok ? __ldg(row + gx[c]) : Tin(0);
            }
        }
    };
    auto store_plane = [&]() {
#pragma unroll
        for (int rr = 0; rr < G::ROWS_PER_WARP; ++rr) {
            const int r = warp + rr * kWarps;
#pragma unroll
            for (int c = 0; c < G::COL_LOADS; ++c)
                if (r < G::ROWS && lane + 32 * c < G::COLS) In[r * G::STRIDE + lane + 32 * c] = to_f32(pre[rr * G::COL_LOADS + c]);
        }
    };

    // y/z ownership: columns tx, tx+1 (a packed pair), rows ry0 .. ry0+kRY-1
    const int tx = (tid % kCP) * 2;
    const int ry0 = (tid / kCP) * kRY;
    const bool c0_ok = (x0 + tx) < W, c1_ok = (x0 + tx + 1) < W;
    const bool pair_store = c1_ok && (W & 1) == 0;     // 8-byte aligned float2 store
    float vmin = INFINITY, vmax = -INFINITY;   // of the stored values (when mm)
    auto store2 = [&](int64_t off, float2 v) {
        if (pair_store) *reinterpret_cast<float2 *>(dst + off) = v;
        else {
            if (c0_ok) dst[off] = v.x;
            if (c1_ok) dst[off + 1] = v.y;
        }
        if (mm) {
            vmin = fminf(vmin, v.x);
            vmax = fmaxf(vmax, v.x);
            if (c1_ok) { vmin = fminf(vmin, v.y); vmax = fmaxf(vmax, v.y); }
        }
    };

    float2 ring[kRY][WIN];
#pragma unroll
    for (int j = 0; j < kRY; ++j)
#pragma unroll
        for (int i = 0; i < WIN; ++i) ring[j][i] = make_float2(0.0f, 0.0f);

    load_plane(0);
    // one plane per iteration, not unrolled (the loop body stays small enough
    // for the instruction caches); the ring shifts by one slot per plane, so
    // ring[j][i] holds plane v - 2R + i
#pragma unroll 1
    for (int v = 0; v < nvirt; ++v) {
        __syncthreads();   // previous plane fully consumed
        store_plane();
        if (v + 1 < nvirt) load_plane(v + 1);
        __syncthreads();
        // x pass: rows 0..ROWS-1, kXO outputs per item as packed pairs; the
        // operand pair of an odd offset is formed from the loaded registers
        if (tid < G::ROWS * (kTX / kXO)) {
            const int r = tid / (kTX / kXO);
            const int xq = (tid - r * (kTX / kXO)) * kXO;
            float2 A[2 * G::QUADS];                    // A[k] = (v[xq+2k], v[xq+2k+1])
            const float4 *pa = reinterpret_cast<const float4 *>(In + r * G::STRIDE + xq);
#pragma unroll
            for (int q = 0; q < G::QUADS; ++q) {
                const float4 f = pa[q];
                A[2 * q] = make_float2(f.x, f.y);
                A[2 * q + 1] = make_float2(f.z, f.w);
            }
            float2 acc[kXO / 2];
#pragma unroll
            for (int p = 0; p < kXO / 2; ++p) acc[p] = make_float2(0.f, 0.f);
#pragma unroll
            for (int i = 0; i < WIN; ++i) {
                const float2 w = make_float2(taps.w[i], taps.w[i]);
#pragma unroll
                for (int p = 0; p < kXO / 2; ++p) {
                    const int o = 2 * p + i;               // operand (v[xq+o], v[xq+o+1])
                    const float2 opnd = (o % 2 == 0) ? A[o / 2] : make_float2(A[o / 2].y, A[o / 2 + 1].x);
                    acc[p] = __ffma2_rn(w, opnd, acc[p]);
                }
            }
            float4 *xo = reinterpret_cast<float4 *>(Xo + r * kTX + xq);
#pragma unroll
            for (int p = 0; p < kXO / 4; ++p)
                xo[p] = make_float4(acc[2 * p].x, acc[2 * p].y, acc[2 * p + 1].x, acc[2 * p + 1].y);
        }
        __syncthreads();
        // y pass: kRY rows of the column pair
        float2 col[kRY + 2 * R];
#pragma unroll
        for (int j = 0; j < kRY + 2 * R; ++j) col[j] = *reinterpret_cast<const float2 *>(Xo + (ry0 + j) * kTX + tx);
        float2 yv[kRY];
#pragma unroll
        for (int j = 0; j < kRY; ++j) {
            float2 a = make_float2(0.f, 0.f);
#pragma unroll
            for (int i = 0; i < WIN; ++i) a = __ffma2_rn(make_float2(taps.w[i], taps.w[i]), col[j + i], a);
            yv[j] = a;
        }
        if constexpr (Z) {
#pragma unroll
            for (int j = 0; j < kRY; ++j) {
#pragma unroll
                for (int i = 0; i < WIN - 1; ++i) ring[j][i] = ring[j][i + 1];
                ring[j][WIN - 1] = yv[j];
            }
            // z pass: output plane z0 + v - 2R once 2R+1 planes are held
            if (v >= 2 * R) {
                const int zo = z0 + v - 2 * R;
#pragma unroll
                for (int j = 0; j < kRY; ++j) {
                    float2 a = make_float2(0.f, 0.f);
#pragma unroll
                    for (int i = 0; i < WIN; ++i) a = __ffma2_rn(make_float2(taps.w[i], taps.w[i]), ring[j][i], a);
                    const int y = y0 + ry0 + j;
                    if (c0_ok && y < H) store2((int64_t)zo * plane + (int64_t)y * W + x0 + tx, a);
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < kRY; ++j) {
                const int y = y0 + ry0 + j;
                if (c0_ok && y < H) store2((int64_t)y * W + x0 + tx, yv[j]);
            }
        }
    }
    if (mm) {
        __shared__ float s_mn[kWarps], s_mx[kWarps];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            vmin = fminf(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
            vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        }
        if (lane == 0) { s_mn[warp] = vmin; s_mx[warp] = vmax; }
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < kWarps; ++w) { vmin = fminf(vmin, s_mn[w]); vmax = fmaxf(vmax, s_mx[w]); }
            const int64_t cta = ((int64_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
            mm[2 * cta] = vmin;
            mm[2 * cta + 1] = vmax;
        }
    }
}

// Grid of the fused launch: (x tiles, y tiles, z chunks); the chunks give about
// 2 x the resident CTAs while keeping the 2R halo planes below ~1/2 of a chunk.
dim3 fused_grid(const Img &src, int R, int &zchunk) {
    const int gx = (int)((src.W + kTX - 1) / kTX);
    const int gy = (int)((src.H + kTY - 1) / kTY);
    int gz = 1;
    zchunk = 1;
    if (src.ndim == 3) {
        int dev = 0;
        cudaGetDevice(&dev);
        const int64_t target = (int64_t)num_sms(dev) * 2 * (R <= 8 ? 2 : 1);   // CTAs
        int64_t chunks = (target + (int64_t)gx * gy - 1) / ((int64_t)gx * gy);
        const int64_t max_chunks = std::max<int64_t>(1, src.D / std::max(2 * R, 1));
        chunks = std::min(chunks, max_chunks);
        chunks = std::max<int64_t>(1, std::min<int64_t>(chunks, src.D));
        zchunk = (int)((src.D + chunks - 1) / chunks);
        gz = (int)((src.D + zchunk - 1) / zchunk);
    }
    return dim3(gx, gy, gz);
}

template <typename Tin, int R, bool Z>
int launch_fused_r(const Img &src, float *dst, const Taps &t, float *mm, cudaStream_t st) {
    using G = Geom<R>;
    static_assert(min_ctas<R>() == (R <= 8 ? 2 : 1), "fused_grid's occupancy rule");
    auto kern = blur_fused_kernel<Tin, R, Z>;
    // set on every call: the attribute belongs to the current device's context
    CLE_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM));
    int zchunk = 1;
    const dim3 grid = fused_grid(src, R, zchunk);
    if (grid.y > 65535 || grid.z > 65535) { set_error("gaussian_blur: image too large for the fused path"); return CLE_ERR_TOO_LARGE; }
    kern<<<grid, kThreads, G::SMEM, st>>>((const Tin *)src.data, dst, (int)src.D, (int)src.H, (int)src.W,
                                          zchunk, t, mm);
    CLE_LAUNCH_CHECK("gaussian_blur fused");
    return CLE_OK;
}

template <typename Tin, bool Z, int R = 1>
int dispatch_r(const Img &src, float *dst, const Taps &t, int r, float *mm, cudaStream_t st) {
    if constexpr (R > kMaxFusedR) {
        set_error("internal: fused radius out of range");
        return CLE_ERR_ARG;
    } else {
        if (r == R) return launch_fused_r<Tin, R, Z>(src, dst, t, mm, st);
        return dispatch_r<Tin, Z, R + 1>(src, dst, t, r, mm, st);
    }
}

}  // namespace

bool fused_blur_applies(const Img &src, double sx, double sy, double sz) {
    if (!(sx > 0) || sx != sy) return false;
    if (src.ndim == 3 && sz != sx) return false;
    if (src.dtype != CLE_F32 && src.dtype != CLE_U16 && src.dtype != CLE_U8) return false;
    const int r = (sigma_to_kernel_size(sx) - 1) / 2;
    return r >= 1 && r <= kMaxFusedR && src.W < (1 << 30) && src.H < (1 << 30);
}

int fused_blur(const Img &src, float *dst, double sigma, cudaStream_t st, float *mm) {
    Taps t;
    CLE_TRY(make_gauss_taps(sigma, t));
    const int r = (t.n - 1) / 2;
    const bool z = src.ndim == 3;
    switch (src.dtype) {
        case CLE_F32: return z ? dispatch_r<float, true>(src, dst, t, r, mm, st) : dispatch_r<float, false>(src, dst, t, r, mm, st);
        case CLE_U16: return z ? dispatch_r<uint16_t, true>(src, dst, t, r, mm, st) : dispatch_r<uint16_t, false>(src, dst, t, r, mm, st);
        case CLE_U8: return z ? dispatch_r<uint8_t, true>(src, dst, t, r, mm, st) : dispatch_r<uint8_t, false>(src, dst, t, r, mm, st);
        default: set_error("gaussian_blur: unsupported source dtype"); return CLE_ERR_DTYPE;
    }
}

size_t blur_minmax_workspace_bytes(const Img &src) {
    // any sigma: the three-pass path with the separate min / max, or the
    // fused partials (at most 4 CTAs per SM's worth of z chunks per tile)
    int dev = 0;
    cudaGetDevice(&dev);
    const int64_t tiles = ((src.W + kTX - 1) / kTX) * ((src.H + kTY - 1) / kTY);
    const int64_t chunks = std::min<int64_t>(std::max<int64_t>(src.D, 1),
                                             ((int64_t)num_sms(dev) * 4 + tiles - 1) / tiles);
    const size_t fused = sizeof(float) * 2 * (size_t)(tiles * chunks) + 256;
    return std::max(fused, separable_workspace_bytes(src) + minmax_workspace_bytes(src));
}

int blur_minmax(const Img &src, float *dst, double sigma, float *d_minmax, Arena &ws, cudaStream_t st) {
    if (!fused_blur_applies(src, sigma, sigma, sigma)) {
        CLE_TRY(gaussian_blur(src, dst, sigma, sigma, sigma, ws, st));
        Img T = src;
        T.data = dst;
        T.dtype = CLE_F32;
        return minmax(T, d_minmax, ws, st);
    }
    int zchunk = 1;
    const dim3 g = fused_grid(src, (sigma_to_kernel_size(sigma) - 1) / 2, zchunk);
    const int ctas = (int)(g.x * g.y * g.z);
    float *partial = ws.take<float>(2 * (size_t)ctas);
    if (!ws.ok()) { set_error("gaussian_blur: workspace too small"); return CLE_ERR_WORKSPACE; }
    CLE_TRY(fused_blur(src, dst, sigma, st, partial));
    return minmax_finish(partial, ctas, d_minmax, st);
}

}  // namespace cle
