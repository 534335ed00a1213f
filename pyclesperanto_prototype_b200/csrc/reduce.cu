// reduce.cu -- global min/max, the 256-bin histogram, device Otsu, and the
// element-wise ops of the path (greater_constant, binary_and, mask).
#include <cfloat>

#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

constexpr int kRedThreads = 512;

template <typename T>
__device__ __forceinline__ void minmax_acc(T v, float &a, float &b) {
    float f = to_f32(v);
    a = fminf(a, f);
    b = fmaxf(b, f);
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads)
minmax_partial_kernel(const T *__restrict__ src, int64_t n, float *__restrict__ partial) {
    float a = INFINITY, b = -INFINITY;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if constexpr (sizeof(T) == 4) {
        // 128-bit loads over the aligned body
        const int64_t n4 = ((reinterpret_cast<uintptr_t>(src) & 15) == 0) ? n / 4 : 0;
        const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
        for (int64_t j = i; j < n4; j += stride) {
            uint4 u = __ldcs(s4 + j);
            T v[4];
            memcpy(v, &u, 16);
#pragma unroll
            for (int k = 0; k < 4; ++k) minmax_acc(v[k], a, b);
        }
        for (int64_t j = n4 * 4 + i; j < n; j += stride) minmax_acc(src[j], a, b);
    } else {
        for (int64_t j = i; j < n; j += stride) minmax_acc(src[j], a, b);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a = fminf(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = fmaxf(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    __shared__ float sa[32], sb[32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sa[w] = a; sb[w] = b; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        a = l < nw ? sa[l] : INFINITY;
        b = l < nw ? sb[l] : -INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a = fminf(a, __shfl_xor_sync(0xffffffffu, a, o));
            b = fmaxf(b, __shfl_xor_sync(0xffffffffu, b, o));
        }
        if (l == 0) {
            partial[2 * blockIdx.x] = a;
            partial[2 * blockIdx.x + 1] = b;
        }
    }
}

__global__ void minmax_final_kernel(const float *__restrict__ partial, int blocks,
                                    float *__restrict__ out) {
    float a = INFINITY, b = -INFINITY;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) {
        a = fminf(a, partial[2 * i]);
        b = fmaxf(b, partial[2 * i + 1]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a = fminf(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = fmaxf(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    __shared__ float sa[32], sb[32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sa[w] = a; sb[w] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            a = fminf(a, sa[k]);
            b = fmaxf(b, sb[k]);
        }
        out[0] = a;
        out[1] = b;
    }
}

int minmax_blocks(int64_t n) { return launch_blocks(n / 4 + 1, kRedThreads, 4); }

// ---------------------------------------------------------------------------
// Histogram (A6): bin = convert_uint_sat(((v - min) * (bins-1)) / range + 0.5f)
// in float32, per-y-row exact integer partials, then a float32 running sum
// over rows in order (_tier3/_histogram.py:97-128).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t cvt_uint_sat_f(float t) {
    if (!(t > 0.0f)) return 0u;
    if (t >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)t;
}

__device__ __forceinline__ int hist_bin(float v, float mn, float range, float bm1, int bins) {
    float t = __fdiv_rn(__fmul_rn(__fsub_rn(v, mn), bm1), range);
    uint32_t b = cvt_uint_sat_f(__fadd_rn(t, 0.5f));
    return b < (uint32_t)bins ? (int)b : -1;
}

// The same bin with a multiply by the reciprocal of the range: the product
// differs from the IEEE quotient by under 2 ulp (< 2^-15 for bins <= 256), so
// wherever q + 0.5 lies at least 2^-8 from an integer the truncation gives
// the same bin; everything else (near a bin edge, NaN, inf, an empty range)
// takes the exact division.
// The bin from q = (v - min) * (bins-1) * (1/range) + 0.5 (each step rounded),
// or the exact division near a bin edge.
__device__ __forceinline__ int hist_bin_from_q(float q, float v, float mn, float range, float bm1, int bins) {
    const float d = fabsf(__fsub_rn(q, rintf(q)));
    if (d >= 0.00390625f && q >= 0.0f && q < 65536.0f) {
        const uint32_t b = (uint32_t)q;
        return b < (uint32_t)bins ? (int)b : -1;
    }
    return hist_bin(v, mn, range, bm1, bins);
}

__device__ __forceinline__ int hist_bin_fast(float v, float mn, float range, float rr, float bm1, int bins) {
    const float a = __fmul_rn(__fsub_rn(v, mn), bm1);
    const float q = __fadd_rn(__fmul_rn(a, rr), 0.5f);
    return hist_bin_from_q(q, v, mn, range, bm1, bins);
}

constexpr int kHistThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kHistThreads)
hist_rows_kernel(const T *__restrict__ src, int64_t D, int64_t H, int64_t W, int bins,
                 int zchunk, const float *__restrict__ d_minmax, uint32_t *__restrict__ part,
                 FastDiv fw, FastDiv fw4) {
    extern __shared__ uint32_t sh[];   // (warps x bins) when private, else bins
    const int nwarps = kHistThreads / 32;
    const bool priv = bins <= 512;
    const int ncopies = priv ? nwarps : 1;
    for (int i = threadIdx.x; i < ncopies * bins; i += kHistThreads) sh[i] = 0;
    __syncthreads();
    const float mn = d_minmax[0];
    const float range = __fsub_rn(d_minmax[1], mn);
    const float bm1 = (float)(bins - 1);
    const float rr = __frcp_rn(range);
    const bool fast = bins <= 256;
    const int64_t y = blockIdx.x;
    const int64_t z0 = (int64_t)blockIdx.y * zchunk;
    const int64_t z1 = min(D, z0 + zchunk);
    uint32_t *mine = sh + (priv ? (threadIdx.x >> 5) * bins : 0);
    const unsigned lane = threadIdx.x & 31;
    auto count = [&](int b) {
        // warp-aggregated increment: one shared atomic per distinct bin
        unsigned peers = __match_any_sync(0xffffffffu, b);
        if (b >= 0 && (__ffs(peers) - 1) == (int)lane) atomicAdd(&mine[b], (uint32_t)__popc(peers));
    };
    auto bin_of = [&](float x) {
        return fast ? hist_bin_fast(x, mn, range, rr, bm1, bins) : hist_bin(x, mn, range, bm1, bins);
    };
    if constexpr (std::is_same<T, float>::value) {
        if ((W & 3) == 0 && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
            // float rows of a multiple of 4: 128-bit loads, 2 per thread per
            // round (8 voxels), all issued before the binning.  A lane whose 8
            // voxels share one bin (most of a blurred image's background)
            // joins one warp-aggregated add of 8 per lane; the other lanes
            // add each run of equal bins with one shared atomic.
            const uint32_t W4 = (uint32_t)(W >> 2);
            const uint32_t span4 = (uint32_t)((z1 - z0) * W4);
            for (uint32_t base = 0; base < span4; base += 2 * kHistThreads) {
                float4 q[2];
                bool ok[2];
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const uint32_t j = base + k * kHistThreads + threadIdx.x;
                    ok[k] = j < span4;
                    const uint32_t zz = fw4.div(j), x4 = j - zz * W4;
                    q[k] = ok[k] ? __ldg(reinterpret_cast<const float4 *>(src + ((z0 + zz) * H + y) * W) + x4)
                                 : make_float4(0.f, 0.f, 0.f, 0.f);
                }
                int b[8];
                if (fast) {
                    // the fast bins two at a time: (v + (-min)) * (bins-1) * (1/range)
                    // + 0.5 in packed round-to-nearest pairs, the same roundings
                    // as hist_bin_fast's scalar operations
                    const float2 nmn = make_float2(-mn, -mn), s2 = make_float2(bm1, bm1);
                    const float2 r2 = make_float2(rr, rr), h2 = make_float2(0.5f, 0.5f);
                    const float v[8] = {q[0].x, q[0].y, q[0].z, q[0].w, q[1].x, q[1].y, q[1].z, q[1].w};
#pragma unroll
                    for (int k = 0; k < 8; k += 2) {
                        const float2 a = __fmul2_rn(__fadd2_rn(make_float2(v[k], v[k + 1]), nmn), s2);
                        const float2 t = __fadd2_rn(__fmul2_rn(a, r2), h2);
                        b[k] = ok[k / 4] ? hist_bin_from_q(t.x, v[k], mn, range, bm1, bins) : -1;
                        b[k + 1] = ok[k / 4] ? hist_bin_from_q(t.y, v[k + 1], mn, range, bm1, bins) : -1;
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 2; ++k) {
                        b[4 * k + 0] = ok[k] ? bin_of(q[k].x) : -1;
                        b[4 * k + 1] = ok[k] ? bin_of(q[k].y) : -1;
                        b[4 * k + 2] = ok[k] ? bin_of(q[k].z) : -1;
                        b[4 * k + 3] = ok[k] ? bin_of(q[k].w) : -1;
                    }
                }
                bool uni = b[0] >= 0;
#pragma unroll
                for (int k = 1; k < 8; ++k) uni = uni && b[k] == b[0];
                {
                    const int key = uni ? b[0] : -1;
                    const unsigned peers = __match_any_sync(0xffffffffu, key);
                    if (key >= 0 && (__ffs(peers) - 1) == (int)lane) atomicAdd(&mine[key], 8u * (uint32_t)__popc(peers));
                }
                if (!uni) {
                    int cur = b[0];
                    uint32_t n = 1;
#pragma unroll
                    for (int k = 1; k < 8; ++k) {
                        if (b[k] == cur) {
                            ++n;
                        } else {
                            if (cur >= 0) atomicAdd(&mine[cur], n);
                            cur = b[k];
                            n = 1;
                        }
                    }
                    if (cur >= 0) atomicAdd(&mine[cur], n);
                }
            }
            goto merge;
        }
    }
    {
    // the block's voxels, (z0..z1) x W, visited 4 per thread per round with
    // all loads issued before the binning
    const uint32_t span = (uint32_t)((z1 - z0) * W);
    for (uint32_t base = 0; base < span; base += 4 * kHistThreads) {
        float v[4];
        bool ok[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t j = base + k * kHistThreads + threadIdx.x;
            ok[k] = j < span;
            const uint32_t zz = fw.div(j), xx = j - zz * (uint32_t)W;
            v[k] = ok[k] ? to_f32(src[((z0 + zz) * H + y) * W + xx]) : 0.0f;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) count(!ok[k] ? -1 : bin_of(v[k]));
    }
    }
merge:
    __syncthreads();
    for (int b = threadIdx.x; b < bins; b += kHistThreads) {
        uint32_t c = 0;
        for (int k = 0; k < ncopies; ++k) c += sh[k * bins + b];
        if (c) atomicAdd(&part[y * bins + b], c);
    }
}

// hist[b] = float32 running sum of the row partials over y = 0..H-1 in order
// (the reference's sum_z_projection).  Partials and their running sums are
// integers, so while the running sum stays below 2^24 every float32 addition
// is exact and the result is the exact integer total.  Bins whose total
// reaches 2^24 (at most voxels / 2^24 of them) are summed in row order by one
// warp each; the others take their exact total.  A CTA owns 32 bins: warp w
// adds rows w, w + 32, ... of its lane's bin with 8 loads in flight, so the
// totals take a few memory round trips instead of one per row.
constexpr int kRowsumBins = 32;
__global__ void __launch_bounds__(1024)
hist_rowsum_kernel(const uint32_t *__restrict__ part, int64_t H, int bins,
                   float *__restrict__ hist) {
    __shared__ unsigned long long s_tot[32][kRowsumBins + 1];
    __shared__ unsigned long long s_bin[kRowsumBins];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int b = blockIdx.x * kRowsumBins + lane;
    unsigned long long acc = 0;
    if (b < bins) {
        int64_t y = warp;
        for (; y + 7 * 32 < H; y += 8 * 32) {
            uint32_t v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = part[(y + q * 32) * bins + b];
#pragma unroll
            for (int q = 0; q < 8; ++q) acc += v[q];
        }
        for (; y < H; y += 32) acc += part[y * bins + b];
    }
    s_tot[warp][lane] = acc;
    __syncthreads();
    if (warp == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < 32; ++w) t += s_tot[w][lane];
        s_bin[lane] = t;
        if (b < bins && t < (1ull << 24)) hist[b] = (float)t;
    }
    __syncthreads();
    // ordered float32 sums: warp j takes bin j of the CTA when its total is
    // at or above 2^24
    const int bb = blockIdx.x * kRowsumBins + warp;
    if (bb >= bins || s_bin[warp] < (1ull << 24)) return;
    float acc32 = 0.0f;
    for (int64_t y0 = 0; y0 < H; y0 += 32) {
        const int64_t y = y0 + lane;
        const uint32_t v = (y < H) ? part[y * bins + bb] : 0u;
        const int n = (H - y0 < 32) ? (int)(H - y0) : 32;
#pragma unroll
        for (int k = 0; k < 32; ++k) {
            const uint32_t x = __shfl_sync(0xffffffffu, v, k);
            if (k < n) acc32 = __fadd_rn(acc32, (float)x);
        }
    }
    if (lane == 0) hist[bb] = acc32;
}

// A7: scikit-image Otsu on the histogram, float64, no contraction, numpy's
// sequential cumsum, first-occurrence argmax with NaN as maximum
// (_tier9/_threshold_otsu.py:38-49, :83-106).  Only the running sums are
// sequential (numpy's cumsum order); the divisions and the between-class
// variances are elementwise and run in parallel.
__global__ void __launch_bounds__(256)
otsu_kernel(const float *__restrict__ hist, const float *__restrict__ d_minmax,
            double *__restrict__ d_thr, float *__restrict__ d_thr32) {
    constexpr int B = 256;
    __shared__ double bc[B], c[B], w1[B], w2[B], s1[B], s2[B], var[B];
    const int t = threadIdx.x;
    const float mn = d_minmax[0];
    const float range32 = __fsub_rn(d_minmax[1], mn);
    bc[t] = __dadd_rn(__ddiv_rn(__dmul_rn((double)t, (double)range32), 255.0), (double)mn);
    c[t] = (double)hist[t];
    __syncthreads();
    if (t == 0) {
        double acc = 0.0, accm = 0.0;
        for (int i = 0; i < B; ++i) {
            acc = __dadd_rn(acc, c[i]);
            accm = __dadd_rn(accm, __dmul_rn(c[i], bc[i]));
            w1[i] = acc;
            s1[i] = accm;
        }
    } else if (t == 32) {
        double acc = 0.0, accm = 0.0;
        for (int i = B - 1; i >= 0; --i) {
            acc = __dadd_rn(acc, c[i]);
            accm = __dadd_rn(accm, __dmul_rn(c[i], bc[i]));
            w2[i] = acc;
            s2[i] = accm;
        }
    }
    __syncthreads();
    if (t < B - 1) {
        const double m1 = __ddiv_rn(s1[t], w1[t]);
        const double m2 = __ddiv_rn(s2[t + 1], w2[t + 1]);
        const double d = __dsub_rn(m1, m2);
        var[t] = __dmul_rn(__dmul_rn(w1[t], w2[t + 1]), __dmul_rn(d, d));
    }
    __syncthreads();
    if (t == 0) {
        int idx = 0;
        double best = 0.0;
        for (int i = 0; i < B - 1; ++i) {
            const double v = var[i];
            if (v != v) { idx = i; break; }
            if (i == 0 || v > best) { best = v; idx = i; }
        }
        const double thr = bc[idx];
        if (d_thr) *d_thr = thr;
        if (d_thr32) *d_thr32 = __double2float_rn(thr);
    }
}

template <typename Ts, typename Td>
__global__ void greater_kernel(const Ts *__restrict__ src, Td *__restrict__ dst, int64_t n,
                               float c, const float *__restrict__ d_c) {
    const float k = d_c ? *d_c : c;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (Td)(to_f32(src[i]) > k ? 1 : 0);
}

template <typename Ta, typename Tb, typename Td>
__global__ void and_kernel(const Ta *__restrict__ a, const Tb *__restrict__ b, Td *__restrict__ d,
                           int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        d[i] = (Td)((a[i] != (Ta)0 && b[i] != (Tb)0) ? 1 : 0);
}

// clij_convert_*_sat (_tier0/preamble.cl:505-591)
template <typename Td> __device__ __forceinline__ Td sat_from_f(float v);
template <> __device__ __forceinline__ float sat_from_f<float>(float v) { return v; }
template <> __device__ __forceinline__ uint32_t sat_from_f<uint32_t>(float v) {
    if (v > 4294967295.0f) return 0xFFFFFFFFu;
    if (!(v >= 0.0f)) return 0u;
    return (uint32_t)v;
}
template <> __device__ __forceinline__ uint8_t sat_from_f<uint8_t>(float v) {
    if (v > 255.0f) return 255;
    if (!(v >= 0.0f)) return 0;
    return (uint8_t)v;
}
template <> __device__ __forceinline__ uint16_t sat_from_f<uint16_t>(float v) {
    if (v > 65535.0f) return 65535;
    if (!(v >= 0.0f)) return 0;
    return (uint16_t)v;
}

template <typename Ts, typename Tm, typename Td>
__global__ void mask_kernel(const Ts *__restrict__ s, const Tm *__restrict__ m, Td *__restrict__ d,
                            int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        d[i] = sat_from_f<Td>(m[i] != (Tm)0 ? to_f32(s[i]) : 0.0f);
}

template <typename T>
__global__ void label_max_partial(const T *__restrict__ s, int64_t n, uint32_t *__restrict__ out) {
    uint32_t m = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t v;
        if constexpr (std::is_floating_point<T>::value) v = s[i] > (T)0 ? (uint32_t)(int64_t)s[i] : 0u;
        else v = (uint32_t)s[i];
        m = max(m, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

}  // namespace

// ---------------------------------------------------------------------------

size_t minmax_workspace_bytes(const Img &im) {
    Arena a(nullptr, 0);
    a.take<float>(2 * (size_t)minmax_blocks(im.n()));
    return a.off;
}

int minmax_finish(const float *partial, int blocks, float *d_out, cudaStream_t st) {
    minmax_final_kernel<<<1, 1024, 0, st>>>(partial, blocks, d_out);
    CLE_LAUNCH_CHECK("minmax finish");
    return CLE_OK;
}

int minmax(const Img &im, float *d_out, Arena &ws, cudaStream_t st) {
    const int blocks = minmax_blocks(im.n());
    float *partial = ws.take<float>(2 * (size_t)blocks);
    if (!ws.ok()) { set_error("minimum_maximum: workspace too small"); return CLE_ERR_WORKSPACE; }
    switch (im.dtype) {
        case CLE_F32: minmax_partial_kernel<float><<<blocks, kRedThreads, 0, st>>>((const float *)im.data, im.n(), partial); break;
        case CLE_U16: minmax_partial_kernel<uint16_t><<<blocks, kRedThreads, 0, st>>>((const uint16_t *)im.data, im.n(), partial); break;
        case CLE_U8: minmax_partial_kernel<uint8_t><<<blocks, kRedThreads, 0, st>>>((const uint8_t *)im.data, im.n(), partial); break;
        case CLE_U32: minmax_partial_kernel<uint32_t><<<blocks, kRedThreads, 0, st>>>((const uint32_t *)im.data, im.n(), partial); break;
        default: set_error("minimum_maximum: unsupported dtype %d", im.dtype); return CLE_ERR_DTYPE;
    }
    minmax_final_kernel<<<1, 1024, 0, st>>>(partial, blocks, d_out);
    CLE_LAUNCH_CHECK_N("minmax", 2);
    return CLE_OK;
}

size_t histogram_workspace_bytes(const Img &im, int bins) {
    Arena a(nullptr, 0);
    a.take<uint32_t>((size_t)im.H * bins);
    return a.off;
}

int histogram(const Img &im, int bins, const float *d_minmax, float *d_hist, Arena &ws,
              cudaStream_t st) {
    if (bins < 1) { set_error("histogram: num_bins must be >= 1"); return CLE_ERR_ARG; }
    uint32_t *part = ws.take<uint32_t>((size_t)im.H * bins);
    if (!ws.ok()) { set_error("histogram: workspace too small"); return CLE_ERR_WORKSPACE; }
    CLE_CUDA(cudaMemsetAsync(part, 0, sizeof(uint32_t) * im.H * bins, st));
    int dev = 0;
    cudaGetDevice(&dev);
    const int64_t target = (int64_t)num_sms(dev) * 8;
    int64_t zchunks = (target + im.H - 1) / im.H;
    if (zchunks > im.D) zchunks = im.D;
    if (zchunks < 1) zchunks = 1;
    const int zchunk = (int)((im.D + zchunks - 1) / zchunks);
    zchunks = (im.D + zchunk - 1) / zchunk;
    if (im.H > 2147483647 || zchunks > 65535) { set_error("histogram: image too large"); return CLE_ERR_TOO_LARGE; }
    dim3 grid((unsigned)im.H, (unsigned)zchunks);
    const size_t smem = sizeof(uint32_t) * bins * (bins <= 512 ? kHistThreads / 32 : 1);
    if (smem > 227 * 1024) { set_error("histogram: too many bins (%d)", bins); return CLE_ERR_ARG; }
    switch (im.dtype) {
        case CLE_F32:
            if (smem > 48 * 1024) CLE_CUDA(cudaFuncSetAttribute(hist_rows_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            hist_rows_kernel<float><<<grid, kHistThreads, smem, st>>>((const float *)im.data, im.D, im.H, im.W, bins, zchunk, d_minmax, part, FastDiv((uint32_t)im.W), FastDiv((uint32_t)std::max<int64_t>(1, im.W / 4)));
            break;
        case CLE_U16:
            if (smem > 48 * 1024) CLE_CUDA(cudaFuncSetAttribute(hist_rows_kernel<uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            hist_rows_kernel<uint16_t><<<grid, kHistThreads, smem, st>>>((const uint16_t *)im.data, im.D, im.H, im.W, bins, zchunk, d_minmax, part, FastDiv((uint32_t)im.W), FastDiv((uint32_t)std::max<int64_t>(1, im.W / 4)));
            break;
        case CLE_U8:
            if (smem > 48 * 1024) CLE_CUDA(cudaFuncSetAttribute(hist_rows_kernel<uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            hist_rows_kernel<uint8_t><<<grid, kHistThreads, smem, st>>>((const uint8_t *)im.data, im.D, im.H, im.W, bins, zchunk, d_minmax, part, FastDiv((uint32_t)im.W), FastDiv((uint32_t)std::max<int64_t>(1, im.W / 4)));
            break;
        default: set_error("histogram: unsupported dtype %d", im.dtype); return CLE_ERR_DTYPE;
    }
    CLE_LAUNCH_CHECK("histogram rows");
    hist_rowsum_kernel<<<(bins + kRowsumBins - 1) / kRowsumBins, 1024, 0, st>>>(part, im.H, bins, d_hist);
    CLE_LAUNCH_CHECK("histogram rowsum");
    return CLE_OK;
}

int otsu(const float *d_hist, const float *d_minmax, double *d_thr, float *d_thr32,
         cudaStream_t st) {
    otsu_kernel<<<1, 256, 0, st>>>(d_hist, d_minmax, d_thr, d_thr32);
    CLE_LAUNCH_CHECK("otsu");
    return CLE_OK;
}

template <typename Ts>
static int greater_dst(const Img &src, const Img &dst, float c, const float *d_c, cudaStream_t st) {
    const int64_t n = src.n();
    const int blocks = launch_blocks(n, 256);
    switch (dst.dtype) {
        case CLE_U8: greater_kernel<Ts, uint8_t><<<blocks, 256, 0, st>>>((const Ts *)src.data, (uint8_t *)dst.data, n, c, d_c); break;
        case CLE_F32: greater_kernel<Ts, float><<<blocks, 256, 0, st>>>((const Ts *)src.data, (float *)dst.data, n, c, d_c); break;
        case CLE_U32: greater_kernel<Ts, uint32_t><<<blocks, 256, 0, st>>>((const Ts *)src.data, (uint32_t *)dst.data, n, c, d_c); break;
        default: set_error("greater_constant: unsupported destination dtype %d", dst.dtype); return CLE_ERR_DTYPE;
    }
    CLE_LAUNCH_CHECK("greater_constant");
    return CLE_OK;
}

int greater_constant(const Img &src, const Img &dst, float c, const float *d_c, cudaStream_t st) {
    CLE_TRY(same_shape(src, dst, "source", "destination"));
    switch (src.dtype) {
        case CLE_F32: return greater_dst<float>(src, dst, c, d_c, st);
        case CLE_U16: return greater_dst<uint16_t>(src, dst, c, d_c, st);
        case CLE_U8: return greater_dst<uint8_t>(src, dst, c, d_c, st);
        case CLE_U32: return greater_dst<uint32_t>(src, dst, c, d_c, st);
        default: set_error("greater_constant: unsupported source dtype %d", src.dtype); return CLE_ERR_DTYPE;
    }
}

template <typename Ta, typename Tb>
static int and_dst(const Img &a, const Img &b, const Img &d, cudaStream_t st) {
    const int64_t n = a.n();
    const int blocks = launch_blocks(n, 256);
    switch (d.dtype) {
        case CLE_U8: and_kernel<Ta, Tb, uint8_t><<<blocks, 256, 0, st>>>((const Ta *)a.data, (const Tb *)b.data, (uint8_t *)d.data, n); break;
        case CLE_F32: and_kernel<Ta, Tb, float><<<blocks, 256, 0, st>>>((const Ta *)a.data, (const Tb *)b.data, (float *)d.data, n); break;
        default: set_error("binary_and: unsupported destination dtype %d", d.dtype); return CLE_ERR_DTYPE;
    }
    CLE_LAUNCH_CHECK("binary_and");
    return CLE_OK;
}

template <typename Ta>
static int and_b(const Img &a, const Img &b, const Img &d, cudaStream_t st) {
    switch (b.dtype) {
        case CLE_U8: return and_dst<Ta, uint8_t>(a, b, d, st);
        case CLE_F32: return and_dst<Ta, float>(a, b, d, st);
        case CLE_U32: return and_dst<Ta, uint32_t>(a, b, d, st);
        default: set_error("binary_and: unsupported dtype %d", b.dtype); return CLE_ERR_DTYPE;
    }
}

int binary_and(const Img &a, const Img &b, const Img &d, cudaStream_t st) {
    CLE_TRY(same_shape(a, b, "operand1", "operand2"));
    CLE_TRY(same_shape(a, d, "operand1", "destination"));
    switch (a.dtype) {
        case CLE_U8: return and_b<uint8_t>(a, b, d, st);
        case CLE_F32: return and_b<float>(a, b, d, st);
        case CLE_U32: return and_b<uint32_t>(a, b, d, st);
        default: set_error("binary_and: unsupported dtype %d", a.dtype); return CLE_ERR_DTYPE;
    }
}

template <typename Ts, typename Tm>
static int mask_dst(const Img &s, const Img &m, const Img &d, cudaStream_t st) {
    const int64_t n = s.n();
    const int blocks = launch_blocks(n, 256);
    switch (d.dtype) {
        case CLE_F32: mask_kernel<Ts, Tm, float><<<blocks, 256, 0, st>>>((const Ts *)s.data, (const Tm *)m.data, (float *)d.data, n); break;
        case CLE_U32: mask_kernel<Ts, Tm, uint32_t><<<blocks, 256, 0, st>>>((const Ts *)s.data, (const Tm *)m.data, (uint32_t *)d.data, n); break;
        case CLE_U8: mask_kernel<Ts, Tm, uint8_t><<<blocks, 256, 0, st>>>((const Ts *)s.data, (const Tm *)m.data, (uint8_t *)d.data, n); break;
        case CLE_U16: mask_kernel<Ts, Tm, uint16_t><<<blocks, 256, 0, st>>>((const Ts *)s.data, (const Tm *)m.data, (uint16_t *)d.data, n); break;
        default: set_error("mask: unsupported destination dtype %d", d.dtype); return CLE_ERR_DTYPE;
    }
    CLE_LAUNCH_CHECK("mask");
    return CLE_OK;
}

template <typename Ts>
static int mask_m(const Img &s, const Img &m, const Img &d, cudaStream_t st) {
    switch (m.dtype) {
        case CLE_U8: return mask_dst<Ts, uint8_t>(s, m, d, st);
        case CLE_F32: return mask_dst<Ts, float>(s, m, d, st);
        case CLE_U32: return mask_dst<Ts, uint32_t>(s, m, d, st);
        default: set_error("mask: unsupported mask dtype %d", m.dtype); return CLE_ERR_DTYPE;
    }
}

int mask_op(const Img &s, const Img &m, const Img &d, cudaStream_t st) {
    CLE_TRY(same_shape(s, m, "source", "mask"));
    CLE_TRY(same_shape(s, d, "source", "destination"));
    switch (s.dtype) {
        case CLE_F32: return mask_m<float>(s, m, d, st);
        case CLE_U32: return mask_m<uint32_t>(s, m, d, st);
        case CLE_U8: return mask_m<uint8_t>(s, m, d, st);
        case CLE_U16: return mask_m<uint16_t>(s, m, d, st);
        default: set_error("mask: unsupported source dtype %d", s.dtype); return CLE_ERR_DTYPE;
    }
}

size_t label_max_workspace_bytes(const Img &) { return 0; }

int label_max(const Img &labels, uint32_t *d_max, Arena &, cudaStream_t st) {
    CLE_CUDA(cudaMemsetAsync(d_max, 0, sizeof(uint32_t), st));
    const int64_t n = labels.n();
    const int blocks = launch_blocks(n, 256, 4);
    switch (labels.dtype) {
        case CLE_U32: label_max_partial<uint32_t><<<blocks, 256, 0, st>>>((const uint32_t *)labels.data, n, d_max); break;
        case CLE_F32: label_max_partial<float><<<blocks, 256, 0, st>>>((const float *)labels.data, n, d_max); break;
        case CLE_U16: label_max_partial<uint16_t><<<blocks, 256, 0, st>>>((const uint16_t *)labels.data, n, d_max); break;
        case CLE_U8: label_max_partial<uint8_t><<<blocks, 256, 0, st>>>((const uint8_t *)labels.data, n, d_max); break;
        default: set_error("label_maximum: unsupported dtype %d", labels.dtype); return CLE_ERR_DTYPE;
    }
    CLE_LAUNCH_CHECK("label_maximum");
    return CLE_OK;
}

}  // namespace cle
