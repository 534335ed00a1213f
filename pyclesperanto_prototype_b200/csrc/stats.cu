// stats.cu -- statistics_of_labelled_pixels
// (_tier9/_statistics_of_labelled_pixels.py:7-293, kernels
// _tier9/statistics_per_label_x.cl:1-146, _tier9/standard_deviation_per_label_x.cl:1-96).
//
// Two passes over (labels, intensity), as in the reference (the second needs
// the per-label centroid, mass centre and mean).  A warp covers 32
// consecutive voxels of one x-row, so y and z are warp-uniform; each run of
// equal labels along x contributes count, x-sum and bbox in closed form and
// the intensity fields through a segmented shuffle scan; the run's last lane
// adds them to per-label accumulators (exact integers for coordinates,
// float64 for intensity products, order-preserving int atomics for min/max).
// The finalise kernels apply the reference's float32 column arithmetic and
// its sentinels for labels absent from the image (min FLT_MAX, max -FLT_MAX,
// sums 0, 0/0 = NaN).
#include <cfloat>

#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

constexpr int kST = 256;
constexpr int kBatch = 4;   // row segments per warp round

struct Acc1 {
    uint32_t *cnt;
    unsigned long long *sx, *sy, *sz;
    double *sv, *svx, *svy, *svz;
    int *vmin, *vmax;
    uint32_t *xmin, *xmax, *ymin, *ymax, *zmin, *zmax;
};

struct Acc2 {
    double *sdc, *sdm, *ssq;
    unsigned long long *mdc, *mdm;   // non-negative doubles as bit patterns
    float4 *pc;                      // per label: centroid x, y, z, mean intensity
    float4 *pm;                      // per label: mass centre x, y, z, area
};

Acc1 take_acc1(Arena &a, int64_t L) {
    Acc1 c;
    c.cnt = a.take<uint32_t>(L);
    c.sx = a.take<unsigned long long>(L);
    c.sy = a.take<unsigned long long>(L);
    c.sz = a.take<unsigned long long>(L);
    c.sv = a.take<double>(L);
    c.svx = a.take<double>(L);
    c.svy = a.take<double>(L);
    c.svz = a.take<double>(L);
    c.vmin = a.take<int>(L);
    c.vmax = a.take<int>(L);
    c.xmin = a.take<uint32_t>(L);
    c.xmax = a.take<uint32_t>(L);
    c.ymin = a.take<uint32_t>(L);
    c.ymax = a.take<uint32_t>(L);
    c.zmin = a.take<uint32_t>(L);
    c.zmax = a.take<uint32_t>(L);
    return c;
}

Acc2 take_acc2(Arena &a, int64_t L) {
    Acc2 c;
    c.sdc = a.take<double>(L);
    c.sdm = a.take<double>(L);
    c.ssq = a.take<double>(L);
    c.mdc = a.take<unsigned long long>(L);
    c.mdm = a.take<unsigned long long>(L);
    c.pc = a.take<float4>(L);
    c.pm = a.take<float4>(L);
    return c;
}

// With a device label count (d_L) the init and finalise kernels touch only the
// first min(count, L) labels; L stays the table's row stride.
__device__ __forceinline__ int64_t live_labels(int64_t L, const uint32_t *d_L) {
    return d_L ? ((int64_t)*d_L < L ? (int64_t)*d_L : L) : L;
}

__global__ void stats_init(Acc1 a, Acc2 b, int64_t L, const uint32_t *__restrict__ d_L) {
    const int64_t n = live_labels(L, d_L);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        a.cnt[i] = 0;
        a.sx[i] = a.sy[i] = a.sz[i] = 0ull;
        a.sv[i] = a.svx[i] = a.svy[i] = a.svz[i] = 0.0;
        a.vmin[i] = 0x7FFFFFFF;
        a.vmax[i] = (int)0x80000000;
        a.xmin[i] = a.ymin[i] = a.zmin[i] = 0xFFFFFFFFu;
        a.xmax[i] = a.ymax[i] = a.zmax[i] = 0u;
        b.sdc[i] = b.sdm[i] = b.ssq[i] = 0.0;
        b.mdc[i] = b.mdm[i] = 0ull;
    }
}

template <typename T>
__device__ __forceinline__ uint32_t lab_of(T v) {
    if constexpr (std::is_floating_point<T>::value) return v > (T)0 ? (uint32_t)(int64_t)v : 0u;
    else return (uint32_t)v;
}

struct Seg {
    int lane, hl;
    bool tail;
    __device__ __forceinline__ double scan_add(double v) const {
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            double t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane - o >= hl) v += t;
        }
        return v;
    }
    __device__ __forceinline__ float scan_min(float v) const {
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            float t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane - o >= hl) v = fminf(v, t);
        }
        return v;
    }
    __device__ __forceinline__ float scan_max(float v) const {
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            float t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane - o >= hl) v = fmaxf(v, t);
        }
        return v;
    }
    __device__ __forceinline__ uint32_t scan_addu(uint32_t v) const {
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane - o >= hl) v += t;
        }
        return v;
    }
    __device__ __forceinline__ uint32_t scan_minu(uint32_t v) const {
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane - o >= hl) v = min(v, t);
        }
        return v;
    }
    __device__ __forceinline__ uint32_t scan_maxu(uint32_t v) const {
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane - o >= hl) v = max(v, t);
        }
        return v;
    }
    __device__ __forceinline__ double scan_maxd(double v) const {
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            double t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane - o >= hl) v = fmax(v, t);
        }
        return v;
    }
};

__device__ __forceinline__ Seg make_seg(uint32_t l) {
    Seg s;
    s.lane = threadIdx.x & 31;
    const uint32_t lp = __shfl_up_sync(0xffffffffu, l, 1);
    const bool head = (s.lane == 0) || (l != lp);
    const unsigned heads = __ballot_sync(0xffffffffu, head);
    const unsigned upto = (s.lane == 31) ? 0xffffffffu : ((2u << s.lane) - 1u);
    s.hl = 31 - __clz(heads & upto);
    s.tail = (s.lane == 31) || ((heads >> (s.lane + 1)) & 1u);
    return s;
}

// 4 CTAs per SM (64 registers): more loads in flight for the latency-bound scan
template <typename TL, typename TI>
__global__ void __launch_bounds__(kST, 4)
stats_pass1(const TL *__restrict__ lab, const TI *__restrict__ inten, int64_t D, int64_t H,
            int64_t W, int64_t Lcap, Acc1 a, FastDiv fc, FastDiv fh, const uint32_t *__restrict__ d_L) {
    const int64_t L = d_L ? ((int64_t)*d_L < Lcap ? (int64_t)*d_L : Lcap) : Lcap;
    const int lane = threadIdx.x & 31;
    const uint32_t chunks = (uint32_t)((W + 31) / 32);
    const uint32_t tasks = (uint32_t)(D * H) * chunks;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    // kBatch row segments per round: every load is issued before its use
    for (uint32_t t0 = warp; t0 < tasks; t0 += kBatch * nwarps) {
        uint32_t lb[kBatch];
        float vb[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint32_t t = t0 + k * nwarps;
            const uint32_t row = fc.div(t);
            const int64_t x = (int64_t)(t - row * chunks) * 32 + lane;
            const uint32_t l = (t < tasks && x < W) ? lab_of(lab[(int64_t)row * W + x]) : 0u;
            lb[k] = (l > (uint32_t)L) ? 0u : l;
        }
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint32_t t = t0 + k * nwarps;
            const uint32_t row = fc.div(t);
            const int64_t x = (int64_t)(t - row * chunks) * 32 + lane;
            vb[k] = lb[k] ? to_f32(inten[(int64_t)row * W + x]) : 0.0f;
        }
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
        const uint32_t l = lb[k];
        if (__ballot_sync(0xffffffffu, l != 0u) == 0u) continue;
        const uint32_t t = t0 + k * nwarps;
        const uint32_t row = fc.div(t);
        const uint32_t c = t - row * chunks;
        const int64_t x = (int64_t)c * 32 + lane;
        const uint32_t z = fh.div(row), y = row - z * (uint32_t)H;
        const float v = vb[k];
        const Seg s = make_seg(l);
        double ssum, ssx;
        float smin, smax;
        if constexpr (sizeof(TI) <= 2) {
            // 8/16-bit intensities: exact uint32 scans of v and v * lane
            // (at most 32 * 65535 * 31 < 2^32), x = 32 c + lane
            const uint32_t iv = (uint32_t)v;
            const uint32_t su = s.scan_addu(iv);
            const uint32_t sl = s.scan_addu(iv * (uint32_t)lane);
            ssum = (double)su;
            ssx = (double)su * (double)(c * 32u) + (double)sl;
            smin = (float)s.scan_minu(iv);
            smax = (float)s.scan_maxu(iv);
        } else {
            const double dv = (double)v;
            ssum = s.scan_add(dv);
            ssx = s.scan_add(dv * (double)x);
            smin = s.scan_min(l ? v : INFINITY);
            smax = s.scan_max(l ? v : -INFINITY);
        }
        if (s.tail && l) {
            const uint32_t i = l - 1;
            const uint32_t cnt = (uint32_t)(s.lane - s.hl + 1);
            const uint32_t xh = (uint32_t)(c * 32 + s.hl), xt = (uint32_t)x;
            atomicAdd(a.cnt + i, cnt);
            atomicAdd(a.sx + i, (unsigned long long)(xh + xt) * cnt / 2ull);
            atomicAdd(a.sy + i, (unsigned long long)y * cnt);
            atomicAdd(a.sz + i, (unsigned long long)z * cnt);
            atomicAdd(a.sv + i, ssum);
            atomicAdd(a.svx + i, ssx);
            atomicAdd(a.svy + i, ssum * (double)y);
            atomicAdd(a.svz + i, ssum * (double)z);
            atomicMin(a.vmin + i, f2ord(smin));
            atomicMax(a.vmax + i, f2ord(smax));
            atomicMin(a.xmin + i, xh);
            atomicMax(a.xmax + i, xt);
            atomicMin(a.ymin + i, (uint32_t)y);
            atomicMax(a.ymax + i, (uint32_t)y);
            atomicMin(a.zmin + i, (uint32_t)z);
            atomicMax(a.zmax + i, (uint32_t)z);
        }
        }
    }
}

// Row indices of the table (the reference's dict order after label columns).
enum {
    C_BBOX_MIN_X, C_BBOX_MIN_Y, C_BBOX_MIN_Z, C_BBOX_MAX_X, C_BBOX_MAX_Y, C_BBOX_MAX_Z,
    C_BBOX_W, C_BBOX_H, C_BBOX_D, C_MIN_I, C_MAX_I, C_SUM_I, C_AREA, C_MEAN_I,
    C_SUM_IX, C_MASS_X, C_SUM_IY, C_MASS_Y, C_SUM_IZ, C_MASS_Z,
    C_SUM_X, C_CEN_X, C_SUM_Y, C_CEN_Y, C_SUM_Z, C_CEN_Z,
    C_SUM_DC, C_MEAN_DC, C_SUM_DM, C_MEAN_DM, C_STD_I, C_MAX_DC, C_MAX_DM,
    C_RATIO_C, C_RATIO_M, C_NCOLS
};
static_assert(C_NCOLS == CLE_STATS_NCOLS, "table width");

__global__ void stats_final1(Acc1 a, Acc2 b, int64_t L, float *__restrict__ T, const uint32_t *__restrict__ d_L) {
    const int64_t n = live_labels(L, d_L);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const bool any = a.cnt[i] != 0u;
        const float area = (float)a.cnt[i];
        const float sum_i = (float)a.sv[i];
        auto put = [&](int c, float v) { T[(int64_t)c * L + i] = v; };
        const float bx0 = any ? (float)a.xmin[i] : FLT_MAX, bx1 = any ? (float)a.xmax[i] : -FLT_MAX;
        const float by0 = any ? (float)a.ymin[i] : FLT_MAX, by1 = any ? (float)a.ymax[i] : -FLT_MAX;
        const float bz0 = any ? (float)a.zmin[i] : FLT_MAX, bz1 = any ? (float)a.zmax[i] : -FLT_MAX;
        put(C_BBOX_MIN_X, bx0); put(C_BBOX_MIN_Y, by0); put(C_BBOX_MIN_Z, bz0);
        put(C_BBOX_MAX_X, bx1); put(C_BBOX_MAX_Y, by1); put(C_BBOX_MAX_Z, bz1);
        put(C_BBOX_W, __fadd_rn(__fsub_rn(bx1, bx0), 1.0f));
        put(C_BBOX_H, __fadd_rn(__fsub_rn(by1, by0), 1.0f));
        put(C_BBOX_D, __fadd_rn(__fsub_rn(bz1, bz0), 1.0f));
        put(C_MIN_I, any ? ord2f(a.vmin[i]) : FLT_MAX);
        put(C_MAX_I, any ? ord2f(a.vmax[i]) : -FLT_MAX);
        put(C_SUM_I, sum_i);
        put(C_AREA, area);
        const float mean = __fdiv_rn(sum_i, area);
        put(C_MEAN_I, mean);
        const float six = (float)a.svx[i], siy = (float)a.svy[i], siz = (float)a.svz[i];
        const float mxc = __fdiv_rn(six, sum_i), myc = __fdiv_rn(siy, sum_i), mzc = __fdiv_rn(siz, sum_i);
        put(C_SUM_IX, six); put(C_MASS_X, mxc);
        put(C_SUM_IY, siy); put(C_MASS_Y, myc);
        put(C_SUM_IZ, siz); put(C_MASS_Z, mzc);
        const float sx = (float)a.sx[i], sy = (float)a.sy[i], sz = (float)a.sz[i];
        const float cx = __fdiv_rn(sx, area), cy = __fdiv_rn(sy, area), cz = __fdiv_rn(sz, area);
        put(C_SUM_X, sx); put(C_CEN_X, cx);
        put(C_SUM_Y, sy); put(C_CEN_Y, cy);
        put(C_SUM_Z, sz); put(C_CEN_Z, cz);
        b.pc[i] = make_float4(cx, cy, cz, mean);
        b.pm[i] = make_float4(mxc, myc, mzc, area);
    }
}

template <typename TL, typename TI>
__global__ void __launch_bounds__(kST)
stats_pass2(const TL *__restrict__ lab, const TI *__restrict__ inten, int64_t D, int64_t H,
            int64_t W, int64_t Lcap, Acc2 b, FastDiv fc, FastDiv fh, const uint32_t *__restrict__ d_L) {
    const int64_t L = d_L ? ((int64_t)*d_L < Lcap ? (int64_t)*d_L : Lcap) : Lcap;
    const int lane = threadIdx.x & 31;
    const uint32_t chunks = (uint32_t)((W + 31) / 32);
    const uint32_t tasks = (uint32_t)(D * H) * chunks;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    // kBatch row segments per round: every load is issued before its use
    for (uint32_t t0 = warp; t0 < tasks; t0 += kBatch * nwarps) {
        uint32_t lb[kBatch];
        float vb[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint32_t t = t0 + k * nwarps;
            const uint32_t row = fc.div(t);
            const int64_t x = (int64_t)(t - row * chunks) * 32 + lane;
            const uint32_t l = (t < tasks && x < W) ? lab_of(lab[(int64_t)row * W + x]) : 0u;
            lb[k] = (l > (uint32_t)L) ? 0u : l;
        }
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint32_t t = t0 + k * nwarps;
            const uint32_t row = fc.div(t);
            const int64_t x = (int64_t)(t - row * chunks) * 32 + lane;
            vb[k] = lb[k] ? to_f32(inten[(int64_t)row * W + x]) : 0.0f;
        }
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
        const uint32_t l = lb[k];
        if (__ballot_sync(0xffffffffu, l != 0u) == 0u) continue;
        const uint32_t t = t0 + k * nwarps;
        const uint32_t row = fc.div(t);
        const uint32_t c = t - row * chunks;
        const int64_t x = (int64_t)c * 32 + lane;
        const uint32_t z = fh.div(row), y = row - z * (uint32_t)H;
        // distances in float32 (relative error a few 1e-7), their sums and the
        // squared deviations in float64; the squared deviations are divided
        // by the area once per label
        float dc = 0.0f, dm = 0.0f;
        double sq = 0.0;
        if (l) {
            const uint32_t i = l - 1;
            const float4 pc = b.pc[i], pm = b.pm[i];
            const float xf = (float)x, yf = (float)y, zf = (float)z;
            const float ex = xf - pc.x, ey = yf - pc.y, ez = zf - pc.z;
            const float fx = xf - pm.x, fy = yf - pm.y, fz = zf - pm.z;
            dc = sqrtf(ex * ex + ey * ey + ez * ez);
            dm = sqrtf(fx * fx + fy * fy + fz * fz);
            const double dv = (double)vb[k] - (double)pc.w;
            sq = dv * dv;
        }
        const Seg s = make_seg(l);
        const double sdc = s.scan_add((double)dc);
        const double sdm = s.scan_add((double)dm);
        const double ssq = s.scan_add(sq);
        const float mdc = s.scan_max(dc);
        const float mdm = s.scan_max(dm);
        if (s.tail && l) {
            const uint32_t i = l - 1;
            atomicAdd(b.sdc + i, sdc);
            atomicAdd(b.sdm + i, sdm);
            atomicAdd(b.ssq + i, ssq);
            atomicMax(b.mdc + i, (unsigned long long)__double_as_longlong((double)mdc));
            atomicMax(b.mdm + i, (unsigned long long)__double_as_longlong((double)mdm));
        }
        }
    }
}

__global__ void stats_final2(Acc2 b, int64_t L, float *__restrict__ T, const uint32_t *__restrict__ d_L) {
    const int64_t n = live_labels(L, d_L);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        auto put = [&](int c, float v) { T[(int64_t)c * L + i] = v; };
        const float area = b.pm[i].w;
        const float sdc = (float)b.sdc[i], sdm = (float)b.sdm[i];
        const float mdc = __fdiv_rn(sdc, area), mdm = __fdiv_rn(sdm, area);
        const float xdc = (float)__longlong_as_double((long long)b.mdc[i]);
        const float xdm = (float)__longlong_as_double((long long)b.mdm[i]);
        put(C_SUM_DC, sdc); put(C_MEAN_DC, mdc);
        put(C_SUM_DM, sdm); put(C_MEAN_DM, mdm);
        // sum of squared deviations / area (0 for a label absent from the image)
        put(C_STD_I, (float)sqrt(area > 0.0f ? b.ssq[i] / (double)area : b.ssq[i]));
        put(C_MAX_DC, xdc); put(C_MAX_DM, xdm);
        put(C_RATIO_C, __fdiv_rn(xdc, mdc));
        put(C_RATIO_M, __fdiv_rn(xdm, mdm));
    }
}

template <typename TL, typename TI>
int stats_typed(const Img &inten, const Img &lab, int64_t L, float *T, const Acc1 &a,
                const Acc2 &b, cudaStream_t st, const uint32_t *d_L) {
    const int64_t tasks = lab.D * lab.H * ((lab.W + 31) / 32);
    const int blocks = launch_blocks(tasks * 32, kST, 8);
    const FastDiv fc((uint32_t)((lab.W + 31) / 32)), fh((uint32_t)lab.H);
    stage_mark(8, st);
    stats_pass1<TL, TI><<<blocks, kST, 0, st>>>((const TL *)lab.data, (const TI *)inten.data, lab.D,
                                                lab.H, lab.W, L, a, fc, fh, d_L);
    stage_mark(9, st);
    stats_final1<<<launch_blocks(L, 256), 256, 0, st>>>(a, b, L, T, d_L);
    stage_mark(10, st);
    stats_pass2<TL, TI><<<blocks, kST, 0, st>>>((const TL *)lab.data, (const TI *)inten.data, lab.D,
                                                lab.H, lab.W, L, b, fc, fh, d_L);
    stage_mark(11, st);
    stats_final2<<<launch_blocks(L, 256), 256, 0, st>>>(b, L, T, d_L);
    stage_mark(12, st);
    CLE_LAUNCH_CHECK_N("statistics", 4);
    return CLE_OK;
}

template <typename TL>
int stats_i(const Img &inten, const Img &lab, int64_t L, float *T, const Acc1 &a, const Acc2 &b,
            cudaStream_t st, const uint32_t *d_L) {
    switch (inten.dtype) {
        case CLE_F32: return stats_typed<TL, float>(inten, lab, L, T, a, b, st, d_L);
        case CLE_U16: return stats_typed<TL, uint16_t>(inten, lab, L, T, a, b, st, d_L);
        case CLE_U8: return stats_typed<TL, uint8_t>(inten, lab, L, T, a, b, st, d_L);
        case CLE_U32: return stats_typed<TL, uint32_t>(inten, lab, L, T, a, b, st, d_L);
        default: set_error("statistics: unsupported intensity dtype %d", inten.dtype); return CLE_ERR_DTYPE;
    }
}

}  // namespace

size_t stats_workspace_bytes(const Img &, int64_t L) {
    Arena a(nullptr, 0);
    take_acc1(a, L < 1 ? 1 : L);
    take_acc2(a, L < 1 ? 1 : L);
    return a.off;
}

int statistics(const Img &inten, const Img &lab, int64_t L, float *T, Arena &ws, cudaStream_t st,
               const uint32_t *d_L) {
    CLE_TRY(same_shape(inten, lab, "intensity_image", "label_image"));
    if (L < 0 || L > 0x7FFFFFFF) { set_error("statistics: bad label count %lld", (long long)L); return CLE_ERR_ARG; }
    if (L == 0) return CLE_OK;
    Acc1 a = take_acc1(ws, L);
    Acc2 b = take_acc2(ws, L);
    if (!ws.ok()) { set_error("statistics: workspace too small"); return CLE_ERR_WORKSPACE; }
    stats_init<<<launch_blocks(L, 256), 256, 0, st>>>(a, b, L, d_L);
    CLE_LAUNCH_CHECK("statistics init");
    switch (lab.dtype) {
        case CLE_U32: return stats_i<uint32_t>(inten, lab, L, T, a, b, st, d_L);
        case CLE_F32: return stats_i<float>(inten, lab, L, T, a, b, st, d_L);
        case CLE_U16: return stats_i<uint16_t>(inten, lab, L, T, a, b, st, d_L);
        case CLE_U8: return stats_i<uint8_t>(inten, lab, L, T, a, b, st, d_L);
        default: set_error("statistics: unsupported label dtype %d", lab.dtype); return CLE_ERR_DTYPE;
    }
}

}  // namespace cle
