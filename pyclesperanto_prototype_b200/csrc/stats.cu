// stats.cu -- statistics_of_labelled_pixels
// (_tier9/_statistics_of_labelled_pixels.py:7-293, kernels
// _tier9/statistics_per_label_x.cl:1-146, _tier9/standard_deviation_per_label_x.cl:1-96).
//
// Sorted-segment reductions: the labelled voxels are first put in label order
// (a count per label, an exclusive scan into offsets, a scatter of voxel
// indices), then warps sweep the sorted index array, each keeping per-lane
// accumulators of the label at hand and adding them to the per-label
// accumulators once the label changes -- a few atomics per label instead of
// one set per row run.  Two sweeps, as in the reference (the second needs the
// per-label centroid, mass centre and mean).  Coordinates and 8/16-bit
// intensities are summed in exact 64-bit integers, other intensities in
// float64; min / max through order-preserving integer atomics.  The finalise
// kernels apply the reference's float32 column arithmetic and its sentinels
// for labels absent from the image (min FLT_MAX, max -FLT_MAX, sums 0,
// 0/0 = NaN).
#include <cfloat>

#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

constexpr int kST = 256;
constexpr int kChunk = 4096;   // sorted positions per warp in a sweep
constexpr int kScanTile = 4096;  // labels per block of the offset scan

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

// Label-sorted voxel indices and the per-label counts / offsets / cursors.
struct Sorted {
    uint32_t *cnt, *off, *cursor, *tsum, *sorted;
};

Sorted take_sorted(Arena &a, const Img &labels, int64_t L) {
    Sorted s;
    s.cnt = a.take<uint32_t>(L);
    s.off = a.take<uint32_t>(L + 1);
    s.cursor = a.take<uint32_t>(L);
    s.tsum = a.take<uint32_t>((L + kScanTile - 1) / kScanTile + 1);
    s.sorted = a.take<uint32_t>(labels.n());
    return s;
}

__device__ __forceinline__ void m2xyz_fd(const FastDiv &fW, const FastDiv &fH, uint32_t m, uint32_t &x,
                                         uint32_t &y, uint32_t &z) {
    const uint32_t r = fW.div(m);
    x = m - r * fW.d;
    z = fH.div(r);
    y = r - z * fH.d;
}

// Run of equal labels along x inside a warp's 32 voxels: head lane, and
// whether this lane ends its run.
struct Run {
    int head;
    bool tail;
};

__device__ __forceinline__ Run make_run(uint32_t l) {
    const int lane = threadIdx.x & 31;
    const uint32_t lp = __shfl_up_sync(0xffffffffu, l, 1);
    const bool hd = (lane == 0) || (l != lp);
    const unsigned heads = __ballot_sync(0xffffffffu, hd);
    const unsigned upto = (lane == 31) ? 0xffffffffu : ((2u << lane) - 1u);
    Run r;
    r.head = 31 - __clz(heads & upto);
    r.tail = (lane == 31) || ((heads >> (lane + 1)) & 1u);
    return r;
}

// Label of one voxel, 0 for background and for labels above the live count.
template <typename TL>
__device__ __forceinline__ uint32_t live_label(const TL *lab, int64_t m, int64_t L) {
    const uint32_t l = lab_of(lab[m]);
    return (l > (uint32_t)L) ? 0u : l;
}

constexpr int kBatch = 4;   // row segments per warp round (loads in flight)
constexpr int kSweepBlocks = 4;   // 32-entry blocks per sweep round (loads in flight)

// Pass A: voxels per label (one atomic per row run).  A warp takes 32 voxels
// of one row at a time, kBatch row segments per round with every load issued
// before its use.
template <typename TL>
__global__ void __launch_bounds__(kST)
count_kernel(const TL *__restrict__ lab, uint32_t W, uint32_t tasks, FastDiv fc, int64_t Lcap,
             const uint32_t *__restrict__ d_L, uint32_t *__restrict__ cnt) {
    const int64_t L = live_labels(Lcap, d_L);
    const int lane = threadIdx.x & 31;
    const uint32_t chunks = fc.d;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t0 = warp; t0 < tasks; t0 += kBatch * nwarps) {
        uint32_t lb[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint32_t t = t0 + (uint32_t)k * nwarps;
            const uint32_t row = fc.div(t), x = (t - row * chunks) * 32u + (uint32_t)lane;
            lb[k] = (t < tasks && x < W) ? live_label(lab, (int64_t)row * W + x, L) : 0u;
        }
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint32_t l = lb[k];
            if (__ballot_sync(0xffffffffu, l != 0u) == 0u) continue;
            const Run r = make_run(l);
            if (r.tail && l) atomicAdd(cnt + (l - 1), (uint32_t)(lane - r.head + 1));
        }
    }
}

// Runs over 128 voxels of a row, 4 per lane (uint32 labels, rows of a multiple
// of 4, 16-byte aligned): position p = 4 lane + k.  Per lane the 4-bit masks
// of run heads and run tails, and for each position the position of its run's
// head (the last head at or before it, in this lane or, through the nearest
// earlier lane that holds a head, before it; position 0 is always a head).
struct Run4 {
    uint32_t hmask, tmask;
    int hpos[4];
};

__device__ __forceinline__ Run4 make_run4(const uint32_t (&l)[4]) {
    const int lane = threadIdx.x & 31;
    const uint32_t prev = __shfl_up_sync(0xffffffffu, l[3], 1);
    const uint32_t next = __shfl_down_sync(0xffffffffu, l[0], 1);
    Run4 r;
    r.hmask = ((lane == 0 || l[0] != prev) ? 1u : 0u) | (l[1] != l[0] ? 2u : 0u) | (l[2] != l[1] ? 4u : 0u) |
              (l[3] != l[2] ? 8u : 0u);
    r.tmask = (r.hmask >> 1) | ((lane == 31 || l[3] != next) ? 8u : 0u);
    const unsigned has = __ballot_sync(0xffffffffu, r.hmask != 0u);
    const int last = r.hmask ? 4 * lane + 31 - __clz(r.hmask) : 0;
    const int j = lane ? 31 - __clz(has & ((1u << lane) - 1u)) : 0;
    const int before = __shfl_sync(0xffffffffu, last, j);   // lane 0: unused (its bit 0 is a head)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t upto = r.hmask & ((2u << k) - 1u);
        r.hpos[k] = upto ? 4 * lane + 31 - __clz(upto) : before;
    }
    return r;
}

// Four labels (uint32 or float32) of one 16-byte aligned group, 0 above L.
template <typename TL>
__device__ __forceinline__ void live4(const TL *lab, int64_t m, int64_t L, uint32_t (&l)[4]) {
    static_assert(sizeof(TL) == 4, "4-byte labels");
    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(lab + m));
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        uint32_t x;
        if constexpr (std::is_same<TL, float>::value) x = lab_of(__uint_as_float(w[k]));
        else x = w[k];
        l[k] = x > (uint32_t)L ? 0u : x;
    }
}

// Pass A, uint32 labels in 128-voxel row segments: one atomic per run.
template <typename TL>
__global__ void __launch_bounds__(kST)
count4_kernel(const TL *__restrict__ lab, uint32_t W, uint32_t tasks, FastDiv fs, int64_t Lcap,
              const uint32_t *__restrict__ d_L, uint32_t *__restrict__ cnt) {
    const int64_t L = live_labels(Lcap, d_L);
    const int lane = threadIdx.x & 31;
    const uint32_t segs = fs.d;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t0 = warp; t0 < tasks; t0 += kBatch * nwarps) {
        uint32_t lb[kBatch][4];
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
            const uint32_t t = t0 + (uint32_t)b * nwarps;
            const uint32_t row = fs.div(t), x = (t - row * segs) * 128u + 4u * (uint32_t)lane;
            if (t < tasks && x < W) live4(lab, (int64_t)row * W + x, L, lb[b]);
            else lb[b][0] = lb[b][1] = lb[b][2] = lb[b][3] = 0u;
        }
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
            const uint32_t(&l)[4] = lb[b];
            if (__ballot_sync(0xffffffffu, (l[0] | l[1] | l[2] | l[3]) != 0u) == 0u) continue;
            const Run4 r = make_run4(l);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (((r.tmask >> k) & 1u) && l[k]) atomicAdd(cnt + (l[k] - 1), (uint32_t)(4 * lane + k - r.hpos[k] + 1));
        }
    }
}

// Pass B, the same segments: each run reserves its place with one atomic (at
// its tail) and every voxel writes its index at the run's base + its offset
// from the head; the base of a run whose tail lies in a later lane comes from
// the nearest later lane holding a tail (its first tail).
template <typename TL>
__global__ void __launch_bounds__(kST)
scatter4_kernel(const TL *__restrict__ lab, uint32_t W, uint32_t tasks, FastDiv fs, int64_t Lcap,
                const uint32_t *__restrict__ d_L, uint32_t *__restrict__ cursor, uint32_t *__restrict__ sorted) {
    const int64_t L = live_labels(Lcap, d_L);
    const int lane = threadIdx.x & 31;
    const uint32_t segs = fs.d;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t0 = warp; t0 < tasks; t0 += kBatch * nwarps) {
        uint32_t lb[kBatch][4], mb[kBatch];
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
            const uint32_t t = t0 + (uint32_t)b * nwarps;
            const uint32_t row = fs.div(t), x = (t - row * segs) * 128u + 4u * (uint32_t)lane;
            mb[b] = row * W + x;
            if (t < tasks && x < W) live4(lab, (int64_t)mb[b], L, lb[b]);
            else lb[b][0] = lb[b][1] = lb[b][2] = lb[b][3] = 0u;
        }
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
            const uint32_t(&l)[4] = lb[b];
            if (__ballot_sync(0xffffffffu, (l[0] | l[1] | l[2] | l[3]) != 0u) == 0u) continue;
            const Run4 r = make_run4(l);
            uint32_t pos[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                pos[k] = 0u;
                if (((r.tmask >> k) & 1u) && l[k])
                    pos[k] = atomicAdd(cursor + (l[k] - 1), (uint32_t)(4 * lane + k - r.hpos[k] + 1));
            }
            // base of the run holding this lane's first voxel when its tail is later
            const uint32_t first = r.tmask & (0u - r.tmask);   // lowest tail bit
            const uint32_t pfirst = first == 1u ? pos[0] : first == 2u ? pos[1] : first == 4u ? pos[2] : pos[3];
            const unsigned hasT = __ballot_sync(0xffffffffu, r.tmask != 0u);
            const unsigned later = hasT & ~((2u << lane) - 1u);   // lane 31 always holds a tail
            const int j = later ? __ffs(later) - 1 : lane;
            const uint32_t after = __shfl_sync(0xffffffffu, pfirst, j);
            // walk the lane's voxels from the last: the base of the run ending at or after k
            uint32_t base = after;
#pragma unroll
            for (int k = 3; k >= 0; --k) {
                if ((r.tmask >> k) & 1u) base = pos[k];
                if (l[k]) sorted[base + (uint32_t)(4 * lane + k - r.hpos[k])] = mb[b] + (uint32_t)k;
            }
        }
    }
}

// Offsets: exclusive scan of the counts (tiles of kScanTile labels: tile sums,
// a one-CTA scan of the tile sums, then each tile's scan); cursor = offset;
// off[L] = total.
__global__ void __launch_bounds__(kST)
tile_sum_kernel(const uint32_t *__restrict__ cnt, int64_t Lcap, const uint32_t *__restrict__ d_L,
                uint32_t *__restrict__ tsum) {
    __shared__ uint32_t red[kST / 32];
    const int64_t L = live_labels(Lcap, d_L);
    const int64_t b0 = (int64_t)blockIdx.x * kScanTile;
    uint32_t s = 0;
    for (int64_t i = b0 + threadIdx.x; i < min(b0 + kScanTile, L); i += kST) s += cnt[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kST / 32; ++w) t += red[w];
        tsum[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(1024)
tile_scan_kernel(uint32_t *__restrict__ tsum, int64_t ntiles) {
    __shared__ uint32_t s_w[32];
    __shared__ uint32_t s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t base = 0; base < ntiles; base += 1024) {
        const int64_t i = base + threadIdx.x;
        const uint32_t v = i < ntiles ? tsum[i] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_w[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = s_w[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            s_w[lane] = w;
        }
        __syncthreads();
        const uint32_t excl = s_carry + (warp ? s_w[warp - 1] : 0u) + x - v;
        if (i < ntiles) tsum[i] = excl;
        __syncthreads();
        if (threadIdx.x == 0) s_carry += s_w[31];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kST)
offset_kernel(const uint32_t *__restrict__ cnt, int64_t Lcap, const uint32_t *__restrict__ d_L,
              const uint32_t *__restrict__ tsum, uint32_t *__restrict__ off, uint32_t *__restrict__ cursor) {
    __shared__ uint32_t s_w[kST / 32];
    __shared__ uint32_t s_carry;
    const int64_t L = live_labels(Lcap, d_L);
    const int64_t b0 = (int64_t)blockIdx.x * kScanTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = tsum[blockIdx.x];
    if (blockIdx.x == 0 && threadIdx.x == 0 && L == 0) off[0] = 0u;   // no live label: empty sweep
    __syncthreads();
    for (int64_t base = b0; base < min(b0 + kScanTile, L); base += kST) {
        const int64_t i = base + threadIdx.x;
        const uint32_t v = i < L ? cnt[i] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_w[warp] = x;
        __syncthreads();
        uint32_t before = s_carry;
        for (int w = 0; w < warp; ++w) before += s_w[w];
        const uint32_t excl = before + x - v;
        if (i < L) {
            off[i] = excl;
            cursor[i] = excl;
            if (i == L - 1) off[L] = excl + v;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t t = 0;
            for (int w = 0; w < kST / 32; ++w) t += s_w[w];
            s_carry += t;
        }
        __syncthreads();
    }
}

// Pass B: each run reserves its place in its label's range (one atomic per
// run) and its lanes write their voxel indices there.
template <typename TL>
__global__ void __launch_bounds__(kST)
scatter_kernel(const TL *__restrict__ lab, uint32_t W, uint32_t tasks, FastDiv fc, int64_t Lcap,
               const uint32_t *__restrict__ d_L, uint32_t *__restrict__ cursor, uint32_t *__restrict__ sorted) {
    const int64_t L = live_labels(Lcap, d_L);
    const int lane = threadIdx.x & 31;
    const uint32_t chunks = fc.d;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t0 = warp; t0 < tasks; t0 += kBatch * nwarps) {
        uint32_t lb[kBatch], mb[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint32_t t = t0 + (uint32_t)k * nwarps;
            const uint32_t row = fc.div(t), x = (t - row * chunks) * 32u + (uint32_t)lane;
            mb[k] = row * W + x;
            lb[k] = (t < tasks && x < W) ? live_label(lab, (int64_t)mb[k], L) : 0u;
        }
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint32_t l = lb[k];
            if (__ballot_sync(0xffffffffu, l != 0u) == 0u) continue;
            const Run r = make_run(l);
            uint32_t pos = 0;
            if (r.tail && l) pos = atomicAdd(cursor + (l - 1), (uint32_t)(lane - r.head + 1));
            // the run's tail lane holds its base: the first tail at or after this lane
            const unsigned tails = __ballot_sync(0xffffffffu, r.tail);
            const int tl = __ffs(tails >> lane) - 1 + lane;
            const uint32_t base = __shfl_sync(0xffffffffu, pos, tl);
            if (l) sorted[base + (uint32_t)(lane - r.head)] = mb[k];
        }
    }
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Per-lane accumulators of pass 1 for the label at hand.
template <bool INT>
struct Lane1 {
    uint32_t cnt;
    unsigned long long sx, sy, sz;
    unsigned long long iv, ivx, ivy, ivz;   // 8/16-bit intensities: exact
    double dv, dvx, dvy, dvz;               // others
    int vmin, vmax;
    uint32_t x0, x1, y0, y1, z0, z1;
    __device__ __forceinline__ void reset() {
        cnt = 0;
        sx = sy = sz = 0ull;
        iv = ivx = ivy = ivz = 0ull;
        dv = dvx = dvy = dvz = 0.0;
        vmin = 0x7FFFFFFF;
        vmax = (int)0x80000000;
        x0 = y0 = z0 = 0xFFFFFFFFu;
        x1 = y1 = z1 = 0u;
    }
    __device__ __forceinline__ void add(uint32_t x, uint32_t y, uint32_t z, float v) {
        ++cnt;
        sx += x; sy += y; sz += z;
        if constexpr (INT) {
            const unsigned long long u = (unsigned long long)v;
            iv += u; ivx += u * x; ivy += u * y; ivz += u * z;
        } else {
            const double d = (double)v;
            dv += d; dvx += d * (double)x; dvy += d * (double)y; dvz += d * (double)z;
        }
        const int o = f2ord(v);
        vmin = min(vmin, o); vmax = max(vmax, o);
        x0 = min(x0, x); x1 = max(x1, x);
        y0 = min(y0, y); y1 = max(y1, y);
        z0 = min(z0, z); z1 = max(z1, z);
    }
    // warp-wide: the label's totals over the lanes, added by lane 0
    __device__ __forceinline__ void flush(const Acc1 &a, uint32_t l) {
        const uint32_t c = warp_sum(cnt);
        const unsigned long long Sx = warp_sum(sx), Sy = warp_sum(sy), Sz = warp_sum(sz);
        double Sv, Svx, Svy, Svz;
        if constexpr (INT) {
            // exact: per-label totals stay far below 2^53
            Sv = (double)warp_sum(iv); Svx = (double)warp_sum(ivx);
            Svy = (double)warp_sum(ivy); Svz = (double)warp_sum(ivz);
        } else {
            Sv = warp_sum(dv); Svx = warp_sum(dvx); Svy = warp_sum(dvy); Svz = warp_sum(dvz);
        }
        const int mn = warp_min(vmin), mx = warp_max(vmax);
        const uint32_t X0 = warp_min(x0), X1 = warp_max(x1), Y0 = warp_min(y0), Y1 = warp_max(y1);
        const uint32_t Z0 = warp_min(z0), Z1 = warp_max(z1);
        if ((threadIdx.x & 31) == 0 && c) {
            const uint32_t i = l - 1;
            atomicAdd(a.cnt + i, c);
            atomicAdd(a.sx + i, Sx); atomicAdd(a.sy + i, Sy); atomicAdd(a.sz + i, Sz);
            atomicAdd(a.sv + i, Sv); atomicAdd(a.svx + i, Svx); atomicAdd(a.svy + i, Svy); atomicAdd(a.svz + i, Svz);
            atomicMin(a.vmin + i, mn); atomicMax(a.vmax + i, mx);
            atomicMin(a.xmin + i, X0); atomicMax(a.xmax + i, X1);
            atomicMin(a.ymin + i, Y0); atomicMax(a.ymax + i, Y1);
            atomicMin(a.zmin + i, Z0); atomicMax(a.zmax + i, Z1);
        }
        reset();
    }
};

// Per-lane accumulators of pass 2 for the label at hand.
struct Lane2 {
    double sdc, sdm, ssq;
    float mdc, mdm;
    __device__ __forceinline__ void reset() { sdc = sdm = ssq = 0.0; mdc = mdm = 0.0f; }
    __device__ __forceinline__ void flush(const Acc2 &b, uint32_t l) {
        const double Sdc = warp_sum(sdc), Sdm = warp_sum(sdm), Ssq = warp_sum(ssq);
        const float Mdc = warp_max(mdc), Mdm = warp_max(mdm);
        if ((threadIdx.x & 31) == 0) {
            const uint32_t i = l - 1;
            atomicAdd(b.sdc + i, Sdc);
            atomicAdd(b.sdm + i, Sdm);
            atomicAdd(b.ssq + i, Ssq);
            atomicMax(b.mdc + i, (unsigned long long)__double_as_longlong((double)Mdc));
            atomicMax(b.mdm + i, (unsigned long long)__double_as_longlong((double)Mdm));
        }
        reset();
    }
};

// Sweeps: each warp takes kChunk consecutive positions of the sorted array
// (labels in order), 32 per round; lanes add their voxels to the accumulators
// of the warp's current label, which are flushed when the label changes.
template <int PASS, typename TL, typename TI>
__global__ void __launch_bounds__(kST)
sweep_kernel(const TL *__restrict__ lab, const TI *__restrict__ inten, const uint32_t *__restrict__ sorted,
             const uint32_t *__restrict__ off, int64_t Lcap, const uint32_t *__restrict__ d_L, FastDiv fW,
             FastDiv fH, Acc1 a, Acc2 b) {
    constexpr bool INT = sizeof(TI) <= 2 && !std::is_floating_point<TI>::value;
    // float64 accumulators (pass 1 of 32-bit intensities) leave room for 2 blocks
    constexpr int NB = (PASS == 1 && !INT) ? 2 : kSweepBlocks;
    const int64_t L = live_labels(Lcap, d_L);
    const uint32_t total = off[L];
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    Lane1<INT> A;
    Lane2 B;
    A.reset();
    B.reset();
    for (uint32_t c0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * (uint32_t)kChunk; c0 < total;
         c0 += nwarps * (uint32_t)kChunk) {
        const uint32_t c1 = min(total, c0 + (uint32_t)kChunk);
        uint32_t cur = 0;
        float4 pc = make_float4(0.f, 0.f, 0.f, 0.f), pm = pc;
        // label of the entries seen last and the end of its range: a block of
        // 32 entries inside that range takes the label without reading it
        uint32_t lc = 0, lend = 0;
        // NB blocks of 32 entries per round: their index loads, then
        // their intensity gathers, are all in flight before any is used
        for (uint32_t q = c0; q < c1; q += 32u * NB) {
            uint32_t mk[NB];
            TI ik[NB];
#pragma unroll
            for (int k = 0; k < NB; ++k) {
                const uint32_t p = q + 32u * k + lane;
                mk[k] = p < c1 ? sorted[p] : 0u;
            }
#pragma unroll
            for (int k = 0; k < NB; ++k) {
                const uint32_t p = q + 32u * k + lane;
                ik[k] = p < c1 ? inten[mk[k]] : TI(0);
            }
#pragma unroll
            for (int k = 0; k < NB; ++k) {
            const uint32_t pb = q + 32u * k;
            if (pb >= c1) break;   // warp-uniform
            const uint32_t p = pb + lane;
            const bool valid = p < c1;
            const uint32_t m = mk[k];
            const uint32_t plast = min(pb + 31u, c1 - 1u);
            uint32_t l;
            if (plast < lend) {
                l = valid ? lc : 0xFFFFFFFFu;
            } else {
                l = valid ? lab_of(lab[m]) : 0xFFFFFFFFu;
                lc = __shfl_sync(0xffffffffu, l, (int)(plast - pb));
                lend = off[lc];
            }
            const float v = valid ? to_f32(ik[k]) : 0.0f;
            uint32_t x = 0, y = 0, z = 0;
            if (valid) m2xyz_fd(fW, fH, m, x, y, z);
            unsigned todo = __ballot_sync(0xffffffffu, valid);
            while (todo) {
                const uint32_t g = __shfl_sync(0xffffffffu, l, __ffs(todo) - 1);
                if (g != cur) {
                    if (cur) {
                        if constexpr (PASS == 1) A.flush(a, cur);
                        else B.flush(b, cur);
                    }
                    cur = g;
                    if constexpr (PASS == 2) { pc = b.pc[cur - 1]; pm = b.pm[cur - 1]; }
                }
                const bool mine = valid && l == g;
                if (mine) {
                    if constexpr (PASS == 1) {
                        A.add(x, y, z, v);
                    } else {
                        // distances in float32 (relative error a few 1e-7), their
                        // sums and the squared deviations in float64; the squared
                        // deviations are divided by the area once per label
                        const float xf = (float)x, yf = (float)y, zf = (float)z;
                        const float ex = xf - pc.x, ey = yf - pc.y, ez = zf - pc.z;
                        const float fx = xf - pm.x, fy = yf - pm.y, fz = zf - pm.z;
                        const float dc = sqrtf(ex * ex + ey * ey + ez * ez);
                        const float dm = sqrtf(fx * fx + fy * fy + fz * fz);
                        const double dv = (double)v - (double)pc.w;
                        B.sdc += (double)dc;
                        B.sdm += (double)dm;
                        B.ssq += dv * dv;
                        B.mdc = fmaxf(B.mdc, dc);
                        B.mdm = fmaxf(B.mdm, dm);
                    }
                }
                todo &= ~__ballot_sync(0xffffffffu, mine);
            }
            }
        }
        if (cur) {
            if constexpr (PASS == 1) A.flush(a, cur);
            else B.flush(b, cur);
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

// The label type of the 128-voxel row-segment passes: the type itself for
// 4-byte labels (uint32, float32); others take the 32-voxel passes.
template <typename TL>
using TL4 = typename std::conditional<sizeof(TL) == 4, TL, uint32_t>::type;

// ---- centroids of labels (the point list, no second pass) ------------------
// Per row run of label l (1..n): the voxel count and the exact 64-bit sums of
// its x, y and z (x from the run's first voxel in closed form), added once per
// run; then centroid = float32(sum) / float32(count), the division the
// statistics table uses for centroid_x/y/z.
template <typename TL>
__global__ void __launch_bounds__(kST)
centroid_sums_kernel(const TL *__restrict__ lab, uint32_t W, uint32_t H, uint32_t tasks, FastDiv fc,
                     int64_t n, uint32_t *__restrict__ cnt, unsigned long long *__restrict__ sums) {
    const int lane = threadIdx.x & 31;
    const uint32_t chunks = fc.d;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t0 = warp; t0 < tasks; t0 += kBatch * nwarps) {
        uint32_t lb[kBatch], rb[kBatch], xb[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint32_t t = t0 + (uint32_t)k * nwarps;
            const uint32_t row = fc.div(t), x = (t - row * chunks) * 32u + (uint32_t)lane;
            rb[k] = row;
            xb[k] = x;
            lb[k] = (t < tasks && x < W) ? live_label(lab, (int64_t)row * W + x, n) : 0u;
        }
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint32_t l = lb[k];
            if (__ballot_sync(0xffffffffu, l != 0u) == 0u) continue;
            const Run r = make_run(l);
            if (r.tail && l) {
                const unsigned long long len = (unsigned long long)(lane - r.head + 1);
                const unsigned long long x0 = xb[k] - (uint32_t)(lane - r.head);
                const uint32_t y = rb[k] % H, z = rb[k] / H;
                const int64_t i = (int64_t)l - 1;
                atomicAdd(cnt + i, (uint32_t)len);
                atomicAdd(sums + 3 * i, len * x0 + len * (len - 1) / 2);
                atomicAdd(sums + 3 * i + 1, len * y);
                atomicAdd(sums + 3 * i + 2, len * z);
            }
        }
    }
}

__global__ void centroid_final_kernel(const uint32_t *__restrict__ cnt, const unsigned long long *__restrict__ sums,
                                      int64_t n, int dims, float *__restrict__ pts) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float area = (float)cnt[i];
        for (int d = 0; d < dims; ++d) pts[d * n + i] = __fdiv_rn((float)sums[3 * i + d], area);
    }
}

template <typename TL, typename TI>
int stats_typed(const Img &inten, const Img &lab, int64_t L, float *T, const Acc1 &a, const Acc2 &b,
                const Sorted &so, cudaStream_t st, const uint32_t *d_L) {
    const int64_t rows = lab.D * lab.H;
    const int64_t tasks = rows * ((lab.W + 31) / 32);
    const int blocks = launch_blocks(tasks * 32, kST, 8);
    const int64_t ntiles = (L + kScanTile - 1) / kScanTile;
    // sweeps: enough warps for every chunk of the worst case (all voxels labelled)
    const int sweep_blocks = launch_blocks((lab.n() + kChunk - 1) / kChunk * 32, kST, 8);
    const FastDiv fW((uint32_t)lab.W), fH((uint32_t)lab.H);
    stage_mark(8, st);
    const FastDiv fc((uint32_t)((lab.W + 31) / 32));
    // uint32 rows of a multiple of 4 voxels on a 16-byte boundary: 128-voxel
    // segments with 128-bit loads
    const bool seg4 = sizeof(TL) == 4 && lab.W % 4 == 0 && (reinterpret_cast<uintptr_t>(lab.data) & 15) == 0;
    const int64_t tasks4 = rows * ((lab.W + 127) / 128);
    const FastDiv fs((uint32_t)((lab.W + 127) / 128));
    const int blocks4 = launch_blocks(tasks4 * 32, kST, 8);
    if (seg4) count4_kernel<TL4<TL>><<<blocks4, kST, 0, st>>>((const TL4<TL> *)lab.data, (uint32_t)lab.W, (uint32_t)tasks4, fs, L, d_L, so.cnt);
    else count_kernel<TL><<<blocks, kST, 0, st>>>((const TL *)lab.data, (uint32_t)lab.W, (uint32_t)tasks, fc, L, d_L, so.cnt);
    tile_sum_kernel<<<(unsigned)ntiles, kST, 0, st>>>(so.cnt, L, d_L, so.tsum);
    tile_scan_kernel<<<1, 1024, 0, st>>>(so.tsum, ntiles);
    offset_kernel<<<(unsigned)ntiles, kST, 0, st>>>(so.cnt, L, d_L, so.tsum, so.off, so.cursor);
    if (seg4) scatter4_kernel<TL4<TL>><<<blocks4, kST, 0, st>>>((const TL4<TL> *)lab.data, (uint32_t)lab.W, (uint32_t)tasks4, fs, L, d_L,
                                                        so.cursor, so.sorted);
    else scatter_kernel<TL><<<blocks, kST, 0, st>>>((const TL *)lab.data, (uint32_t)lab.W, (uint32_t)tasks, fc, L, d_L,
                                                    so.cursor, so.sorted);
    sweep_kernel<1, TL, TI><<<sweep_blocks, kST, 0, st>>>((const TL *)lab.data, (const TI *)inten.data, so.sorted,
                                                          so.off, L, d_L, fW, fH, a, b);
    stage_mark(9, st);
    stats_final1<<<launch_blocks(L, 256), 256, 0, st>>>(a, b, L, T, d_L);
    stage_mark(10, st);
    sweep_kernel<2, TL, TI><<<sweep_blocks, kST, 0, st>>>((const TL *)lab.data, (const TI *)inten.data, so.sorted,
                                                          so.off, L, d_L, fW, fH, a, b);
    stage_mark(11, st);
    stats_final2<<<launch_blocks(L, 256), 256, 0, st>>>(b, L, T, d_L);
    stage_mark(12, st);
    CLE_LAUNCH_CHECK_N("statistics", 9);
    return CLE_OK;
}

template <typename TL>
int stats_i(const Img &inten, const Img &lab, int64_t L, float *T, const Acc1 &a, const Acc2 &b,
            const Sorted &so, cudaStream_t st, const uint32_t *d_L) {
    switch (inten.dtype) {
        case CLE_F32: return stats_typed<TL, float>(inten, lab, L, T, a, b, so, st, d_L);
        case CLE_U16: return stats_typed<TL, uint16_t>(inten, lab, L, T, a, b, so, st, d_L);
        case CLE_U8: return stats_typed<TL, uint8_t>(inten, lab, L, T, a, b, so, st, d_L);
        case CLE_U32: return stats_typed<TL, uint32_t>(inten, lab, L, T, a, b, so, st, d_L);
        default: set_error("statistics: unsupported intensity dtype %d", inten.dtype); return CLE_ERR_DTYPE;
    }
}

}  // namespace

size_t stats_workspace_bytes(const Img &labels, int64_t L) {
    Arena a(nullptr, 0);
    take_acc1(a, L < 1 ? 1 : L);
    take_acc2(a, L < 1 ? 1 : L);
    take_sorted(a, labels, L < 1 ? 1 : L);
    return a.off;
}

int statistics(const Img &inten, const Img &lab, int64_t L, float *T, Arena &ws, cudaStream_t st,
               const uint32_t *d_L) {
    CLE_TRY(same_shape(inten, lab, "intensity_image", "label_image"));
    if (L < 0 || L > 0x7FFFFFFF) { set_error("statistics: bad label count %lld", (long long)L); return CLE_ERR_ARG; }
    if (L == 0) return CLE_OK;
    Acc1 a = take_acc1(ws, L);
    Acc2 b = take_acc2(ws, L);
    Sorted so = take_sorted(ws, lab, L);
    if (!ws.ok()) { set_error("statistics: workspace too small"); return CLE_ERR_WORKSPACE; }
    stats_init<<<launch_blocks(L, 256), 256, 0, st>>>(a, b, L, d_L);
    CLE_LAUNCH_CHECK("statistics init");
    CLE_CUDA(cudaMemsetAsync(so.cnt, 0, sizeof(uint32_t) * (size_t)L, st));
    switch (lab.dtype) {
        case CLE_U32: return stats_i<uint32_t>(inten, lab, L, T, a, b, so, st, d_L);
        case CLE_F32: return stats_i<float>(inten, lab, L, T, a, b, so, st, d_L);
        case CLE_U16: return stats_i<uint16_t>(inten, lab, L, T, a, b, so, st, d_L);
        case CLE_U8: return stats_i<uint8_t>(inten, lab, L, T, a, b, so, st, d_L);
        default: set_error("statistics: unsupported label dtype %d", lab.dtype); return CLE_ERR_DTYPE;
    }
}

size_t centroids_workspace_bytes(int64_t n) {
    Arena a(nullptr, 0);
    a.take<uint32_t>(n);
    a.take<unsigned long long>(3 * n);
    return a.off;
}

int label_centroids(const Img &lab, int64_t n, float *pts, Arena &ws, cudaStream_t st) {
    if (n < 0 || n > 0x7FFFFFFF) { set_error("centroids: bad label count %lld", (long long)n); return CLE_ERR_ARG; }
    if (n == 0) return CLE_OK;
    uint32_t *cnt = ws.take<uint32_t>(n);
    unsigned long long *sums = ws.take<unsigned long long>(3 * n);
    if (!ws.ok()) { set_error("centroids: workspace too small"); return CLE_ERR_WORKSPACE; }
    CLE_CUDA(cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * n, st));
    CLE_CUDA(cudaMemsetAsync(sums, 0, sizeof(unsigned long long) * 3 * n, st));
    const int64_t rows = lab.D * lab.H;
    const int64_t tasks = rows * ((lab.W + 31) / 32);
    if (tasks > 0xFFFFFFFFll) { set_error("centroids: image too large"); return CLE_ERR_TOO_LARGE; }
    const int blocks = launch_blocks(tasks * 32, kST, 8);
    const FastDiv fc((uint32_t)((lab.W + 31) / 32));
    switch (lab.dtype) {
        case CLE_U32:
            centroid_sums_kernel<uint32_t><<<blocks, kST, 0, st>>>((const uint32_t *)lab.data, (uint32_t)lab.W,
                                                                 (uint32_t)lab.H, (uint32_t)tasks, fc, n, cnt, sums);
            break;
        case CLE_F32:
            centroid_sums_kernel<float><<<blocks, kST, 0, st>>>((const float *)lab.data, (uint32_t)lab.W,
                                                              (uint32_t)lab.H, (uint32_t)tasks, fc, n, cnt, sums);
            break;
        default: set_error("centroids: unsupported label dtype %d", lab.dtype); return CLE_ERR_DTYPE;
    }
    centroid_final_kernel<<<launch_blocks(n, 256), 256, 0, st>>>(cnt, sums, n, lab.ndim == 3 ? 3 : 2, pts);
    CLE_LAUNCH_CHECK_N("centroids", 2);
    return CLE_OK;
}

}  // namespace cle
