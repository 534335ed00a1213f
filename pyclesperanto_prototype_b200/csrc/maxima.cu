// maxima.cu -- detect_maxima_box with radius 1 (_tier1/detect_maxima_3d_x.cl:1-49,
// _tier1/detect_maxima_2d_x.cl:1-35).
//
// The reference kernel walks the 3^d box in order dx (outer), dy, dz (inner),
// starting from localMax = v(p) - 1, skipping positions with a negative
// coordinate, reading clamp-to-edge and keeping the first strict maximum;
// p is flagged iff that arg-max is p itself.  For v(p) - 1 < v(p) this is
// exactly:  v(p) > max(in-bounds neighbours preceding p in walk order)  and
// v(p) >= max(in-bounds neighbours following p)  -- clamped re-reads of the
// upper border only repeat voxels whose constraint is already implied.  When
// v(p) - 1 == v(p) (|v| >= 2^24, inf) both comparisons are >=; a NaN centre
// always wins and NaN neighbours never do.
//
// The preceding set is {dx=-1: all} + {dx=0, dy=-1: all dz} + {(0,0,-1)}, so
// with T(x,y) = max_dz v and S(x,y) = max_dy T:
//   A = max(S(x-1,y), T(x,y-1), v(z-1)),  B = max(S(x+1,y), T(x,y+1), v(z+1)).
// Each thread owns 4 consecutive rows of one x column and marches along z
// with a 3-plane x 6-row register window; x neighbours come from warp
// shuffles (a warp covers 30 output columns plus one halo lane each side).
#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

constexpr int kRows = 4;          // output rows per thread
constexpr int kWin = kRows + 2;   // rows held (halo above and below)
constexpr int kOutX = 30;         // output columns per warp
constexpr int kGroups = 4;        // y-groups (warps) per block

template <typename Ts, typename Td>
__global__ void __launch_bounds__(32 * kGroups)
maxima_kernel(const Ts *__restrict__ src, Td *__restrict__ dst, int D, int H, int W, int zchunk) {
    const int lane = threadIdx.x;
    const int x = (int)blockIdx.x * kOutX + lane - 1;
    const int y0 = ((int)blockIdx.y * kGroups + threadIdx.y) * kRows;
    const int z0 = (int)blockIdx.z * zchunk;
    const int z1 = min(D, z0 + zchunk);
    if (y0 >= H) return;   // whole warp leaves together (y0 is warp-uniform)
    const bool xin = (x >= 0 && x < W);
    const float NEG = -INFINITY;

    auto load = [&](int z, int j) -> float {
        int y = y0 - 1 + j;
        if (!xin || z < 0 || z >= D || y < 0 || y >= H) return NEG;
        return to_f32(src[((int64_t)z * H + y) * W + x]);
    };

    float vm[kWin], vc[kWin], vp[kWin];
#pragma unroll
    for (int j = 0; j < kWin; ++j) {
        vm[j] = load(z0 - 1, j);
        vc[j] = load(z0, j);
    }
    for (int z = z0; z < z1; ++z) {
#pragma unroll
        for (int j = 0; j < kWin; ++j) vp[j] = load(z + 1, j);
        float T[kWin];
#pragma unroll
        for (int j = 0; j < kWin; ++j) T[j] = fmaxf(fmaxf(vm[j], vc[j]), vp[j]);
        float S[kRows];
#pragma unroll
        for (int j = 0; j < kRows; ++j) S[j] = fmaxf(fmaxf(T[j], T[j + 1]), T[j + 2]);
#pragma unroll
        for (int j = 0; j < kRows; ++j) {
            const float sl = __shfl_up_sync(0xffffffffu, S[j], 1);
            const float sr = __shfl_down_sync(0xffffffffu, S[j], 1);
            const int y = y0 + j;
            if (lane >= 1 && lane <= kOutX && xin && y < H) {
                const float v = vc[j + 1];
                const float A = fmaxf(fmaxf(sl, T[j]), vm[j + 1]);
                const float B = fmaxf(fmaxf(sr, T[j + 2]), vp[j + 1]);
                bool win;
                if (v != v) {
                    win = true;
                } else if (__fsub_rn(v, 1.0f) < v) {
                    win = (v > A) && (v >= B);
                } else {
                    win = (v >= A) && (v >= B);
                }
                dst[((int64_t)z * H + y) * W + x] = (Td)(win ? 1 : 0);
            }
        }
#pragma unroll
        for (int j = 0; j < kWin; ++j) {
            vm[j] = vc[j];
            vc[j] = vp[j];
        }
    }
}

// voronoi_otsu_labeling's steps 2 and 7 in one pass when both blurs are the
// same image T (equal sigmas): the maxima flag of detect_maxima_box (as
// above), then seg = T > t (greater_constant with the float32 threshold) and
// seed = flag & seg (binary_and), with the seeds' initial CCL keys
// (x-major pixel index + 1) in the label buffer and the seeds listed -- the
// spots image is never written or re-read.  Every voxel's seg and label entry
// is written.
// ROWS output rows per thread (the window holds ROWS + 2), so rows are read
// (ROWS + 2) / ROWS times.  Row offsets inside a plane and their validity are
// computed once; per plane only the plane's base moves.  Every owned voxel's
// seg and label entry is written.
template <int ROWS>
__global__ void __launch_bounds__(32 * kGroups, 5)
maxima_seeds_kernel(const float *__restrict__ T, const float *__restrict__ d_thr32, Geo g, int zchunk,
                    uint8_t *__restrict__ seg, uint32_t *__restrict__ lab, uint32_t *__restrict__ seeds,
                    uint32_t *__restrict__ d_count) {
    constexpr int kRows = ROWS, kWin = ROWS + 2;
    const int D = (int)g.D, H = (int)g.H, W = (int)g.W;
    const uint32_t HW = g.H * g.W;
    const int lane = threadIdx.x;
    const int x = (int)blockIdx.x * kOutX + lane - 1;
    const int y0 = ((int)blockIdx.y * kGroups + threadIdx.y) * kRows;
    const int z0 = (int)blockIdx.z * zchunk;
    const int z1 = min(D, z0 + zchunk);
    if (y0 >= H) return;   // whole warp leaves together (y0 is warp-uniform)
    const bool xin = (x >= 0 && x < W);
    const bool own = lane >= 1 && lane <= kOutX && xin;
    const float NEG = -INFINITY;
    const float t = *d_thr32;
    uint32_t roff[kWin];
    bool rok[kWin];
#pragma unroll
    for (int j = 0; j < kWin; ++j) {
        const int y = y0 - 1 + j;
        rok[j] = xin && y >= 0 && y < H;
        roff[j] = rok[j] ? (uint32_t)y * g.W + (uint32_t)x : 0u;
    }
    auto load_plane = [&](int z, float *v) {
        const bool zok = z >= 0 && z < D;
        const float *P = T + (size_t)(zok ? z : 0) * HW;
#pragma unroll
        for (int j = 0; j < kWin; ++j) v[j] = (zok && rok[j]) ? P[roff[j]] : NEG;
    };

    // planes z-1, z, z+1 held; plane z+2 loads while plane z is computed
    float vm[kWin], vc[kWin], vp[kWin], vn[kWin];
    load_plane(z0 - 1, vm);
    load_plane(z0, vc);
    load_plane(z0 + 1, vp);
    for (int z = z0; z < z1; ++z) {
        if (z + 1 < z1) load_plane(z + 2, vn);
        float Tm[kWin];
#pragma unroll
        for (int j = 0; j < kWin; ++j) Tm[j] = fmaxf(fmaxf(vm[j], vc[j]), vp[j]);
        float S[kRows];
#pragma unroll
        for (int j = 0; j < kRows; ++j) S[j] = fmaxf(fmaxf(Tm[j], Tm[j + 1]), Tm[j + 2]);
        const uint32_t zoff = (uint32_t)z * HW;
#pragma unroll
        for (int j = 0; j < kRows; ++j) {
            const float sl = __shfl_up_sync(0xffffffffu, S[j], 1);
            const float sr = __shfl_down_sync(0xffffffffu, S[j], 1);
            const bool mine = own && rok[j + 1];
            bool seed = false;
            const uint32_t m = zoff + roff[j + 1];
            if (mine) {
                const float v = vc[j + 1];
                const float A = fmaxf(fmaxf(sl, Tm[j]), vm[j + 1]);
                const float B = fmaxf(fmaxf(sr, Tm[j + 2]), vp[j + 1]);
                bool win;
                if (v != v) {
                    win = true;
                } else if (__fsub_rn(v, 1.0f) < v) {
                    win = (v > A) && (v >= B);
                } else {
                    win = (v >= A) && (v >= B);
                }
                const bool sg = v > t;
                seed = sg && win;
                seg[m] = sg ? kMaskByte : 0;
                lab[m] = seed ? xyz2k(g, (uint32_t)x, (uint32_t)(y0 + j), (uint32_t)z) + 1u : 0u;
            }
            const unsigned b = __ballot_sync(0xffffffffu, seed);
            if (b) {
                uint32_t base = 0;
                const int leader = __ffs(b) - 1;
                if (lane == leader) base = atomicAdd(d_count, (uint32_t)__popc(b));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (seed) seeds[base + __popc(b & ((1u << lane) - 1u))] = m;
            }
        }
#pragma unroll
        for (int j = 0; j < kWin; ++j) {
            vm[j] = vc[j];
            vc[j] = vp[j];
            vp[j] = vn[j];
        }
    }
}

// The same pass with two adjacent columns per lane (rows of an even length,
// 8-byte aligned T and labels): 64-bit loads of T, a 16-bit store of the two
// mask bytes and a 64-bit store of the two labels; the x neighbours of a
// column come from the lane's other column or, across lanes, by shuffles.
// A warp covers 60 output columns (lanes 1..30; lanes 0 and 31 load the halo
// pairs).
constexpr int kOutX2 = 60;

template <int ROWS>
__global__ void __launch_bounds__(32 * kGroups)
maxima_seeds2_kernel(const float *__restrict__ T, const float *__restrict__ d_thr32, Geo g, int zchunk,
                     uint8_t *__restrict__ seg, uint32_t *__restrict__ lab, uint32_t *__restrict__ seeds,
                     uint32_t *__restrict__ d_count) {
    constexpr int kRows = ROWS, kWin = ROWS + 2;
    const int D = (int)g.D, H = (int)g.H, W = (int)g.W;
    const uint32_t HW = g.H * g.W;
    const int lane = threadIdx.x;
    const int xa = (int)blockIdx.x * kOutX2 + 2 * lane - 2;   // columns xa, xa + 1
    const int y0 = ((int)blockIdx.y * kGroups + threadIdx.y) * kRows;
    const int z0 = (int)blockIdx.z * zchunk;
    const int z1 = min(D, z0 + zchunk);
    if (y0 >= H) return;   // whole warp leaves together (y0 is warp-uniform)
    const bool xin = xa >= 0 && xa < W;   // W even: xa + 1 < W as well
    const bool own = lane >= 1 && lane <= kOutX2 / 2 && xin;
    const float NEG = -INFINITY;
    const float t = *d_thr32;
    uint32_t roff[kWin];
    bool rok[kWin];
#pragma unroll
    for (int j = 0; j < kWin; ++j) {
        const int y = y0 - 1 + j;
        rok[j] = xin && y >= 0 && y < H;
        roff[j] = rok[j] ? (uint32_t)y * g.W + (uint32_t)xa : 0u;
    }
    auto load_plane = [&](int z, float2 *v) {
        const bool zok = z >= 0 && z < D;
        const float *P = T + (size_t)(zok ? z : 0) * HW;
#pragma unroll
        for (int j = 0; j < kWin; ++j)
            v[j] = (zok && rok[j]) ? *reinterpret_cast<const float2 *>(P + roff[j]) : make_float2(NEG, NEG);
    };
    auto winner = [](float v, float A, float B) {
        if (v != v) return true;
        if (__fsub_rn(v, 1.0f) < v) return (v > A) && (v >= B);
        return (v >= A) && (v >= B);
    };

    // planes z-1, z, z+1 held; plane z+2 loads while plane z is computed
    float2 vm[kWin], vc[kWin], vp[kWin], vn[kWin];
    load_plane(z0 - 1, vm);
    load_plane(z0, vc);
    load_plane(z0 + 1, vp);
    for (int z = z0; z < z1; ++z) {
        if (z + 1 < z1) load_plane(z + 2, vn);
        float2 Tm[kWin];
#pragma unroll
        for (int j = 0; j < kWin; ++j)
            Tm[j] = make_float2(fmaxf(fmaxf(vm[j].x, vc[j].x), vp[j].x), fmaxf(fmaxf(vm[j].y, vc[j].y), vp[j].y));
        const uint32_t zoff = (uint32_t)z * HW;
#pragma unroll
        for (int j = 0; j < kRows; ++j) {
            const float Sa = fmaxf(fmaxf(Tm[j].x, Tm[j + 1].x), Tm[j + 2].x);
            const float Sb = fmaxf(fmaxf(Tm[j].y, Tm[j + 1].y), Tm[j + 2].y);
            const float sl = __shfl_up_sync(0xffffffffu, Sb, 1);     // column xa - 1
            const float sr = __shfl_down_sync(0xffffffffu, Sa, 1);   // column xa + 2
            const bool mine = own && rok[j + 1];
            bool seed_a = false, seed_b = false;
            const uint32_t m = zoff + roff[j + 1];
            if (mine) {
                const float va = vc[j + 1].x, vb = vc[j + 1].y;
                const bool wa = winner(va, fmaxf(fmaxf(sl, Tm[j].x), vm[j + 1].x), fmaxf(fmaxf(Sb, Tm[j + 2].x), vp[j + 1].x));
                const bool wb = winner(vb, fmaxf(fmaxf(Sa, Tm[j].y), vm[j + 1].y), fmaxf(fmaxf(sr, Tm[j + 2].y), vp[j + 1].y));
                const bool ga = va > t, gb = vb > t;
                seed_a = ga && wa;
                seed_b = gb && wb;
                *reinterpret_cast<uint16_t *>(seg + m) = (uint16_t)((ga ? (uint32_t)kMaskByte : 0u) | (gb ? (uint32_t)kMaskByte << 8 : 0u));
                uint2 lv = make_uint2(0u, 0u);
                if (seed_a | seed_b) {
                    const uint32_t k = xyz2k(g, (uint32_t)xa, (uint32_t)(y0 + j), (uint32_t)z) + 1u;
                    lv.x = seed_a ? k : 0u;
                    lv.y = seed_b ? k + g.H * g.D : 0u;   // key of column xa + 1
                }
                *reinterpret_cast<uint2 *>(lab + m) = lv;
            }
            const unsigned ba = __ballot_sync(0xffffffffu, seed_a), bb = __ballot_sync(0xffffffffu, seed_b);
            if (ba | bb) {
                uint32_t base = 0;
                const int leader = __ffs(ba | bb) - 1;
                if (lane == leader) base = atomicAdd(d_count, (uint32_t)(__popc(ba) + __popc(bb)));
                base = __shfl_sync(0xffffffffu, base, leader);
                const unsigned below = (1u << lane) - 1u;
                const uint32_t at = base + __popc(ba & below) + __popc(bb & below);
                if (seed_a) seeds[at] = m;
                if (seed_b) seeds[at + (seed_a ? 1u : 0u)] = m + 1u;
            }
        }
#pragma unroll
        for (int j = 0; j < kWin; ++j) {
            vm[j] = vc[j];
            vc[j] = vp[j];
            vp[j] = vn[j];
        }
    }
}

// Grid of the z-marching kernels: 30 columns per warp, kGroups x kRows rows
// per block, z chunks so that about 12 blocks per SM are launched.
int maxima_grid(const Img &src, dim3 &grid, int &zchunk, int rows = kRows, int cols = kOutX) {
    const int D = (int)src.D, H = (int)src.H, W = (int)src.W;
    const int gx = (W + cols - 1) / cols;
    const int gy = (H + rows * kGroups - 1) / (rows * kGroups);
    int dev = 0;
    cudaGetDevice(&dev);
    const int64_t target = (int64_t)num_sms(dev) * 12;   // blocks
    int64_t zchunks = (target + (int64_t)gx * gy - 1) / ((int64_t)gx * gy);
    if (zchunks > D) zchunks = D;
    if (zchunks < 1) zchunks = 1;
    zchunk = (int)((D + zchunks - 1) / zchunks);
    if (zchunk < 4 && D >= 4) zchunk = 4;
    zchunks = (D + zchunk - 1) / zchunk;
    if (gy > 65535 || zchunks > 65535) { set_error("detect_maxima: image too large"); return CLE_ERR_TOO_LARGE; }
    grid = dim3(gx, gy, (unsigned)zchunks);
    return CLE_OK;
}

template <typename Ts, typename Td>
int launch_maxima(const Img &src, const Img &dst, cudaStream_t st) {
    const int D = (int)src.D, H = (int)src.H, W = (int)src.W;
    dim3 grid;
    int zchunk = 1;
    CLE_TRY(maxima_grid(src, grid, zchunk));
    dim3 block(32, kGroups);
    maxima_kernel<Ts, Td><<<grid, block, 0, st>>>((const Ts *)src.data, (Td *)dst.data, D, H, W, zchunk);
    CLE_LAUNCH_CHECK("detect_maxima");
    return CLE_OK;
}

template <typename Ts>
int maxima_dst(const Img &src, const Img &dst, cudaStream_t st) {
    switch (dst.dtype) {
        case CLE_U8: return launch_maxima<Ts, uint8_t>(src, dst, st);
        case CLE_F32: return launch_maxima<Ts, float>(src, dst, st);
        case CLE_U32: return launch_maxima<Ts, uint32_t>(src, dst, st);
        default: set_error("detect_maxima_box: unsupported destination dtype %d", dst.dtype); return CLE_ERR_DTYPE;
    }
}

}  // namespace

int maxima_seeds(const Img &T, const float *d_thr32, uint8_t *seg, uint32_t *lab, uint32_t *seeds,
                 uint32_t *d_count, cudaStream_t st) {
    if (T.dtype != CLE_F32) { set_error("internal: maxima_seeds needs a float32 image"); return CLE_ERR_DTYPE; }
    constexpr int kSeedRows = 8;
    dim3 grid;
    int zchunk = 1;
    const bool pairs = T.W % 2 == 0 && (reinterpret_cast<uintptr_t>(T.data) & 7) == 0 &&
                       (reinterpret_cast<uintptr_t>(lab) & 7) == 0 && (reinterpret_cast<uintptr_t>(seg) & 1) == 0;
    if (pairs) {
        constexpr int kPairRows = 4;
        CLE_TRY(maxima_grid(T, grid, zchunk, kPairRows, kOutX2));
        maxima_seeds2_kernel<kPairRows><<<grid, dim3(32, kGroups), 0, st>>>(
            (const float *)T.data, d_thr32, make_geo(T), zchunk, seg, lab, seeds, d_count);
        CLE_LAUNCH_CHECK("detect_maxima + seeds (column pairs)");
        return CLE_OK;
    }
    CLE_TRY(maxima_grid(T, grid, zchunk, kSeedRows));
    maxima_seeds_kernel<kSeedRows><<<grid, dim3(32, kGroups), 0, st>>>((const float *)T.data, d_thr32, make_geo(T),
                                                                     zchunk, seg, lab, seeds, d_count);
    CLE_LAUNCH_CHECK("detect_maxima + seeds");
    return CLE_OK;
}

int detect_maxima(const Img &src, const Img &dst, cudaStream_t st) {
    CLE_TRY(same_shape(src, dst, "source", "destination"));
    switch (src.dtype) {
        case CLE_F32: return maxima_dst<float>(src, dst, st);
        case CLE_U16: return maxima_dst<uint16_t>(src, dst, st);
        case CLE_U8: return maxima_dst<uint8_t>(src, dst, st);
        default: set_error("detect_maxima_box: unsupported source dtype %d", src.dtype); return CLE_ERR_DTYPE;
    }
}

}  // namespace cle
