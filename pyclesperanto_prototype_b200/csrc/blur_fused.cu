// blur_fused.cu -- one-launch separable Gaussian blur for isotropic sigma.
//
// Same arithmetic as the three-pass path in blur.cu (x pass, then y, then z,
// float32 intermediates, clamp-to-edge, acc = fma(w_i, v_i, acc) for
// i = -R..R from 0), fused so the source is read once and the result written
// once:
//   * a CTA owns a kTX x kTY output tile in (x, y) and marches along z over a
//     chunk of planes (plus R halo planes at each end, clamped);
//   * per input plane it stages the clamped (kTY+2R) x (kTX+2R) tile in
//     shared memory as float32.  On volumes whose rows are a multiple of 16
//     bytes and whose grid fills two waves of resident CTAs (and when the
//     caller gives a status word) one thread fetches
//     each plane's raw tile with a TMA copy (cp.async.bulk.tensor) into a ring
//     of kStages shared-memory stages, kStages-1 planes ahead, completion
//     counted by an mbarrier per stage; the CTA converts the landed tile to
//     float32 with 64/128-bit shared loads.  Otherwise the next plane's raw
//     values are loaded into registers while the current one is computed
//     and converted when stored;
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
#include <cuda.h>
#include <cudaTypedefs.h>
#include <atomic>
#include <cstring>

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
    static constexpr size_t SMEM = sizeof(float) * (ROWS * STRIDE + ROWS * kTX);
    static_assert(ROWS * (kTX / kXO) <= kThreads, "x pass: at most one item per thread");
};

// Two CTAs per SM (<= 128 registers, no spills) while the z ring is small.
template <int R>
constexpr int min_ctas() { return R <= 8 ? 2 : 1; }

// ---- TMA staging ------------------------------------------------------------
// The box of a plane starts at x = x0 - R - OFF (OFF rounds it down so that
// x * sizeof(Tin) is a multiple of 16 bytes, the tiled copy's rule for the
// innermost coordinate), y = y0 - R and z = the clamped plane.  Box parts
// outside the image arrive zero-filled and are never read: the conversion
// gathers every staged element from its clamped coordinate, which lies inside
// both the image and the box.
constexpr int kStages = 3;
constexpr uint64_t kStageWaitNs = 2000000000ull;   // bound of one stage wait

template <typename Tin, int R>
struct TmaGeom {
    static constexpr int ES = (int)sizeof(Tin);
    static constexpr int A = 16 / ES;                                   // x alignment (elements)
    static constexpr int OFF = (R + A - 1) / A * A - R;
    static constexpr int BX = (Geom<R>::COLS + OFF + A - 1) / A * A;    // box columns
    static constexpr int BY = Geom<R>::ROWS;                            // box rows
    static constexpr uint32_t BYTES = (uint32_t)(BX * BY * ES);         // one plane's copy
    static constexpr int STAGE = (int)((BYTES + 127) / 128 * 128);
    static constexpr bool VEC = OFF % 4 == 0;                           // quads start 4-aligned
    static constexpr int QC = (Geom<R>::COLS + 3) / 4;                  // quads per staged row
    static constexpr int QPT = (BY * QC + kThreads - 1) / kThreads;     // quads per thread
    static constexpr size_t SMEM = 128 + (size_t)kStages * STAGE + Geom<R>::SMEM;
    static_assert(BX <= 256 && BY <= 256, "TMA box dimension above 256");
    static_assert(!VEC || 4 * QC + OFF <= BX, "quad conversion reads inside the box row");
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}
// Waits for the phase of `parity` to complete; false after kStageWaitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > kStageWaitNs) return false;
    return true;
}
// Orders this thread's earlier shared-memory accesses before its next
// async-proxy (TMA) write into the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tma_load_plane(void *dst, const CUtensorMap *map, int x, int y, int z,
                                               uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

// four consecutive staged source values as float32 (the same values as to_f32)
__device__ __forceinline__ float4 quad_f32(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float4 quad_f32(const uint16_t *p) {
    const uint2 u = *reinterpret_cast<const uint2 *>(p);
    return make_float4((float)(u.x & 0xFFFFu), (float)(u.x >> 16), (float)(u.y & 0xFFFFu), (float)(u.y >> 16));
}
__device__ __forceinline__ float4 quad_f32(const uint8_t *p) {
    const uint32_t u = *reinterpret_cast<const uint32_t *>(p);
    return make_float4((float)(u & 0xFFu), (float)((u >> 8) & 0xFFu), (float)((u >> 16) & 0xFFu), (float)(u >> 24));
}

// TMA: stage planes with the tensor map `tmap` (3D only); a stage wait that
// runs out sets *status and ends the CTA after its copies have landed.
template <typename Tin, int R, bool Z, bool TMA>
__global__ void __launch_bounds__(kThreads, min_ctas<R>())
blur_fused_kernel(const Tin *__restrict__ src, const __grid_constant__ CUtensorMap tmap,
                  float *__restrict__ dst, int D, int H, int W, int zchunk,
                  const __grid_constant__ Taps taps, float *__restrict__ mm, int *__restrict__ status) {
    static_assert(!TMA || Z, "TMA staging is for volumes");
    using G = Geom<R>;
    using TG = TmaGeom<Tin, R>;
    constexpr int WIN = 2 * R + 1;
    extern __shared__ __align__(16) float smem[];
    // TMA: kStages raw stages first (128-byte aligned), then In and Xo
    uint8_t *raw = reinterpret_cast<uint8_t *>(smem);
    if constexpr (TMA) raw += (128u - (smem_addr(smem) & 127u)) & 127u;
    float *In = TMA ? reinterpret_cast<float *>(raw + kStages * TG::STAGE) : smem;   // [ROWS][STRIDE]
    float *Xo = In + G::ROWS * G::STRIDE;                                             // [ROWS][kTX]

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
    Tin pre[TMA ? 1 : G::LOADS];
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
                if constexpr (!TMA) pre[rr * G::COL_LOADS + c] = ok ? __ldg(row + gx[c]) : Tin(0);
            }
        }
    };
    auto store_plane = [&]() {
#pragma unroll
        for (int rr = 0; rr < G::ROWS_PER_WARP; ++rr) {
            const int r = warp + rr * kWarps;
#pragma unroll
            for (int c = 0; c < G::COL_LOADS; ++c)
                if constexpr (!TMA)
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

    // TMA staging state: per-stage barriers, box origin, and for tiles that
    // need no x clamp the quads this thread converts (raw offset in elements,
    // In offset in floats; -1 = none)
    __shared__ __align__(8) uint64_t bars[kStages];
    const int xs = x0 - R - TG::OFF, ys = y0 - R;
    const bool quads = TG::VEC && x0 - R >= 0 && x0 - R + G::COLS <= W;
    int qsrc[TG::QPT], qdst[TG::QPT];
    auto issue = [&](int v) {   // one thread: plane v into stage v % kStages
        uint64_t *bar = &bars[v % kStages];
        fence_proxy_async_smem();
        mbar_expect_tx(bar, TG::BYTES);
        tma_load_plane(raw + (v % kStages) * TG::STAGE, &tmap, xs, ys, clampi(zbase + v, 0, D - 1), bar);
    };
    auto convert = [&](const Tin *rs) {
        if (quads) {
#pragma unroll
            for (int k = 0; k < TG::QPT; ++k)
                if (qsrc[k] >= 0) *reinterpret_cast<float4 *>(In + qdst[k]) = quad_f32(rs + qsrc[k]);
        } else {
            for (int e = tid; e < G::ROWS * G::COLS; e += kThreads) {
                const int r = e / G::COLS, c = e - r * G::COLS;
                const int sr = clampi(ys + r, 0, H - 1) - ys;
                const int sc = clampi(x0 - R + c, 0, W - 1) - xs;
                In[r * G::STRIDE + c] = to_f32(rs[sr * TG::BX + sc]);
            }
        }
    };
    if constexpr (TMA) {
#pragma unroll
        for (int k = 0; k < TG::QPT; ++k) {
            const int e = tid + k * kThreads;
            const int r = e / TG::QC, q = e - r * TG::QC;
            const bool ok = e < TG::BY * TG::QC;
            qsrc[k] = ok ? (clampi(ys + r, 0, H - 1) - ys) * TG::BX + 4 * q + TG::OFF : -1;
            qdst[k] = r * G::STRIDE + 4 * q;
        }
        if (tid == 0) {
            for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
            mbar_init_fence();
        }
        __syncthreads();
        if (tid == 0)
            for (int v = 0; v < kStages - 1 && v < nvirt; ++v) issue(v);
    } else {
        load_plane(0);
    }
    int failed_at = -1;   // TMA: plane whose stage wait ran out
    // one plane per iteration, not unrolled (the loop body stays small enough
    // for the instruction caches); the ring shifts by one slot per plane, so
    // ring[j][i] holds plane v - 2R + i
#pragma unroll 1
    for (int v = 0; v < nvirt; ++v) {
        __syncthreads();   // previous plane fully consumed (In, Xo, its stage)
        if constexpr (TMA) {
            if (tid == 0 && v + kStages - 1 < nvirt) issue(v + kStages - 1);
            const bool ok = mbar_wait(&bars[v % kStages], (uint32_t)(v / kStages) & 1u);
            if (ok) convert(reinterpret_cast<const Tin *>(raw + (v % kStages) * TG::STAGE));
            if (__syncthreads_or(!ok)) { failed_at = v; break; }
        } else {
            store_plane();
            if (v + 1 < nvirt) load_plane(v + 1);
            __syncthreads();
        }
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
    if constexpr (TMA) {
        if (failed_at >= 0) {
            // the copies still in flight (planes failed_at .. issued-1) land
            // before the CTA's shared memory is released
            if (tid == 0) {
                const int issued = min(nvirt, failed_at + kStages);
                for (int p = failed_at; p < issued; ++p) mbar_wait(&bars[p % kStages], (uint32_t)(p / kStages) & 1u);
                atomicCAS(status, 0, (int)CLE_ERR_ITER_LIMIT);
            }
            return;
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

// Upper bound on the z chunks of the fused launch: four waves of two CTAs per
// SM (the most a tile count could use), at most one chunk per plane.
int64_t fused_chunk_cap(int64_t tiles, int64_t D, int sms) {
    return std::max<int64_t>(1, std::min<int64_t>(D, (8 * (int64_t)sms + tiles - 1) / tiles));
}

// Grid of the fused launch: (x tiles, y tiles, z chunks).  A CTA's time is
// about its planes (chunk + 2R halo), and CTAs run in waves of the resident
// slots, so the chunk count minimises waves x (chunk + 2R): 512 x 1024 x 1024
// at R = 8 takes 2 chunks (2048 CTAs, 6.9 waves of 296) rather than 1
// (1024 CTAs, a half-empty fourth wave).
dim3 fused_grid(const Img &src, int R, int &zchunk) {
    const int gx = (int)((src.W + kTX - 1) / kTX);
    const int gy = (int)((src.H + kTY - 1) / kTY);
    int gz = 1;
    zchunk = 1;
    if (src.ndim == 3) {
        int dev = 0;
        cudaGetDevice(&dev);
        const int sms = num_sms(dev);
        const int64_t slots = (int64_t)sms * (R <= 8 ? 2 : 1);
        const int64_t tiles = (int64_t)gx * gy;
        const int64_t cap = fused_chunk_cap(tiles, src.D, sms);
        int64_t best = -1;
        for (int64_t c = 1; c <= cap; ++c) {
            const int64_t zc = (src.D + c - 1) / c;
            const int64_t g = (src.D + zc - 1) / zc;
            const int64_t waves = (tiles * g + slots - 1) / slots;
            const int64_t cost = waves * (zc + 2 * R);
            if (best < 0 || cost < best) {
                best = cost;
                zchunk = (int)zc;
                gz = (int)g;
            }
        }
    }
    return dim3(gx, gy, gz);
}

// The source as a 3D tiled tensor map (x = W innermost) with the box of
// TmaGeom<Tin, R>; false when the layout does not allow one (row pitch or base
// address not a multiple of 16 bytes) or the driver lacks the encoder.
// The driver's tensor-map encoder, looked up once outside any stream capture
// (an immutable function pointer; until then, and if the driver lacks it,
// the register-staged path runs).
void *tensor_map_encoder(cudaStream_t st) {
    static std::atomic<void *> fn{nullptr};
    static std::atomic<bool> looked{false};
    if (looked.load(std::memory_order_acquire)) return fn.load(std::memory_order_acquire);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        (void)cudaGetLastError();
        return nullptr;
    }
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
        (void)cudaGetLastError();
        f = nullptr;
    }
    fn.store(f, std::memory_order_release);
    looked.store(true, std::memory_order_release);
    return f;
}

template <typename Tin, int R>
bool encode_source_map(const Img &src, CUtensorMap &map, cudaStream_t st) {
    using TG = TmaGeom<Tin, R>;
    const uint64_t pitch = (uint64_t)src.W * sizeof(Tin);
    if (pitch % 16 != 0 || (reinterpret_cast<uintptr_t>(src.data) & 15) != 0) return false;
    void *const fn = tensor_map_encoder(st);
    if (fn == nullptr) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)src.W, (cuuint64_t)src.H, (cuuint64_t)src.D};
    const cuuint64_t strides[2] = {(cuuint64_t)pitch, (cuuint64_t)(pitch * (uint64_t)src.H)};
    const cuuint32_t box[3] = {(cuuint32_t)TG::BX, (cuuint32_t)TG::BY, 1u};
    const cuuint32_t estride[3] = {1u, 1u, 1u};
    const CUtensorMapDataType dt = sizeof(Tin) == 1 ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                 : sizeof(Tin) == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16
                                                    : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const CUresult r = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn)(
        &map, dt, 3, src.data, dims, strides, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

template <typename Tin, int R, bool Z>
int launch_fused_r(const Img &src, float *dst, const Taps &t, float *mm, int *status, cudaStream_t st) {
    using G = Geom<R>;
    static_assert(min_ctas<R>() == (R <= 8 ? 2 : 1), "fused_grid's occupancy rule");
    int zchunk = 1;
    const dim3 grid = fused_grid(src, R, zchunk);
    if (grid.y > 65535 || grid.z > 65535) { set_error("gaussian_blur: image too large for the fused path"); return CLE_ERR_TOO_LARGE; }
    alignas(64) CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    if constexpr (Z) {
        // TMA staging once the grid fills two waves of resident CTAs: with
        // fewer CTAs (one wave, one or two per SM) the register-staged path
        // measured faster (128 x 512 x 512 at R = 8: 0.265 vs 0.305 ms;
        // 512 x 1024 x 1024: 3.19 vs 3.12 ms the other way)
        int dev = 0;
        cudaGetDevice(&dev);
        const int64_t ctas = (int64_t)grid.x * grid.y * grid.z;
        const bool waves2 = ctas >= 2 * (int64_t)num_sms(dev) * min_ctas<R>();
        if (status != nullptr && waves2 && encode_source_map<Tin, R>(src, map, st)) {
            auto kern = blur_fused_kernel<Tin, R, true, true>;
            const size_t smem = TmaGeom<Tin, R>::SMEM;
            // set on every call: the attribute belongs to the current device's context
            CLE_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            kern<<<grid, kThreads, smem, st>>>((const Tin *)src.data, map, dst, (int)src.D, (int)src.H,
                                               (int)src.W, zchunk, t, mm, status);
            CLE_LAUNCH_CHECK("gaussian_blur fused (TMA)");
            return CLE_OK;
        }
    }
    auto kern = blur_fused_kernel<Tin, R, Z, false>;
    CLE_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM));
    kern<<<grid, kThreads, G::SMEM, st>>>((const Tin *)src.data, map, dst, (int)src.D, (int)src.H, (int)src.W,
                                          zchunk, t, mm, status);
    CLE_LAUNCH_CHECK("gaussian_blur fused");
    return CLE_OK;
}

template <typename Tin, bool Z, int R = 1>
int dispatch_r(const Img &src, float *dst, const Taps &t, int r, float *mm, int *status, cudaStream_t st) {
    if constexpr (R > kMaxFusedR) {
        set_error("internal: fused radius out of range");
        return CLE_ERR_ARG;
    } else {
        if (r == R) return launch_fused_r<Tin, R, Z>(src, dst, t, mm, status, st);
        return dispatch_r<Tin, Z, R + 1>(src, dst, t, r, mm, status, st);
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

int fused_blur(const Img &src, float *dst, double sigma, cudaStream_t st, float *mm, int *status) {
    Taps t;
    CLE_TRY(make_gauss_taps(sigma, t));
    const int r = (t.n - 1) / 2;
    const bool z = src.ndim == 3;
    switch (src.dtype) {
        case CLE_F32: return z ? dispatch_r<float, true>(src, dst, t, r, mm, status, st) : dispatch_r<float, false>(src, dst, t, r, mm, status, st);
        case CLE_U16: return z ? dispatch_r<uint16_t, true>(src, dst, t, r, mm, status, st) : dispatch_r<uint16_t, false>(src, dst, t, r, mm, status, st);
        case CLE_U8: return z ? dispatch_r<uint8_t, true>(src, dst, t, r, mm, status, st) : dispatch_r<uint8_t, false>(src, dst, t, r, mm, status, st);
        default: set_error("gaussian_blur: unsupported source dtype"); return CLE_ERR_DTYPE;
    }
}

size_t blur_minmax_workspace_bytes(const Img &src) {
    // any sigma: the three-pass path with the separate min / max, or the
    // fused partials (at most fused_chunk_cap z chunks per tile)
    int dev = 0;
    cudaGetDevice(&dev);
    const int64_t tiles = ((src.W + kTX - 1) / kTX) * ((src.H + kTY - 1) / kTY);
    const int64_t chunks = fused_chunk_cap(tiles, std::max<int64_t>(src.D, 1), num_sms(dev));
    const size_t fused = sizeof(float) * 2 * (size_t)(tiles * chunks) + 256;
    return std::max(fused, separable_workspace_bytes(src) + minmax_workspace_bytes(src));
}

int blur_minmax(const Img &src, float *dst, double sigma, float *d_minmax, Arena &ws, cudaStream_t st,
                int *status) {
    if (!fused_blur_applies(src, sigma, sigma, sigma)) {
        CLE_TRY(gaussian_blur(src, dst, sigma, sigma, sigma, ws, st, status));
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
    CLE_TRY(fused_blur(src, dst, sigma, st, partial, status));
    return minmax_finish(partial, ctas, d_minmax, st);
}

}  // namespace cle
