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

}  // namespace

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
