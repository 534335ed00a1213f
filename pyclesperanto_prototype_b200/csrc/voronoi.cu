// voronoi.cu -- masked_voronoi_labeling growth (_tier5/_masked_voronoi_labeling.py:44-76).
//
// Reference: state S0 = (mask - 1) + CCL(seeds) in float32; Jacobi steps of
// onlyzero_overwrite_maximum -- box stencil (3^d) on even steps, diamond
// (face neighbours) on odd steps -- where a voxel is rewritten only while it
// is 0, with the maximum over the stencil including itself; stop after the
// first step that changes nothing; output mask(S, mask).
//
// The path inside voronoi_otsu_labeling (0/1 mask, seeds inside it) runs the
// same steps on active row bricks only: voronoi_bricks.cu.
//
// masked_voronoi_dense is the general form (any mask values, seeds anywhere)
// used by the standalone op: the reference's float32 state and dense Jacobi
// steps, in one cooperative kernel.
#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

constexpr int kVT = 512;

__device__ __forceinline__ uint32_t block_sum(uint32_t v) {
    __shared__ uint32_t red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t s = 0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
    return s;   // valid in thread 0
}

// ---- dense general form ----------------------------------------------------
struct DenseState {
    GridBarrier bar;
    int err;
    int pad;
    uint32_t changes[4];
};

template <typename Tb, typename Tm>
__global__ void vor_dense_init(const Tb *__restrict__ bin_unused, const Tm *__restrict__ mask,
                               const uint32_t *__restrict__ cc, float *__restrict__ A, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        A[i] = __fadd_rn(__fsub_rn(to_f32(mask[i]), 1.0f), (float)cc[i]);
}

__global__ void __launch_bounds__(kVT)
vor_dense_kernel(float *A, float *B, Geo g, int is3d, int64_t n, DenseState *S, int *d_status,
                 int *d_parity, uint32_t max_steps, uint64_t loop_ns, uint64_t barrier_ns,
                 const volatile int *cancel) {
    const int64_t gtid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
    const int zr = is3d ? 1 : 0;
    bool ok = true, done = false;
    uint32_t t = 0;
    const uint64_t t_start = global_ns();
    while (ok && t < max_steps) {
        if (gtid == 0) {
            if (global_ns() - t_start > loop_ns) atomicExch(&S->err, (int)CLE_ERR_ITER_LIMIT);
            else if (cancel && *cancel) atomicExch(&S->err, (int)CLE_ERR_CANCELLED);
        }
        const float *cur = (t & 1) ? B : A;
        float *nxt = (t & 1) ? A : B;
        const bool box = (t & 1) == 0;
        uint32_t changed = 0;
        for (int64_t i = gtid; i < n; i += gstride) {
            const float v = __ldcg(cur + i);
            if (v != 0.0f) { __stcg(nxt + i, v); continue; }
            uint32_t x, y, z;
            m2xyz(g, (uint32_t)i, x, y, z);
            float mx = v;
            for (int dz = -zr; dz <= zr; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (!box && (abs(dx) + abs(dy) + abs(dz)) > 1) continue;
                        const int qx = (int)x + dx, qy = (int)y + dy, qz = (int)z + dz;
                        if (qx < 0 || qy < 0 || qz < 0 || qx >= (int)g.W || qy >= (int)g.H || qz >= (int)g.D) continue;
                        const float w = __ldcg(cur + xyz2m(g, qx, qy, qz));
                        if (w > mx) mx = w;
                    }
            __stcg(nxt + i, mx);
            changed += (mx != v);
        }
        uint32_t bs = block_sum(changed);
        if (threadIdx.x == 0 && bs) atomicAdd(&S->changes[t & 3], bs);
        ok = grid_sync(&S->bar, &S->err, barrier_ns);
        if (!ok) break;
        const uint32_t c = __ldcg(&S->changes[t & 3]);
        if (gtid == 0) S->changes[(t + 2) & 3] = 0u;
        ++t;
        if (c == 0u) { done = true; break; }
    }
    if (gtid == 0) {
        *d_parity = (int)(t & 1);   // result lives in A when even, B when odd
        int e = *(volatile int *)&S->err;
        *d_status = done ? CLE_OK : (e ? e : (int)CLE_ERR_ITER_LIMIT);
    }
}

template <typename Tm, typename Td>
__global__ void vor_dense_out(const float *__restrict__ A, const float *__restrict__ B,
                              const int *__restrict__ d_parity, const Tm *__restrict__ mask,
                              Td *__restrict__ dst, int64_t n) {
    const float *S = (*d_parity) ? B : A;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        float v = mask[i] != (Tm)0 ? S[i] : 0.0f;
        if constexpr (std::is_same<Td, float>::value) {
            dst[i] = v;
        } else {
            dst[i] = (v > 4294967295.0f) ? 0xFFFFFFFFu : (!(v >= 0.0f) ? 0u : (uint32_t)v);
        }
    }
}

int coop_grid(const void *func, int threads, size_t smem, int64_t work, const Limits &lim,
              int max_per_sm = 64) {
    int dev = 0;
    cudaGetDevice(&dev);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, threads, smem) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    if (per_sm > max_per_sm) per_sm = max_per_sm;
    int64_t cap = (int64_t)per_sm * cooperative_ctas(dev, lim);
    int64_t want = (work + threads * 4 - 1) / (threads * 4);
    if (want < 1) want = 1;
    return (int)(want < cap ? want : cap);
}

}  // namespace

size_t voronoi_dense_workspace_bytes(const Img &im) {
    Arena a(nullptr, 0);
    a.take<DenseState>(1);
    a.take<int>(64);
    a.take<uint32_t>(im.n());   // CCL labels
    a.take<float>(im.n());      // A
    a.take<float>(im.n());      // B
    a.off += ccl_workspace_bytes(im);
    return a.off;
}

template <typename Tm, typename Td>
static int dense_out(const float *A, const float *B, const int *par, const Img &mask,
                     const Img &dst, cudaStream_t st) {
    vor_dense_out<Tm, Td><<<launch_blocks(dst.n(), 256), 256, 0, st>>>(
        A, B, par, (const Tm *)mask.data, (Td *)dst.data, dst.n());
    CLE_LAUNCH_CHECK("voronoi dense out");
    return CLE_OK;
}

int masked_voronoi_dense(const Img &bin, const Img &mask, const Img &dst, int *d_status,
                         Arena &ws, cudaStream_t st, const Limits &lim) {
    CLE_TRY(same_shape(bin, mask, "binary_source", "mask_image"));
    CLE_TRY(same_shape(bin, dst, "binary_source", "labeling_destination"));
    DenseState *S = ws.take<DenseState>(1);
    int *par = ws.take<int>(64);
    uint32_t *cc = ws.take<uint32_t>(bin.n());
    float *A = ws.take<float>(bin.n());
    float *B = ws.take<float>(bin.n());
    if (!ws.ok()) { set_error("masked_voronoi_labeling: workspace too small"); return CLE_ERR_WORKSPACE; }
    CLE_TRY(ccl_dense(bin, cc, ws, st));
    const int64_t n = bin.n();
    const int b = launch_blocks(n, 256);
    switch (mask.dtype) {
        case CLE_U8: vor_dense_init<uint8_t, uint8_t><<<b, 256, 0, st>>>(nullptr, (const uint8_t *)mask.data, cc, A, n); break;
        case CLE_F32: vor_dense_init<uint8_t, float><<<b, 256, 0, st>>>(nullptr, (const float *)mask.data, cc, A, n); break;
        case CLE_U32: vor_dense_init<uint8_t, uint32_t><<<b, 256, 0, st>>>(nullptr, (const uint32_t *)mask.data, cc, A, n); break;
        default: set_error("masked_voronoi_labeling: unsupported mask dtype %d", mask.dtype); return CLE_ERR_DTYPE;
    }
    CLE_LAUNCH_CHECK("voronoi dense init");
    CLE_CUDA(cudaMemsetAsync(S, 0, sizeof(DenseState), st));
    Geo g = make_geo(bin);
    int is3d = bin.ndim == 3 ? 1 : 0;
    uint32_t max_steps = lim.steps_for(bin.n());
    uint64_t loop_ns = lim.loop_ns, barrier_ns = lim.barrier_ns;
    const volatile int *cancel = lim.cancel;
    int64_t nn = n;
    const int grid = coop_grid((const void *)vor_dense_kernel, kVT, 0, n, lim);
    void *args[] = {&A, &B, &g, &is3d, &nn, &S, &d_status, &par, &max_steps, &loop_ns, &barrier_ns,
                    (void *)&cancel};
    CLE_CUDA(cudaLaunchCooperativeKernel((const void *)vor_dense_kernel, dim3(grid), dim3(kVT), args,
                                         0, st));
    count_launches(1);
    switch (mask.dtype) {
        case CLE_U8:
            return dst.dtype == CLE_F32 ? dense_out<uint8_t, float>(A, B, par, mask, dst, st)
                                        : dense_out<uint8_t, uint32_t>(A, B, par, mask, dst, st);
        case CLE_F32:
            return dst.dtype == CLE_F32 ? dense_out<float, float>(A, B, par, mask, dst, st)
                                        : dense_out<float, uint32_t>(A, B, par, mask, dst, st);
        default:
            return dst.dtype == CLE_F32 ? dense_out<uint32_t, float>(A, B, par, mask, dst, st)
                                        : dense_out<uint32_t, uint32_t>(A, B, par, mask, dst, st);
    }
}

}  // namespace cle
