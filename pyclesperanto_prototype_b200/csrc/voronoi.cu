// voronoi.cu -- masked_voronoi_labeling growth (_tier5/_masked_voronoi_labeling.py:44-76).
//
// Reference: state S0 = (mask - 1) + CCL(seeds) in float32; Jacobi steps of
// onlyzero_overwrite_maximum -- box stencil (3^d) on even steps, diamond
// (face neighbours) on odd steps -- where a voxel is rewritten only while it
// is 0, with the maximum over the stencil including itself; stop after the
// first step that changes nothing; output mask(S, mask).
//
// voronoi_frontier (the path used by voronoi_otsu_labeling, where the mask is
// a 0/1 segmentation and every seed lies inside it) runs the same steps but
// visits only the frontier: the zero voxels of the mask with a labelled voxel
// in their box neighbourhood.  A step is two phases separated by grid
// barriers: (A) every frontier voxel computes its new value from the state
// of the previous step; (B) new values are written, and the zero mask
// neighbours of newly labelled voxels plus the voxels that stayed zero form
// the next frontier.  Membership in the next frontier is claimed with a CAS
// that stores kMarkBit|step in the label buffer (mark bits read as 0 in the
// maximum), so the label buffer doubles as the visited set; marks left when
// the loop ends are cleared.  Outside-mask voxels hold 0 and are never
// candidates, which matches -1 in the reference for every output voxel.
//
// masked_voronoi_dense is the general form (any mask values, seeds anywhere)
// used by the standalone op: the reference's float32 state and dense Jacobi
// steps, in one cooperative kernel.
#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

constexpr int kVT = 512;
constexpr int kFT = 384;                   // frontier kernel block (one per SM)
constexpr int kBuf = 16384;                // block-local append buffer (entries)
constexpr int kFlushAt = kBuf - 27 * kFT;  // flush threshold
constexpr size_t kBufBytes = sizeof(uint32_t) * kBuf;
constexpr uint32_t kSkip = 0xFFFFFFFFu;
constexpr uint32_t kTraceSteps = 256;
constexpr uint64_t kBarrierLimitNs = 4000000000ull;   // 4 s per barrier wait
constexpr uint64_t kKernelLimitNs = 20000000000ull;   // 20 s per launch

struct VorState {
    GridBarrier bar;
    int err;
    int done;
    uint32_t sizes[4];
    uint32_t changes[4];
    uint32_t steps;
    uint32_t pad[3];
};

// Block-local append buffer in shared memory.  Loops that push run with a
// block-uniform trip count and call maybe_flush() after each round, which
// moves the buffer to the global list (one atomicAdd per flush) once it is
// past kFlushAt; a round pushes at most 27 entries per thread, so the buffer
// never overflows.
struct Appender {
    uint32_t *buf;      // shared, kBuf entries
    uint32_t *cnt;      // shared
    __device__ __forceinline__ void push(uint32_t v) {
        const uint32_t pos = atomicAdd(cnt, 1u);
        buf[pos] = v;
    }
    // All threads of the block must call.
    __device__ __forceinline__ void flush(uint32_t *dst, uint32_t *dst_size) {
        __shared__ uint32_t base;
        __syncthreads();
        const uint32_t n = *cnt;
        if (threadIdx.x == 0) base = n ? atomicAdd(dst_size, n) : 0u;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) dst[base + i] = buf[i];
        __syncthreads();
        if (threadIdx.x == 0) *cnt = 0;
        __syncthreads();
    }
    // All threads of the block must call (after a round of pushes).
    __device__ __forceinline__ void maybe_flush(uint32_t *dst, uint32_t *dst_size) {
        __syncthreads();
        if (*cnt >= (uint32_t)kFlushAt) flush(dst, dst_size);
    }
};

// Claims voxel q (whose label word was read as v) for the frontier of `step`.
__device__ __forceinline__ void try_mark_from(uint32_t *lab, uint32_t q, uint32_t v, uint32_t step,
                                              Appender &ap, uint32_t *dst, uint32_t *dst_size) {
    const uint32_t mark = kMarkBit | step;
    for (;;) {
        if (v != 0u && !(v & kMarkBit)) return;   // already labelled
        if (v == mark) return;                     // already queued for this step
        uint32_t old = atomicCAS(lab + q, v, mark);
        if (old == v) {
            ap.push(q);
            return;
        }
        v = old;
    }
}

__device__ __forceinline__ bool needs_mark(uint32_t v, uint32_t step) {
    return v == 0u || ((v & kMarkBit) && v != (kMarkBit | step));
}

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

// Clamped neighbour coordinates: reading the clamp-to-edge neighbourhood
// (the reference's own read semantics) only repeats voxels of the stencil,
// so no per-neighbour bounds test is needed and every load can be in flight.
struct Nbr {
    uint32_t xs[3], ys[3], zs[3];
};

__device__ __forceinline__ Nbr nbr_of(const Geo &g, uint32_t m, bool is3d) {
    uint32_t x, y, z;
    m2xyz(g, m, x, y, z);
    Nbr n;
    n.xs[0] = x ? x - 1 : 0; n.xs[1] = x; n.xs[2] = (x + 1 < g.W) ? x + 1 : x;
    n.ys[0] = y ? y - 1 : 0; n.ys[1] = y; n.ys[2] = (y + 1 < g.H) ? y + 1 : y;
    if (is3d) {
        n.zs[0] = z ? z - 1 : 0; n.zs[1] = z; n.zs[2] = (z + 1 < g.D) ? z + 1 : z;
    } else {
        n.zs[0] = n.zs[1] = n.zs[2] = z;
    }
    return n;
}

// Maximum label (mark bits read as 0) over the box or the face stencil.
__device__ __forceinline__ uint32_t stencil_max(const uint32_t *lab, const Geo &g, const Nbr &n,
                                                bool box) {
    uint32_t v[27];
#pragma unroll
    for (int k = 0; k < 27; ++k) {
        const int dz = k / 9, dy = (k / 3) % 3, dx = k % 3;
        const bool face = (abs(dx - 1) + abs(dy - 1) + abs(dz - 1)) <= 1;
        v[k] = (box || face) ? lab[xyz2m(g, n.xs[dx], n.ys[dy], n.zs[dz])] : 0u;
    }
    uint32_t mx = 0;
#pragma unroll
    for (int k = 0; k < 27; ++k)
        if (!(v[k] & kMarkBit)) mx = max(mx, v[k]);
    return mx;
}

// Predicated compare-and-swap: issued only when `pred`; returns `cmp` when
// not issued.  Written as one predicated instruction so that a thread's CAS
// attempts on several neighbours are all in flight together instead of each
// waiting behind a divergent branch.
__device__ __forceinline__ uint32_t cas_if(uint32_t *addr, uint32_t cmp, uint32_t val, bool pred) {
    uint32_t old = cmp;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.u32 p, %4, 0;\n\t"
        "@p atom.global.cas.b32 %0, [%1], %2, %3;\n\t}"
        : "+r"(old)
        : "l"(addr), "r"(cmp), "r"(val), "r"((uint32_t)pred)
        : "memory");
    return old;
}

// Queues the zero mask voxels of the box neighbourhood of p for `step`.
__device__ __forceinline__ void mark_neighbours(uint32_t *lab, const uint8_t *seg, const Geo &g,
                                                const Nbr &n, uint32_t step, Appender &ap,
                                                uint32_t *dst, uint32_t *dst_size) {
    const uint32_t mark = kMarkBit | step;
    uint32_t v[27];
    uint32_t segbits = 0;
#pragma unroll
    for (int k = 0; k < 27; ++k) {
        const int dz = k / 9, dy = (k / 3) % 3, dx = k % 3;
        const uint32_t q = xyz2m(g, n.xs[dx], n.ys[dy], n.zs[dz]);
        segbits |= (seg[q] ? 1u : 0u) << k;
        v[k] = lab[q];
    }
    uint32_t old[27];
#pragma unroll
    for (int k = 0; k < 27; ++k) {
        const int dz = k / 9, dy = (k / 3) % 3, dx = k % 3;
        const bool c = k != 13 && ((segbits >> k) & 1u) && needs_mark(v[k], step);
        old[k] = cas_if(lab + xyz2m(g, n.xs[dx], n.ys[dy], n.zs[dz]), v[k], mark, c);
    }
#pragma unroll
    for (int k = 0; k < 27; ++k) {
        const int dz = k / 9, dy = (k / 3) % 3, dx = k % 3;
        const bool c = k != 13 && ((segbits >> k) & 1u) && needs_mark(v[k], step);
        if (!c) continue;
        const uint32_t q = xyz2m(g, n.xs[dx], n.ys[dy], n.zs[dz]);
        if (old[k] == v[k]) ap.push(q);                                // claimed
        else try_mark_from(lab, q, old[k], step, ap, dst, dst_size);   // lost a race: re-check
    }
}

// Loads of the label buffer go through L1: every phase starts after a grid
// barrier whose gpu-scope acquire invalidates the SM's L1, and within phase
// B a stale neighbour value can only be older, which the CAS corrects.
__global__ void __launch_bounds__(kFT, 1)
voronoi_frontier_kernel(uint32_t *lab, const uint8_t *__restrict__ seg, Geo g, int is3d,
                        const uint32_t *seeds, const uint32_t *d_seed_count, uint32_t *L0,
                        uint32_t *L1, uint32_t *Mv, VorState *S, int *d_status,
                        uint32_t max_steps, unsigned long long *trace) {
    extern __shared__ uint32_t s_buf[];   // kBuf entries
    __shared__ uint32_t s_cnt;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    Appender ap{s_buf, &s_cnt};
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t gstride = gridDim.x * blockDim.x;

    // frontier 0: zero mask voxels in the box neighbourhood of the seeds
    const uint32_t ns = __ldcg(d_seed_count);
    for (uint32_t base = blockIdx.x * blockDim.x; base < ns; base += gstride) {
        const uint32_t i = base + threadIdx.x;
        if (i < ns) mark_neighbours(lab, seg, g, nbr_of(g, __ldcg(seeds + i), is3d), 0u, ap, L0, &S->sizes[0]);
        ap.maybe_flush(L0, &S->sizes[0]);
    }
    ap.flush(L0, &S->sizes[0]);
    bool ok = grid_sync(&S->bar, &S->err, kBarrierLimitNs);

    const uint64_t t_start = global_ns();
    uint32_t t = 0;
    bool done = false;
    while (ok && t < max_steps) {
        if (gtid == 0 && global_ns() - t_start > kKernelLimitNs) atomicExch(&S->err, (int)CLE_ERR_ITER_LIMIT);
        uint32_t *F = (t & 1) ? L1 : L0;
        uint32_t *Fn = (t & 1) ? L0 : L1;
        const uint32_t nF = __ldcg(&S->sizes[t & 3]);
        const bool box = (t & 1) == 0;
        // phase A: new values from the current state
        uint32_t changed = 0;
        for (uint32_t i = gtid; i < nF; i += gstride) {
            const uint32_t p = F[i];
            const uint32_t v = lab[p];
            if (v != 0u && !(v & kMarkBit)) { Mv[i] = kSkip; continue; }
            const uint32_t mx = stencil_max(lab, g, nbr_of(g, p, is3d), box);
            Mv[i] = mx;
            changed += (mx != 0u);
        }
        uint32_t bs = block_sum(changed);
        if (threadIdx.x == 0 && bs) atomicAdd(&S->changes[t & 3], bs);
        ok = grid_sync(&S->bar, &S->err, kBarrierLimitNs);
        if (!ok) break;
        if (trace && gtid == 0 && t < kTraceSteps) {
            trace[3 * t] = global_ns() - t_start;
            trace[3 * t + 1] = nF;
            trace[3 * t + 2] = __ldcg(&S->changes[t & 3]);
        }
        if (__ldcg(&S->changes[t & 3]) == 0u) { done = true; break; }
        // phase B: write, then build the next frontier
        if (gtid == 0) {
            S->changes[(t + 2) & 3] = 0u;
            S->sizes[(t + 2) & 3] = 0u;
        }
        uint32_t *nsize = &S->sizes[(t + 1) & 3];
        for (uint32_t base = blockIdx.x * blockDim.x; base < nF; base += gstride) {
            const uint32_t i = base + threadIdx.x;
            const uint32_t mv = (i < nF) ? Mv[i] : kSkip;
            if (mv != kSkip) {
                const uint32_t p = F[i];
                if (mv == 0u) {
                    try_mark_from(lab, p, lab[p], t + 1, ap, Fn, nsize);
                } else {
                    lab[p] = mv;
                    mark_neighbours(lab, seg, g, nbr_of(g, p, is3d), t + 1, ap, Fn, nsize);
                }
            }
            ap.maybe_flush(Fn, nsize);
        }
        ap.flush(Fn, nsize);
        ok = grid_sync(&S->bar, &S->err, kBarrierLimitNs);
        ++t;
    }
    if (done) {
        // clear the marks of the voxels that stayed zero
        uint32_t *F = (t & 1) ? L1 : L0;
        const uint32_t nF = __ldcg(&S->sizes[t & 3]);
        for (uint32_t i = gtid; i < nF; i += gstride) {
            const uint32_t p = __ldcg(F + i);
            if (ld_cg(lab + p) & kMarkBit) st_cg(lab + p, 0u);
        }
    }
    if (gtid == 0) {
        S->steps = t + 1;
        S->done = done ? 1 : 0;
        int e = *(volatile int *)&S->err;
        *d_status = done ? CLE_OK : (e ? e : (int)CLE_ERR_ITER_LIMIT);
    }
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
                 int *d_parity, uint32_t max_steps) {
    const int64_t gtid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
    const int zr = is3d ? 1 : 0;
    bool ok = true, done = false;
    uint32_t t = 0;
    const uint64_t t_start = global_ns();
    while (ok && t < max_steps) {
        if (gtid == 0 && global_ns() - t_start > kKernelLimitNs) atomicExch(&S->err, (int)CLE_ERR_ITER_LIMIT);
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
        ok = grid_sync(&S->bar, &S->err, kBarrierLimitNs);
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

int coop_grid(const void *func, int threads, size_t smem, int64_t work, int max_per_sm = 64) {
    int dev = 0;
    cudaGetDevice(&dev);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, threads, smem) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    if (per_sm > max_per_sm) per_sm = max_per_sm;
    int64_t cap = (int64_t)per_sm * num_sms(dev);
    int64_t want = (work + threads * 4 - 1) / (threads * 4);
    if (want < 1) want = 1;
    return (int)(want < cap ? want : cap);
}

}  // namespace

size_t voronoi_frontier_workspace_bytes(const Img &im) {
    Arena a(nullptr, 0);
    a.take<VorState>(1);
    a.take<uint32_t>(im.n());   // L0
    a.take<uint32_t>(im.n());   // Mv
    return a.off;
}

// L1 (the second frontier list) is the seed list buffer: the seeds are
// consumed while frontier 0 is built into L0, before L1 is first written.
int voronoi_frontier(const Img &im, uint32_t *lab, const uint8_t *seg, const uint32_t *seeds,
                     const uint32_t *d_seed_count, int *d_status, Arena &ws, cudaStream_t st) {
    VorState *S = ws.take<VorState>(1);
    uint32_t *L0 = ws.take<uint32_t>(im.n());
    uint32_t *Mv = ws.take<uint32_t>(im.n());
    if (!ws.ok()) { set_error("masked_voronoi_labeling: workspace too small"); return CLE_ERR_WORKSPACE; }
    uint32_t *L1 = const_cast<uint32_t *>(seeds);
    CLE_CUDA(cudaMemsetAsync(S, 0, sizeof(VorState), st));
    Geo g = make_geo(im);
    int is3d = im.ndim == 3 ? 1 : 0;
    uint32_t max_steps = (uint32_t)im.n() + 16u;   // each step that changes labels >= 1 voxel
    static bool attr = false;
    if (!attr) {
        CLE_CUDA(cudaFuncSetAttribute((const void *)voronoi_frontier_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBufBytes));
        attr = true;
    }
    const int grid = coop_grid((const void *)voronoi_frontier_kernel, kFT, kBufBytes, im.n() / 16 + 1, 1);
    unsigned long long *trace = (unsigned long long *)profile_trace_buffer(3 * kTraceSteps * sizeof(unsigned long long));
    void *args[] = {&lab, (void *)&seg, &g, &is3d, (void *)&seeds, (void *)&d_seed_count, &L0, &L1,
                    &Mv, &S, &d_status, &max_steps, &trace};
    CLE_CUDA(cudaLaunchCooperativeKernel((const void *)voronoi_frontier_kernel, dim3(grid), dim3(kFT),
                                         args, kBufBytes, st));
    count_launches(1);
    return CLE_OK;
}

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
                         Arena &ws, cudaStream_t st) {
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
    uint32_t max_steps = (uint32_t)bin.n() + 16u;
    int64_t nn = n;
    const int grid = coop_grid((const void *)vor_dense_kernel, kVT, 0, n);
    void *args[] = {&A, &B, &g, &is3d, &nn, &S, &d_status, &par, &max_steps};
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
