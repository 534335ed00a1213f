// ccl.cu -- connected_components_labeling_box and relabel_sequential.
//
// Reference semantics (_tier4/_connected_components_labeling_box.py:39-64):
// every foreground voxel starts with its pixel-index key K+1 held in float32
// (set_nonzero_pixels_to_pixelindex, key x-major: K = (x*H + y)*D + z,
// tests/test_set_nonzero_pixels_to_pixelindex.py), Jacobi min-propagation
// over the 3^d box until stable, then relabel_sequential ranks the distinct
// float32 values (_tier3/_relabel_sequential.py:42-57).  So a component's
// label is the rank of float32(min K + 1) among all components, and
// components whose float32 keys round to the same value share a label.
//
// Here: union-find whose parent pointers are K values (stored as K+1 in the
// u32 label buffer, 0 = background), linked with atomicMin so every root is
// its component's minimum key; the distinct float32 root keys are marked in
// a bitmap over integer-valued floats (fkey_index) and ranked with a
// per-word popcount prefix.  No N-sized float vectors, no host round trips.
#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

constexpr int kT = 256;

__device__ __forceinline__ uint32_t find_root(const uint32_t *lab, const Geo &g, uint32_t k) {
    uint32_t p = ld_cg(lab + k2m(g, k)) - 1u;
    while (p != k) {
        k = p;
        p = ld_cg(lab + k2m(g, k)) - 1u;
    }
    return k;
}

// find_root with path halving, for the union phase: a visited non-root
// entry is lowered to its grandparent with atomicMin.  Entries only ever move
// to an ancestor in the same tree and roots are never touched, so concurrent
// unions (which link roots only) are unaffected.
__device__ __forceinline__ uint32_t find_root_halve(uint32_t *lab, const Geo &g, uint32_t k) {
    uint32_t mk = k2m(g, k);
    uint32_t p = ld_cg(lab + mk) - 1u;
    while (p != k) {
        const uint32_t mp = k2m(g, p);
        const uint32_t gp = ld_cg(lab + mp) - 1u;
        if (gp == p) return p;
        atomicMin(lab + mk, gp + 1u);
        k = gp;
        mk = k2m(g, k);
        p = ld_cg(lab + mk) - 1u;
    }
    return k;
}

__device__ __forceinline__ void unite(uint32_t *lab, const Geo &g, uint32_t a, uint32_t b) {
    for (;;) {
        a = find_root_halve(lab, g, a);
        b = find_root_halve(lab, g, b);
        if (a == b) return;
        if (a < b) { uint32_t t = a; a = b; b = t; }
        // link root a (larger key) under b
        uint32_t old = atomicMin(lab + k2m(g, a), b + 1u) - 1u;
        if (old == a) return;
        a = old;
    }
}

// Unions voxel (x,y,z) (foreground) with its 13 memory-order predecessors.
__device__ __forceinline__ void union_back(uint32_t *lab, const Geo &g, uint32_t x, uint32_t y,
                                           uint32_t z) {
    const uint32_t kp = xyz2k(g, x, y, z);
#pragma unroll
    for (int dz = -1; dz <= 0; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                if (dz == 0 && (dy > 0 || (dy == 0 && dx >= 0))) continue;
                const int qz = (int)z + dz, qy = (int)y + dy, qx = (int)x + dx;
                if (qz < 0 || qy < 0 || qy >= (int)g.H || qx < 0 || qx >= (int)g.W) continue;
                const uint32_t v = ld_cg(lab + xyz2m(g, qx, qy, qz));
                if (v) unite(lab, g, kp, xyz2k(g, qx, qy, qz));
            }
}

// ---- dense labelling on row runs ------------------------------------------
// A warp covers one row segment: 32 consecutive x of one (z, y) row.  In a
// row, x-major keys grow with x, so the first voxel of a run holds the run's
// smallest key: init links every foreground voxel straight to the start of
// its run inside the segment.  The union step then joins whole runs: a run
// [a, b] of the segment is united once with every run of each backward row
// ((y-1, z) and (y-1..y+1, z-1)) that overlaps it (through the first voxel of
// the overlap), with a run of that row that touches it only diagonally at
// a-1 or b+1, and with the run that continues it from the previous segment.
// That is every 26-neighbour contact (each adjacent pair has one backward
// side), with a few unions per run instead of 13 per voxel.
constexpr int kRowWarps = 8;   // warps (row segments in flight) per CTA

struct Rows {
    uint32_t WS;     // segments per row
    FastDiv fWS;
    uint32_t nseg;   // D * H * WS
};

template <typename T>
__global__ void __launch_bounds__(kRowWarps * 32)
ccl_init_rows(const T *__restrict__ bin, uint32_t *__restrict__ lab, Geo g, Rows R) {
    const int lane = threadIdx.x & 31;
    for (uint32_t s = blockIdx.x * kRowWarps + (threadIdx.x >> 5); s < R.nseg; s += gridDim.x * kRowWarps) {
        const uint32_t r = R.fWS.div(s), xs = s - r * R.WS;       // r = z * H + y
        const uint32_t z = g.fH.div(r), y = r - z * g.H;
        const uint32_t x = xs * 32u + (uint32_t)lane;
        const bool in = x < g.W;
        const bool fg = in && bin[r * g.W + x] != (T)0;
        const unsigned F = __ballot_sync(0xffffffffu, fg);
        const unsigned starts = F & ~(F << 1);                    // fg lanes after a bg lane (or lane 0)
        if (in) {
            uint32_t v = 0u;
            if (fg) {
                const uint32_t a = 31u - __clz(starts & (0xffffffffu >> (31 - lane)));   // run start lane
                v = xyz2k(g, xs * 32u + a, y, z) + 1u;
            }
            lab[r * g.W + x] = v;
        }
    }
}

// DIAMOND: face connectivity (connected_components_labeling_diamond): only
// the backward rows (y-1, z) and (y, z-1) at the same x, no diagonal contacts.
template <bool DIAMOND>
__global__ void __launch_bounds__(kRowWarps * 32)
ccl_union_rows(uint32_t *lab, Geo g, Rows R) {
    const int lane = threadIdx.x & 31;
    const uint32_t xstep = g.H * g.D;                             // key distance of x +- 1
    for (uint32_t s = blockIdx.x * kRowWarps + (threadIdx.x >> 5); s < R.nseg; s += gridDim.x * kRowWarps) {
        const uint32_t r = R.fWS.div(s), xs = s - r * R.WS;
        const uint32_t z = g.fH.div(r), y = r - z * g.H;
        const uint32_t x = xs * 32u + (uint32_t)lane;
        const bool in = x < g.W;
        // foreground-ness never changes while parents are relinked
        const bool fg = in && ld_cg(lab + r * g.W + x) != 0u;
        const unsigned F = __ballot_sync(0xffffffffu, fg);
        if (!F) continue;
        const unsigned starts = F & ~(F << 1);
        const bool is_start = starts >> lane & 1u;
        const bool is_end = (F & ~(F >> 1)) >> lane & 1u;
        const uint32_t kp = xyz2k(g, x, y, z);
        // unions start from the run's first voxel (every run voxel points at it)
        const uint32_t a = fg ? 31u - __clz(starts & (0xffffffffu >> (31 - lane))) : (uint32_t)lane;
        const uint32_t ka = kp - ((uint32_t)lane - a) * xstep;
        // the run continued from the previous segment
        if (lane == 0 && fg && xs > 0 && ld_cg(lab + r * g.W + x - 1u) != 0u) unite(lab, g, kp, kp - xstep);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (DIAMOND && (k == 1 || k == 3)) continue;        // (y-1, z-1), (y+1, z-1): no face contact
            const int qy = (int)y + (k == 0 ? -1 : k - 2), qz = (int)z - (k == 0 ? 0 : 1);
            if (qy < 0 || qy >= (int)g.H || qz < 0) continue;    // warp-uniform
            const uint32_t *row = lab + ((uint32_t)qz * g.H + (uint32_t)qy) * g.W;
            const bool q = in && ld_cg(row + x) != 0u;
            bool qe = false;                                     // lane 0: row[x-1], lane 31: row[x+1]
            if (lane == 0 && xs > 0) qe = ld_cg(row + x - 1u) != 0u;
            if (lane == 31 && x + 1u < g.W) qe = ld_cg(row + x + 1u) != 0u;
            const unsigned Q = __ballot_sync(0xffffffffu, q);
            const bool qL = (lane == 0) ? qe : ((Q >> (lane - 1)) & 1u);
            const bool qR = (lane == 31) ? qe : ((Q >> (lane + 1)) & 1u);
            if (!fg) continue;
            const uint32_t kq = xyz2k(g, x, (uint32_t)qy, (uint32_t)qz);
            if (q && (is_start || !qL)) unite(lab, g, ka, kq);            // first voxel of an overlap
            if (DIAMOND) continue;
            if (is_start && qL && !q) unite(lab, g, ka, kq - xstep);     // diagonal contact at a-1
            if (is_end && qR && !q) unite(lab, g, ka, kq + xstep);       // diagonal contact at b+1
        }
    }
}

// Flatten on row runs: the run-start lane of each run (whose voxels all
// point at it after init) walks to the root; its run gets the root by shuffle.
// The forest no longer changes here except that entries move to their roots.
__global__ void __launch_bounds__(kRowWarps * 32)
ccl_flatten_rows(uint32_t *lab, Geo g, Rows R) {
    const int lane = threadIdx.x & 31;
    for (uint32_t s = blockIdx.x * kRowWarps + (threadIdx.x >> 5); s < R.nseg; s += gridDim.x * kRowWarps) {
        const uint32_t r = R.fWS.div(s), xs = s - r * R.WS;
        const uint32_t z = g.fH.div(r), y = r - z * g.H;
        const uint32_t x = xs * 32u + (uint32_t)lane;
        const bool in = x < g.W;
        const uint32_t v = in ? ld_cg(lab + r * g.W + x) : 0u;
        const unsigned F = __ballot_sync(0xffffffffu, v != 0u);
        if (!F) continue;
        const unsigned starts = F & ~(F << 1);
        uint32_t root = 0u;
        if ((starts >> lane) & 1u) root = find_root(lab, g, xyz2k(g, x, y, z)) + 1u;
        const int a = (v != 0u) ? 31 - __clz(starts & (0xffffffffu >> (31 - lane))) : lane;
        root = __shfl_sync(0xffffffffu, root, a);
        if (v != 0u && root != v) st_cg(lab + r * g.W + x, root);
    }
}

__global__ void ccl_mark_dense(const uint32_t *__restrict__ lab, Geo g, int64_t n,
                               uint32_t *__restrict__ bitmap) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t v = lab[i];
        if (!v) continue;
        uint32_t x, y, z;
        m2xyz(g, (uint32_t)i, x, y, z);
        if (v - 1u != xyz2k(g, x, y, z)) continue;   // not a root
        uint32_t idx = fkey_index((float)v);          // float32(K + 1)
        atomicOr(bitmap + (idx >> 5), 1u << (idx & 31));
    }
}

__device__ __forceinline__ uint32_t rank_of(const uint32_t *bitmap, const uint32_t *prefix,
                                            uint32_t idx) {
    const uint32_t w = idx >> 5, b = idx & 31;
    return prefix[w] + __popc(bitmap[w] & ((1u << b) - 1u)) + 1u;
}

__global__ void ccl_label_dense(uint32_t *__restrict__ lab, int64_t n,
                                const uint32_t *__restrict__ bitmap,
                                const uint32_t *__restrict__ prefix) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t v = lab[i];
        if (!v) continue;
        lab[i] = rank_of(bitmap, prefix, fkey_index((float)v));
    }
}

// ---- list variants (sparse seeds) ---------------------------------------
__global__ void ccl_union_list(uint32_t *lab, Geo g, const uint32_t *__restrict__ list,
                               const uint32_t *__restrict__ d_count) {
    const uint32_t cnt = *d_count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        uint32_t x, y, z;
        m2xyz(g, list[i], x, y, z);
        union_back(lab, g, x, y, z);
    }
}

__global__ void ccl_flatten_list(uint32_t *lab, Geo g, const uint32_t *__restrict__ list,
                                 const uint32_t *__restrict__ d_count) {
    const uint32_t cnt = *d_count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const uint32_t m = list[i];
        uint32_t v = ld_cg(lab + m);
        uint32_t r = find_root(lab, g, v - 1u);
        if (r != v - 1u) st_cg(lab + m, r + 1u);
    }
}

__global__ void ccl_mark_list(const uint32_t *__restrict__ lab, Geo g,
                              const uint32_t *__restrict__ list,
                              const uint32_t *__restrict__ d_count, uint32_t *__restrict__ bitmap) {
    const uint32_t cnt = *d_count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const uint32_t m = list[i];
        const uint32_t v = lab[m];
        uint32_t x, y, z;
        m2xyz(g, m, x, y, z);
        if (v - 1u != xyz2k(g, x, y, z)) continue;
        uint32_t idx = fkey_index((float)v);
        atomicOr(bitmap + (idx >> 5), 1u << (idx & 31));
    }
}

__global__ void ccl_label_list(uint32_t *__restrict__ lab, const uint32_t *__restrict__ list,
                               const uint32_t *__restrict__ d_count,
                               const uint32_t *__restrict__ bitmap,
                               const uint32_t *__restrict__ prefix) {
    const uint32_t cnt = *d_count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const uint32_t m = list[i];
        lab[m] = rank_of(bitmap, prefix, fkey_index((float)lab[m]));
    }
}

__global__ void count_ranks_kernel(const uint32_t *__restrict__ bitmap,
                                   const uint32_t *__restrict__ prefix, uint32_t words,
                                   uint32_t *__restrict__ out) {
    *out = prefix[words - 1] + __popc(bitmap[words - 1]);
}

// ---- rank machinery -------------------------------------------------------
__global__ void chunk_count_kernel(const uint32_t *__restrict__ bitmap, uint32_t words,
                                   uint32_t *__restrict__ chunk) {
    const uint32_t nchunks = (words + 31) / 32;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nchunks; c += gridDim.x * blockDim.x) {
        uint32_t s = 0;
        const uint32_t w1 = min(words, (c + 1) * 32);
        for (uint32_t w = c * 32; w < w1; ++w) s += __popc(bitmap[w]);
        chunk[c] = s;
    }
}

// Exclusive scan of n uint32 in place, one CTA of 1024 threads.
__global__ void __launch_bounds__(1024) scan_single_cta(uint32_t *__restrict__ a, uint32_t n) {
    __shared__ uint32_t warp_tot[32];
    const uint32_t per = (n + 1023) / 1024;
    const uint32_t b0 = threadIdx.x * per;
    const uint32_t b1 = min(n, b0 + per);
    uint32_t s = 0;
    for (uint32_t i = b0; i < b1; ++i) s += a[i];
    // inclusive scan of s over the block
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t v = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) warp_tot[wid] = v;
    __syncthreads();
    if (wid == 0) {
        uint32_t t = warp_tot[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t u = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += u;
        }
        warp_tot[lane] = t;
    }
    __syncthreads();
    uint32_t run = v - s + (wid ? warp_tot[wid - 1] : 0u);
    for (uint32_t i = b0; i < b1; ++i) {
        uint32_t x = a[i];
        a[i] = run;
        run += x;
    }
}

__global__ void word_prefix_kernel(const uint32_t *__restrict__ bitmap, uint32_t words,
                                   const uint32_t *__restrict__ chunk, uint32_t *__restrict__ prefix) {
    const uint32_t nchunks = (words + 31) / 32;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nchunks; c += gridDim.x * blockDim.x) {
        uint32_t run = chunk[c];
        const uint32_t w1 = min(words, (c + 1) * 32);
        for (uint32_t w = c * 32; w < w1; ++w) {
            prefix[w] = run;
            run += __popc(bitmap[w]);
        }
    }
}

struct Rank {
    uint32_t *bitmap, *chunk, *prefix;
    uint32_t words, nchunks;
};

Rank take_rank(Arena &ws, uint64_t bits) {
    Rank r;
    r.words = (uint32_t)((bits + 31) / 32 + 1);
    r.nchunks = (r.words + 31) / 32;
    r.bitmap = ws.take<uint32_t>(r.words);
    r.chunk = ws.take<uint32_t>(r.nchunks);
    r.prefix = ws.take<uint32_t>(r.words);
    return r;
}

int rank_build(const Rank &r, cudaStream_t st) {
    const int b = launch_blocks(r.nchunks, kT);
    chunk_count_kernel<<<b, kT, 0, st>>>(r.bitmap, r.words, r.chunk);
    scan_single_cta<<<1, 1024, 0, st>>>(r.chunk, r.nchunks);
    word_prefix_kernel<<<b, kT, 0, st>>>(r.bitmap, r.words, r.chunk, r.prefix);
    CLE_LAUNCH_CHECK_N("rank build", 3);
    return CLE_OK;
}

template <typename T>
int launch_ccl_init(const Img &bin, uint32_t *lab, const Geo &g, const Rows &R, int blocks,
                    cudaStream_t st) {
    ccl_init_rows<T><<<blocks, kRowWarps * 32, 0, st>>>((const T *)bin.data, lab, g, R);
    CLE_LAUNCH_CHECK("ccl init");
    return CLE_OK;
}

// ---- relabel ------------------------------------------------------------
template <typename T>
__device__ __forceinline__ uint32_t label_value(T v) {
    if constexpr (std::is_floating_point<T>::value) {
        return v > (T)0 ? (uint32_t)(int64_t)v : 0u;
    } else {
        return (uint32_t)v;
    }
}

template <typename T>
__global__ void relabel_mark_kernel(const T *__restrict__ s, int64_t n, uint32_t maxv,
                                    uint32_t *__restrict__ bitmap) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t v = label_value(s[i]);
        if (v == 0 || v > maxv) continue;
        atomicOr(bitmap + (v >> 5), 1u << (v & 31));
    }
}

template <typename T, typename Td>
__global__ void relabel_apply_kernel(const T *__restrict__ s, Td *__restrict__ d, int64_t n,
                                     uint32_t maxv, const uint32_t *__restrict__ bitmap,
                                     const uint32_t *__restrict__ prefix) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t v = label_value(s[i]);
        uint32_t out = (v == 0 || v > maxv) ? 0u : rank_of(bitmap, prefix, v);
        d[i] = (Td)out;
    }
}

template <typename T>
int relabel_typed(const Img &src, const Img &dst, uint32_t maxv, const Rank &r, cudaStream_t st) {
    const int64_t n = src.n();
    const int b = launch_blocks(n, kT);
    relabel_mark_kernel<T><<<b, kT, 0, st>>>((const T *)src.data, n, maxv, r.bitmap);
    CLE_LAUNCH_CHECK("relabel mark");
    CLE_TRY(rank_build(r, st));
    switch (dst.dtype) {
        case CLE_U32: relabel_apply_kernel<T, uint32_t><<<b, kT, 0, st>>>((const T *)src.data, (uint32_t *)dst.data, n, maxv, r.bitmap, r.prefix); break;
        case CLE_F32: relabel_apply_kernel<T, float><<<b, kT, 0, st>>>((const T *)src.data, (float *)dst.data, n, maxv, r.bitmap, r.prefix); break;
        default: set_error("relabel_sequential: unsupported destination dtype %d", dst.dtype); return CLE_ERR_DTYPE;
    }
    CLE_LAUNCH_CHECK("relabel apply");
    return CLE_OK;
}

__global__ void u32_to_f32_kernel(const uint32_t *__restrict__ s, float *__restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        d[i] = (float)s[i];
}

}  // namespace

size_t rank_workspace_bytes(uint64_t bits) {
    Arena a(nullptr, 0);
    take_rank(a, bits);
    return a.off;
}

size_t ccl_workspace_bytes(const Img &im) {
    Arena a(nullptr, 0);
    a.take<uint32_t>(im.n());   // u32 labels when the destination is f32
    take_rank(a, fkey_bits_for(im.n()));
    return a.off;
}

int ccl_dense(const Img &bin, uint32_t *lab, Arena &ws, cudaStream_t st, bool diamond) {
    const int64_t n = bin.n();
    Rank r = take_rank(ws, fkey_bits_for(n));
    if (!ws.ok()) { set_error("connected_components_labeling_box: workspace too small"); return CLE_ERR_WORKSPACE; }
    const Geo g = make_geo(bin);
    Rows R;
    R.WS = (uint32_t)((bin.W + 31) / 32);
    R.fWS = FastDiv(R.WS);
    R.nseg = (uint32_t)(bin.D * bin.H) * R.WS;
    const int rb = launch_blocks((int64_t)R.nseg * 32, kRowWarps * 32);
    switch (bin.dtype) {
        case CLE_U8: CLE_TRY(launch_ccl_init<uint8_t>(bin, lab, g, R, rb, st)); break;
        case CLE_U32: CLE_TRY(launch_ccl_init<uint32_t>(bin, lab, g, R, rb, st)); break;
        case CLE_F32: CLE_TRY(launch_ccl_init<float>(bin, lab, g, R, rb, st)); break;
        case CLE_U16: CLE_TRY(launch_ccl_init<uint16_t>(bin, lab, g, R, rb, st)); break;
        default: set_error("connected_components_labeling_box: unsupported dtype %d", bin.dtype); return CLE_ERR_DTYPE;
    }
    const int b = launch_blocks(n, kT);
    if (diamond) ccl_union_rows<true><<<rb, kRowWarps * 32, 0, st>>>(lab, g, R);
    else ccl_union_rows<false><<<rb, kRowWarps * 32, 0, st>>>(lab, g, R);
    ccl_flatten_rows<<<rb, kRowWarps * 32, 0, st>>>(lab, g, R);
    CLE_CUDA(cudaMemsetAsync(r.bitmap, 0, sizeof(uint32_t) * r.words, st));
    ccl_mark_dense<<<b, kT, 0, st>>>(lab, g, n, r.bitmap);
    CLE_LAUNCH_CHECK_N("ccl dense", 3);
    CLE_TRY(rank_build(r, st));
    ccl_label_dense<<<b, kT, 0, st>>>(lab, n, r.bitmap, r.prefix);
    CLE_LAUNCH_CHECK("ccl label");
    return CLE_OK;
}

int ccl_list(const Geo &g, int64_t n, uint32_t *lab, const uint32_t *list,
             const uint32_t *d_count, int64_t cap, Arena &ws, cudaStream_t st,
             uint32_t *d_nlabels) {
    Rank r = take_rank(ws, fkey_bits_for(n));
    if (!ws.ok()) { set_error("seed labeling: workspace too small"); return CLE_ERR_WORKSPACE; }
    const int b = launch_blocks(cap, kT);
    ccl_union_list<<<b, kT, 0, st>>>(lab, g, list, d_count);
    ccl_flatten_list<<<b, kT, 0, st>>>(lab, g, list, d_count);
    CLE_CUDA(cudaMemsetAsync(r.bitmap, 0, sizeof(uint32_t) * r.words, st));
    ccl_mark_list<<<b, kT, 0, st>>>(lab, g, list, d_count, r.bitmap);
    CLE_LAUNCH_CHECK_N("ccl list", 3);
    CLE_TRY(rank_build(r, st));
    ccl_label_list<<<b, kT, 0, st>>>(lab, list, d_count, r.bitmap, r.prefix);
    CLE_LAUNCH_CHECK("ccl list label");
    if (d_nlabels) {
        count_ranks_kernel<<<1, 1, 0, st>>>(r.bitmap, r.prefix, r.words, d_nlabels);
        CLE_LAUNCH_CHECK("label count");
    }
    return CLE_OK;
}

int ccl_to_dst(const uint32_t *lab, const Img &dst, cudaStream_t st) {
    if (dst.dtype == CLE_F32) {
        u32_to_f32_kernel<<<launch_blocks(dst.n(), kT), kT, 0, st>>>(lab, (float *)dst.data, dst.n());
        CLE_LAUNCH_CHECK("u32 to f32");
    }
    return CLE_OK;
}

size_t relabel_workspace_bytes(uint32_t max_label) {
    return rank_workspace_bytes((uint64_t)max_label + 1u);
}

int relabel_sequential(const Img &src, const Img &dst, uint32_t maxv, Arena &ws, cudaStream_t st) {
    CLE_TRY(same_shape(src, dst, "source", "output"));
    Rank r = take_rank(ws, (uint64_t)maxv + 1u);
    if (!ws.ok()) { set_error("relabel_sequential: workspace too small"); return CLE_ERR_WORKSPACE; }
    CLE_CUDA(cudaMemsetAsync(r.bitmap, 0, sizeof(uint32_t) * r.words, st));
    switch (src.dtype) {
        case CLE_U32: return relabel_typed<uint32_t>(src, dst, maxv, r, st);
        case CLE_F32: return relabel_typed<float>(src, dst, maxv, r, st);
        case CLE_U16: return relabel_typed<uint16_t>(src, dst, maxv, r, st);
        case CLE_U8: return relabel_typed<uint8_t>(src, dst, maxv, r, st);
        default: set_error("relabel_sequential: unsupported dtype %d", src.dtype); return CLE_ERR_DTYPE;
    }
}

}  // namespace cle
