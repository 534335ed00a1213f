// pipeline.cu -- voronoi_otsu_labeling (_tier9/_voronoi_otsu_labeling.py:49-73) as one
// stream-ordered sequence with no host round trip:
//   T = gaussian_blur(src, spot_sigma)            (blur.cu)
//   spots = detect_maxima_box(T)                  (maxima.cu; mean_box r=0 is a copy)
//   T = gaussian_blur(src, outline_sigma)
//   {min,max} -> histogram -> Otsu -> t32         (reduce.cu, all on the device)
//   seg = T > t32; seeds = spots & seg            (seed kernel below; emits the seed list
//                                                  and the seeds' initial CCL keys)
//   labels(seeds) = CCL                           (ccl.cu, list form)
//   labels = masked Voronoi growth inside seg     (voronoi.cu, frontier form)
// The label output buffer is the CCL parent store and the Voronoi state, so
// the only full-size scratch is T (f32), spots/seg (u8), the seed list and
// the two frontier arrays (which also serve as the blur's temporaries).
#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

struct Scalars {
    int status;
    uint32_t seed_count;
    uint32_t nlabels;        // labels of the last call (= its maximum label)
    uint32_t pad0;
    float minmax[2];
    float thr32;
    float pad;
    double thr;
    float hist[256];
};

__global__ void seeds_kernel(const float *__restrict__ T, const uint8_t *__restrict__ spots,
                             const float *__restrict__ d_thr32, Geo g, int64_t n,
                             uint8_t *__restrict__ seg, uint32_t *__restrict__ lab,
                             uint32_t *__restrict__ seeds, uint32_t *__restrict__ d_count) {
    const float t = *d_thr32;
    const int lane = threadIdx.x & 31;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n;
         base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        bool s = false, seed = false;
        uint32_t key = 0;
        if (i < n) {
            s = T[i] > t;
            seed = s && spots[i] != 0;
            if (seed) {
                uint32_t x, y, z;
                m2xyz(g, (uint32_t)i, x, y, z);
                key = xyz2k(g, x, y, z) + 1u;
            }
            seg[i] = s ? kMaskByte : 0;
            lab[i] = key;
        }
        const unsigned b = __ballot_sync(0xffffffffu, seed);
        if (b) {
            uint32_t base_pos = 0;
            const int leader = __ffs(b) - 1;
            if (lane == leader) base_pos = atomicAdd(d_count, (uint32_t)__popc(b));
            base_pos = __shfl_sync(0xffffffffu, base_pos, leader);
            if (seed) seeds[base_pos + __popc(b & ((1u << lane) - 1u))] = (uint32_t)i;
        }
    }
}

// Seeds of masked_voronoi_labeling with a 0/1 mask: seg = mask != 0,
// seed = binary != 0 inside the mask; seeds get their CCL key and are listed.
template <typename Tb, typename Tm>
__global__ void mask_seeds_kernel(const Tb *__restrict__ bin, const Tm *__restrict__ mask, Geo g,
                                  int64_t n, uint8_t *__restrict__ seg, uint32_t *__restrict__ lab,
                                  uint32_t *__restrict__ seeds, uint32_t *__restrict__ d_count) {
    const int lane = threadIdx.x & 31;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n;
         base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        bool seed = false;
        if (i < n) {
            const bool s = mask[i] != (Tm)0;
            seed = s && bin[i] != (Tb)0;
            uint32_t key = 0;
            if (seed) {
                uint32_t x, y, z;
                m2xyz(g, (uint32_t)i, x, y, z);
                key = xyz2k(g, x, y, z) + 1u;
            }
            seg[i] = s ? kMaskByte : 0;
            lab[i] = key;
        }
        const unsigned b = __ballot_sync(0xffffffffu, seed);
        if (b) {
            uint32_t base_pos = 0;
            const int leader = __ffs(b) - 1;
            if (lane == leader) base_pos = atomicAdd(d_count, (uint32_t)__popc(b));
            base_pos = __shfl_sync(0xffffffffu, base_pos, leader);
            if (seed) seeds[base_pos + __popc(b & ((1u << lane) - 1u))] = (uint32_t)i;
        }
    }
}

__global__ void u32_to_f32(const uint32_t *__restrict__ s, float *__restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        d[i] = (float)s[i];
}

struct Layout {
    Scalars *sc;
    float *T;
    uint8_t *spots, *seg;
    uint32_t *seeds;
    size_t fixed_end;
};

Layout take_layout(Arena &a, const Img &im) {
    Layout l;
    l.sc = a.take<Scalars>(1);
    l.T = a.take<float>(im.n());
    l.spots = a.take<uint8_t>(im.n());
    l.seg = a.take<uint8_t>(im.n());
    l.seeds = a.take<uint32_t>(im.n());
    l.fixed_end = a.off;
    return l;
}

struct BinLayout {
    Scalars *sc;
    uint8_t *seg;
    uint32_t *seeds;
    uint32_t *lab;   // used when the destination is float32
};

BinLayout take_bin_layout(Arena &a, const Img &im) {
    BinLayout l;
    l.sc = a.take<Scalars>(1);
    l.seg = a.take<uint8_t>(im.n());
    l.seeds = a.take<uint32_t>(im.n());
    l.lab = a.take<uint32_t>(im.n());
    return l;
}

template <typename Tb>
int launch_mask_seeds(const Img &bin, const Img &mask, const Geo &g, const BinLayout &l,
                      uint32_t *lab, cudaStream_t st) {
    const int64_t n = bin.n();
    const int b = launch_blocks(n, 256);
    switch (mask.dtype) {
        case CLE_U8: mask_seeds_kernel<Tb, uint8_t><<<b, 256, 0, st>>>((const Tb *)bin.data, (const uint8_t *)mask.data, g, n, l.seg, lab, l.seeds, &l.sc->seed_count); break;
        case CLE_F32: mask_seeds_kernel<Tb, float><<<b, 256, 0, st>>>((const Tb *)bin.data, (const float *)mask.data, g, n, l.seg, lab, l.seeds, &l.sc->seed_count); break;
        case CLE_U32: mask_seeds_kernel<Tb, uint32_t><<<b, 256, 0, st>>>((const Tb *)bin.data, (const uint32_t *)mask.data, g, n, l.seg, lab, l.seeds, &l.sc->seed_count); break;
        default: set_error("masked_voronoi_labeling: unsupported mask dtype %d", mask.dtype); return CLE_ERR_DTYPE;
    }
    CLE_LAUNCH_CHECK("mask seeds");
    return CLE_OK;
}

}  // namespace

size_t masked_voronoi_binary_workspace_bytes(const Img &im) {
    Arena a(nullptr, 0);
    take_bin_layout(a, im);
    size_t tail = std::max(rank_workspace_bytes(fkey_bits_for(im.n())), voronoi_grow_workspace_bytes(im));
    return a.off + tail;
}

int masked_voronoi_binary(const Img &bin, const Img &mask, const Img &dst, Arena &ws, cudaStream_t st,
                          const Limits &lim) {
    CLE_TRY(same_shape(bin, mask, "binary_source", "mask_image"));
    CLE_TRY(same_shape(bin, dst, "binary_source", "labeling_destination"));
    if (dst.dtype != CLE_U32 && dst.dtype != CLE_F32) {
        set_error("masked_voronoi_labeling: destination must be uint32 or float32");
        return CLE_ERR_DTYPE;
    }
    BinLayout l = take_bin_layout(ws, bin);
    const size_t tail_off = ws.off;
    if (!ws.measuring && ws.cap < masked_voronoi_binary_workspace_bytes(bin)) {
        set_error("masked_voronoi_labeling: workspace too small");
        return CLE_ERR_WORKSPACE;
    }
    CLE_CUDA(cudaMemsetAsync(l.sc, 0, sizeof(Scalars), st));
    uint32_t *lab = dst.dtype == CLE_U32 ? (uint32_t *)dst.data : l.lab;
    const Geo g = make_geo(bin);
    switch (bin.dtype) {
        case CLE_U8: CLE_TRY(launch_mask_seeds<uint8_t>(bin, mask, g, l, lab, st)); break;
        case CLE_F32: CLE_TRY(launch_mask_seeds<float>(bin, mask, g, l, lab, st)); break;
        case CLE_U32: CLE_TRY(launch_mask_seeds<uint32_t>(bin, mask, g, l, lab, st)); break;
        default: set_error("masked_voronoi_labeling: unsupported binary dtype %d", bin.dtype); return CLE_ERR_DTYPE;
    }
    CLE_TRY(ccl_list(g, bin.n(), lab, l.seeds, &l.sc->seed_count, bin.n(), ws, st, &l.sc->nlabels));
    ws.off = tail_off;
    CLE_TRY(voronoi_grow(bin, lab, l.seg, l.seeds, &l.sc->seed_count, &l.sc->nlabels, &l.sc->status, ws, st,
                         lim));
    if (dst.dtype == CLE_F32) {
        u32_to_f32<<<launch_blocks(dst.n(), 256), 256, 0, st>>>(lab, (float *)dst.data, dst.n());
        CLE_LAUNCH_CHECK("labels to f32");
    }
    return CLE_OK;
}

// ---- extend_labeling_via_voronoi / voronoi_labeling -------------------------
// _tier4/_extend_labeling_via_voronoi.py:13-60: the labels (uint32, any values)
// grow into every zero voxel with the onlyzero_overwrite_maximum box/diamond
// Jacobi steps until a step changes nothing -- the brick growth kernel with a
// mask that covers the whole image.  voronoi_labeling (_tier5/_voronoi_labeling.py:
// 8-40) is connected_components_labeling_box followed by that growth.
namespace {

template <typename T>
__global__ void to_labels_kernel(const T *__restrict__ src, uint32_t *__restrict__ lab, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const T v = src[i];
        uint32_t o;
        if constexpr (std::is_floating_point<T>::value)   // clij_convert_uint_sat
            o = !(v > (T)0) ? 0u : (v >= (T)4294967295.0 ? 0xFFFFFFFFu : (uint32_t)v);
        else if constexpr (std::is_signed<T>::value)
            o = v < (T)0 ? 0u : (uint32_t)v;
        else
            o = (uint32_t)v;
        lab[i] = o;
    }
}

constexpr int kSeedWarps = 8;

// One seed voxel per 8-voxel row segment (x aligned to 8) that holds a label;
// the segment lies in one growth brick (8 x by 4 y), so the 3x3x3 brick
// neighbourhood of the seed's brick covers every voxel next to a label of the
// segment.  A warp reads 32 x of one row.  One global atomic per CTA.
__global__ void __launch_bounds__(kSeedWarps * 32)
brick_seeds_kernel(const uint32_t *__restrict__ lab, uint32_t W, uint32_t WB, FastDiv fWB, uint32_t nb,
                   uint32_t *__restrict__ seeds, uint32_t *__restrict__ d_count) {
    __shared__ uint32_t s_n, s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t base = blockIdx.x * kSeedWarps; base < nb; base += gridDim.x * kSeedWarps) {
        if (threadIdx.x == 0) s_n = 0;
        __syncthreads();
        const uint32_t b = base + warp;
        uint32_t pos = 0, m = 0;
        bool has = false;
        if (b < nb) {
            const uint32_t r = fWB.div(b), xb = b - r * WB, x = xb * 32u + (uint32_t)lane;
            const unsigned bal = __ballot_sync(0xffffffffu, x < W && lab[r * W + x] != 0u);
            const unsigned seg8 = (bal >> (lane & 24)) & 0xFFu;   // this lane's 8-voxel segment
            has = (lane & 7) == 0 && seg8 != 0u;
            if (has) {
                m = r * W + xb * 32u + (uint32_t)(lane & 24) + (uint32_t)(__ffs(seg8) - 1);
                pos = atomicAdd(&s_n, 1u);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_base = s_n ? atomicAdd(d_count, s_n) : 0u;
        __syncthreads();
        if (has) seeds[s_base + pos] = m;
    }
}

struct ExtLayout {
    Scalars *sc;
    uint8_t *seg;
    uint32_t *seeds;
    uint32_t *lab;    // used when the destination is float32
};

ExtLayout take_ext_layout(Arena &a, const Img &im) {
    ExtLayout l;
    l.sc = a.take<Scalars>(1);
    l.seg = a.take<uint8_t>(im.n());
    l.seeds = a.take<uint32_t>((im.n() + 7) / 8 + (size_t)(im.D * im.H));
    l.lab = a.take<uint32_t>(im.n());
    return l;
}

// Grows `lab` in place over the whole image; status in l.sc.
int grow_everywhere(const Img &im, uint32_t *lab, ExtLayout &l, Arena &tail, cudaStream_t st,
                    const Limits &lim) {
    CLE_CUDA(cudaMemsetAsync(l.seg, 1, (size_t)im.n(), st));
    const uint32_t WB = (uint32_t)((im.W + 31) / 32);
    const uint32_t nb = (uint32_t)(im.D * im.H) * WB;
    brick_seeds_kernel<<<launch_blocks((int64_t)nb * 32, kSeedWarps * 32), kSeedWarps * 32, 0, st>>>(
        lab, (uint32_t)im.W, WB, FastDiv(WB), nb, l.seeds, &l.sc->seed_count);
    CLE_LAUNCH_CHECK("brick seeds");
    return voronoi_frontier(im, lab, l.seg, l.seeds, &l.sc->seed_count, &l.sc->status, tail, st, lim);
}

}  // namespace

size_t extend_voronoi_workspace_bytes(const Img &im) {
    Arena a(nullptr, 0);
    take_ext_layout(a, im);
    const size_t tail = std::max(ccl_workspace_bytes(im), voronoi_frontier_workspace_bytes(im));
    return a.off + tail;
}

int extend_labeling_via_voronoi(const Img &src, const Img &dst, Arena &ws, cudaStream_t st,
                                const Limits &lim) {
    CLE_TRY(same_shape(src, dst, "labeling_source", "labeling_destination"));
    if (dst.dtype != CLE_U32 && dst.dtype != CLE_F32) {
        set_error("extend_labeling_via_voronoi: destination must be uint32 or float32");
        return CLE_ERR_DTYPE;
    }
    ExtLayout l = take_ext_layout(ws, src);
    if (!ws.measuring && ws.cap < extend_voronoi_workspace_bytes(src)) {
        set_error("extend_labeling_via_voronoi: workspace too small");
        return CLE_ERR_WORKSPACE;
    }
    CLE_CUDA(cudaMemsetAsync(l.sc, 0, sizeof(Scalars), st));
    uint32_t *lab = dst.dtype == CLE_U32 ? (uint32_t *)dst.data : l.lab;
    const int64_t n = src.n();
    const int b = launch_blocks(n, 256);
    switch (src.dtype) {
        case CLE_U8: to_labels_kernel<uint8_t><<<b, 256, 0, st>>>((const uint8_t *)src.data, lab, n); break;
        case CLE_U16: to_labels_kernel<uint16_t><<<b, 256, 0, st>>>((const uint16_t *)src.data, lab, n); break;
        case CLE_U32:
            if (src.data != (void *)lab) to_labels_kernel<uint32_t><<<b, 256, 0, st>>>((const uint32_t *)src.data, lab, n);
            break;
        case CLE_I32: to_labels_kernel<int32_t><<<b, 256, 0, st>>>((const int32_t *)src.data, lab, n); break;
        case CLE_F32: to_labels_kernel<float><<<b, 256, 0, st>>>((const float *)src.data, lab, n); break;
        default: set_error("extend_labeling_via_voronoi: unsupported source dtype %d", src.dtype); return CLE_ERR_DTYPE;
    }
    CLE_LAUNCH_CHECK("labels");
    CLE_TRY(grow_everywhere(src, lab, l, ws, st, lim));
    if (dst.dtype == CLE_F32) {
        u32_to_f32<<<launch_blocks(n, 256), 256, 0, st>>>(lab, (float *)dst.data, n);
        CLE_LAUNCH_CHECK("labels to f32");
    }
    return CLE_OK;
}

int voronoi_labeling(const Img &bin, const Img &dst, Arena &ws, cudaStream_t st, const Limits &lim) {
    CLE_TRY(same_shape(bin, dst, "binary_source", "labeling_destination"));
    if (dst.dtype != CLE_U32 && dst.dtype != CLE_F32) {
        set_error("voronoi_labeling: destination must be uint32 or float32");
        return CLE_ERR_DTYPE;
    }
    ExtLayout l = take_ext_layout(ws, bin);
    const size_t tail_off = ws.off;
    if (!ws.measuring && ws.cap < extend_voronoi_workspace_bytes(bin)) {
        set_error("voronoi_labeling: workspace too small");
        return CLE_ERR_WORKSPACE;
    }
    CLE_CUDA(cudaMemsetAsync(l.sc, 0, sizeof(Scalars), st));
    uint32_t *lab = dst.dtype == CLE_U32 ? (uint32_t *)dst.data : l.lab;
    CLE_TRY(ccl_dense(bin, lab, ws, st));
    ws.off = tail_off;
    CLE_TRY(grow_everywhere(bin, lab, l, ws, st, lim));
    if (dst.dtype == CLE_F32) {
        u32_to_f32<<<launch_blocks(dst.n(), 256), 256, 0, st>>>(lab, (float *)dst.data, dst.n());
        CLE_LAUNCH_CHECK("labels to f32");
    }
    return CLE_OK;
}

int *workspace_status_ptr(void *ws) { return &reinterpret_cast<Scalars *>(ws)->status; }
uint32_t *workspace_label_count_ptr(void *ws) { return &reinterpret_cast<Scalars *>(ws)->nlabels; }

size_t vol_workspace_bytes(const Img &im) {
    Arena a(nullptr, 0);
    take_layout(a, im);
    const size_t base = a.off;
    // phase-dependent tail (max over the phases that use it)
    size_t tail = 0;
    tail = std::max(tail, separable_workspace_bytes(im));
    tail = std::max(tail, minmax_workspace_bytes(im) + histogram_workspace_bytes(im, 256));
    tail = std::max(tail, blur_minmax_workspace_bytes(im));
    tail = std::max(tail, rank_workspace_bytes(fkey_bits_for(im.n())));
    tail = std::max(tail, voronoi_grow_workspace_bytes(im));
    return base + tail;
}

int voronoi_otsu_labeling(const Img &src, const Img &dst, double spot_sigma, double outline_sigma,
                          Arena &ws, cudaStream_t st, const Limits &lim) {
    CLE_TRY(same_shape(src, dst, "source", "label_image_destination"));
    if (dst.dtype != CLE_U32 && dst.dtype != CLE_F32) {
        set_error("voronoi_otsu_labeling: destination must be uint32 or float32 (got %d)", dst.dtype);
        return CLE_ERR_DTYPE;
    }
    Layout l = take_layout(ws, src);
    const size_t tail_off = ws.off;
    if (!ws.ok() || (!ws.measuring && ws.cap < vol_workspace_bytes(src))) {
        set_error("voronoi_otsu_labeling: workspace too small (%zu < %zu)", ws.cap, vol_workspace_bytes(src));
        return CLE_ERR_WORKSPACE;
    }
    const int64_t n = src.n();
    stage_mark(0, st);
    CLE_CUDA(cudaMemsetAsync(l.sc, 0, sizeof(Scalars), st));

    // 1-3: blurs and maxima (the blur's temporaries live in the tail).  The
    // two blurs build their taps from the float32 sigma and the kernel size
    // int(8 sigma)|1, so equal float32 sigmas with equal kernel sizes give the
    // same image bit for bit: then it is computed once (with the min / max the
    // outline blur reduces) and serves both the spot detection and the
    // threshold, as the reference's second blur would have recomputed it.
    const bool same_blur = (float)spot_sigma == (float)outline_sigma &&
                           sigma_to_kernel_size(spot_sigma) == sigma_to_kernel_size(outline_sigma);
    if (same_blur) CLE_TRY(blur_minmax(src, l.T, spot_sigma, l.sc->minmax, ws, st, &l.sc->status));
    else CLE_TRY(gaussian_blur(src, l.T, spot_sigma, spot_sigma, spot_sigma, ws, st, &l.sc->status));
    stage_mark(1, st);
    ws.off = tail_off;
    Img Ti = src;
    Ti.data = l.T;
    Ti.dtype = CLE_F32;
    Img Si = src;
    Si.data = l.spots;
    Si.dtype = CLE_U8;
    // with one blur the maxima are found in the seed pass below (the spots
    // image is never stored)
    if (!same_blur) CLE_TRY(detect_maxima(Ti, Si, st));
    stage_mark(2, st);
    // the outline blur also reduces the blurred image's min / max (step 4)
    if (!same_blur) CLE_TRY(blur_minmax(src, l.T, outline_sigma, l.sc->minmax, ws, st, &l.sc->status));
    ws.off = tail_off;
    stage_mark(3, st);

    // 4-6: threshold on the device
    CLE_TRY(histogram(Ti, 256, l.sc->minmax, l.sc->hist, ws, st));
    ws.off = tail_off;
    CLE_TRY(otsu(l.sc->hist, l.sc->minmax, &l.sc->thr, &l.sc->thr32, st));
    stage_mark(4, st);

    // 7: segmentation, seeds, seed keys
    uint32_t *lab = (dst.dtype == CLE_U32) ? (uint32_t *)dst.data : (uint32_t *)l.T;
    const Geo g = make_geo(src);
    const float *Tsrc = l.T;
    if (dst.dtype == CLE_F32) {
        // the labels are built in T's buffer; the seed pass reads a copy in dst
        CLE_CUDA(cudaMemcpyAsync(dst.data, l.T, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
        Tsrc = (const float *)dst.data;
    }
    if (same_blur) {
        Img Tc = Ti;
        Tc.data = (void *)Tsrc;
        CLE_TRY(maxima_seeds(Tc, &l.sc->thr32, l.seg, lab, l.seeds, &l.sc->seed_count, st));
    } else {
        seeds_kernel<<<launch_blocks(n, 256), 256, 0, st>>>(Tsrc, l.spots, &l.sc->thr32, g, n, l.seg, lab, l.seeds, &l.sc->seed_count);
        CLE_LAUNCH_CHECK("seeds");
    }
    stage_mark(5, st);

    // 8: label the seeds
    CLE_TRY(ccl_list(g, n, lab, l.seeds, &l.sc->seed_count, n, ws, st, &l.sc->nlabels));
    ws.off = tail_off;
    stage_mark(6, st);

    // 9: grow inside the segmentation
    CLE_TRY(voronoi_grow(src, lab, l.seg, l.seeds, &l.sc->seed_count, &l.sc->nlabels, &l.sc->status, ws, st,
                         lim));
    ws.off = tail_off;
    stage_mark(7, st);

    if (dst.dtype == CLE_F32) {
        u32_to_f32<<<launch_blocks(n, 256), 256, 0, st>>>(lab, (float *)dst.data, n);
        CLE_LAUNCH_CHECK("labels to f32");
    }
    return CLE_OK;
}

}  // namespace cle
