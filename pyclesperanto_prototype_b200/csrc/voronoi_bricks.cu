// voronoi_bricks.cu -- the Voronoi growth of voronoi_otsu_labeling, masked_voronoi_labeling
// with a 0/1 mask, extend_labeling_via_voronoi and voronoi_labeling
// (_tier5/_masked_voronoi_labeling.py:44-76 with a 0/1 mask and seeds inside it,
// _tier4/_extend_labeling_via_voronoi.py:30-56 with the whole image as mask).
//
// The reference's Jacobi steps (box stencil on even steps, face stencil on odd
// steps, a voxel rewritten only while 0 with the maximum over the stencil
// including itself, stop at the first step that changes nothing) run on
// bricks of 8 x by 4 y voxels by BZ z planes (BZ = 4 in 3D, 1 in 2D), one
// warp each (lane = 8 y + x, marching the brick's planes).  Only active
// bricks are visited -- those that may hold a voxel able to change in this
// step -- so the work per step follows the growth front.  A front crosses a
// compact brick in few steps, so a brick is visited few times; a warp reads
// per z plane its 32 voxels as 4 aligned 32-byte row segments plus the
// brick's halo (all BZ + 2 planes issued at once), and x / y neighbours come
// by warp shuffles.
//
// A step is two phases separated by grid barriers:
//   A  every active brick computes its candidates' new values from the state
//      of the previous step (candidates: mask voxels still 0);
//   B  new labels are written, and the bricks of the next step are queued:
//      the 3x3x3 brick neighbourhood of every brick that changed, plus any
//      brick with a voxel that the face stencil could not reach but the box
//      stencil will (it changes at the next step).
// Queueing deduplicates with an atomicMax on a per-brick step tag, so the
// label buffer holds labels only; a brick left without unlabelled mask voxels
// gets the maximal tag and is never queued again.  Every voxel that can change at a step lies
// in a queued brick (a voxel whose labelled neighbour is older was already
// visited and either changed or was re-queued), so the result equals the
// reference's dense iteration.  Once few bricks remain active, one CTA
// finishes the remaining steps with block barriers instead of grid barriers.
#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

constexpr int kBT = 1024;                       // threads per CTA
constexpr int kWPB = kBT / 32;                  // warps per CTA
constexpr int kSlice = 256;                     // per-warp append slice (entries)
constexpr size_t kBBufBytes = sizeof(uint32_t) * kSlice * kWPB;
constexpr uint32_t kTailBricks = 128;           // single-CTA finish at or below this
constexpr uint32_t kBitmapBricks = 16384;       // bitmap queueing at or above this (large volumes)
#ifndef CLE_VORONOI_WIDE_VOXELS
#define CLE_VORONOI_WIDE_VOXELS (int64_t(64) << 20)
#endif
constexpr int64_t kWideVoxels = CLE_VORONOI_WIDE_VOXELS;  // 2 CTAs per SM above this many voxels
constexpr uint32_t kTraceSteps = 256;

struct BState {
    GridBarrier bar;
    int err;
    int done;
    uint32_t sizes[4];
    uint32_t changes[4];
    uint32_t steps;
    uint32_t pad[3];
};

constexpr int kBX = 8;                          // brick: 8 x ...
constexpr int kBY = 4;                          // ... by 4 y voxels of one z plane
static_assert(kBX == 8 && kBY == 4, "the brick-edge lane masks assume 8x4 bricks");

// Bricks of 3D images hold kBZ planes (8 x 4 x kBZ voxels, one warp, each
// lane owning one (x, y) column of the brick): a warp loads the kBZ + 2
// planes a visit needs at once, so the per-visit memory latency is shared by
// kBZ planes, and a front crosses a taller brick in fewer visits (a CPU
// replay of the growth on light-sheet data: 0.64M visits of 8x4x4 bricks
// against 1.46M of 8x4x1).  2D images use 8 x 4 x 1.
#ifndef CLE_VORONOI_BZ
#define CLE_VORONOI_BZ 4
#endif
constexpr int kBZ3 = CLE_VORONOI_BZ;

struct BGeo {
    Geo g;
    uint32_t WB, HB, DB; // bricks along x, y, z
    FastDiv fWB, fHB;
    int is3d;
};

// brick b -> (zb, yb, xb)
__device__ __forceinline__ void brick_zyx(const BGeo &G, uint32_t b, uint32_t &zb, uint32_t &yb, uint32_t &xb) {
    const uint32_t r = G.fWB.div(b);
    xb = b - r * G.WB;
    zb = G.fHB.div(r);
    yb = r - zb * G.HB;
}

// Per-warp append slice in shared memory, flushed to a global list by the
// warp alone, so no CTA barrier sits inside the brick loops.
struct WarpAppender {
    int *err;
    uint32_t cnt;       // warp-uniform fill
    // this warp's kSlice entries of the dynamic shared buffer
    __device__ __forceinline__ uint32_t *buf() const {
        extern __shared__ uint32_t s_buf[];
        return s_buf + (threadIdx.x >> 5) * kSlice;
    }
    // Warp-wide: lanes with `take` append v.  A call appends at most 27
    // entries and maybe_flush empties the slice above kSlice - 27, so it
    // cannot overflow; the check turns a broken bound into an error status.
    __device__ __forceinline__ void push(bool take, uint32_t v) {
        const unsigned bal = __ballot_sync(0xffffffffu, take);
        if (!bal) return;
        if (take) {
            const uint32_t pos = cnt + (uint32_t)__popc(bal & ((1u << (threadIdx.x & 31)) - 1u));
            if (pos < (uint32_t)kSlice) buf()[pos] = v;
            else atomicExch(err, (int)CLE_ERR_ITER_LIMIT);
        }
        cnt += (uint32_t)__popc(bal);
        __syncwarp();
    }
    __device__ __forceinline__ void flush(uint32_t *dst, uint32_t *dst_size) {
        const uint32_t k = min(cnt, (uint32_t)kSlice);
        if (!k) return;
        const int lane = threadIdx.x & 31;
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(dst_size, k);
        base = __shfl_sync(0xffffffffu, base, 0);
        const uint32_t *b = buf();
        for (uint32_t i = lane; i < k; i += 32) dst[base + i] = b[i];
        __syncwarp();
        cnt = 0;
    }
    __device__ __forceinline__ void maybe_flush(uint32_t *dst, uint32_t *dst_size) {
        if (cnt > (uint32_t)(kSlice - 27)) flush(dst, dst_size);
    }
};

// The next step's bricks while several CTAs run: phase B sets their bits in
// `q` (fire-and-forget atomicOr, so repeats cost nothing), bricks without an
// unlabelled mask voxel are set in `done`, and a two-pass grid compaction
// turns q & ~done into the next list in brick-index order -- warps that run
// at the same time then visit neighbouring bricks, whose halo rows and label
// sectors they share in L2.  `ccount` holds one count per CTA.
struct BQueue {
    uint32_t *q, *done, *ccount;
    uint32_t nwords;
};

// Brick at offset `lane` (0..26) of the 3x3x3 neighbourhood, if inside.
__device__ __forceinline__ bool neighbour_brick(const BGeo &G, uint32_t zb, uint32_t yb, uint32_t xb, int lane,
                                                uint32_t &nb) {
    const int dz = lane / 9 - 1, dyb = (lane / 3) % 3 - 1, dxb = lane % 3 - 1;
    const int zz = (int)zb + dz, yy = (int)yb + dyb, xx = (int)xb + dxb;
    if (zz < 0 || yy < 0 || xx < 0 || zz >= (int)G.DB || yy >= (int)G.HB || xx >= (int)G.WB) return false;
    nb = ((uint32_t)zz * G.HB + (uint32_t)yy) * G.WB + (uint32_t)xx;
    return true;
}

// Exclusive prefix of v over the CTA (kBT threads); total of the CTA in `total`.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *s_w, uint32_t &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) s_w[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kWPB ? s_w[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kWPB) s_w[lane] = w;
    }
    __syncthreads();
    total = s_w[kWPB - 1];
    return (warp ? s_w[warp - 1] : 0u) + x - v;
}

__device__ __forceinline__ uint32_t block_total(uint32_t v, uint32_t *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t s = 0;
    if (threadIdx.x == 0)
        for (int i = 0; i < kWPB; ++i) s += red[i];
    return s;   // thread 0
}



// Queues bricks (z+dz, yb+dyb, xb+dxb) for the step tagged `tag`; lane k of
// the warp handles offset k of the 3x3x3 neighbourhood when want.  Warp-wide.
__device__ __forceinline__ void queue_neighbours(const BGeo &G, uint32_t zb, uint32_t yb, uint32_t xb,
                                                 bool want, uint32_t tag, uint32_t *bstep,
                                                 WarpAppender &ap) {
    const int lane = threadIdx.x & 31;
    bool take = false;
    uint32_t nb = 0;
    if (want && lane < 27) {
        const int dz = lane / 9 - 1, dyb = (lane / 3) % 3 - 1, dxb = lane % 3 - 1;
        const int zz = (int)zb + dz, yy = (int)yb + dyb, xx = (int)xb + dxb;
        if (zz >= 0 && yy >= 0 && xx >= 0 && zz < (int)G.DB && yy < (int)G.HB && xx < (int)G.WB) {
            nb = ((uint32_t)zz * G.HB + (uint32_t)yy) * G.WB + (uint32_t)xx;
            take = atomicMax(bstep + nb, tag) < tag;
        }
    }
    ap.push(take, nb);
}

// Two-pass grid compaction of the queue bitmap (q & ~done) into the list F in
// brick-index order, its length in *nsize; clears q.  Grid-wide: every CTA
// calls it; returns false when a barrier gave up.
__device__ bool compact_queue(const BQueue &Qb, uint32_t *F, uint32_t *nsize, BState *S, uint64_t barrier_ns,
                              uint32_t *s_red, uint32_t *s_scan, uint32_t *s_off) {
    // pass 1: each CTA counts the queued bricks of its contiguous range of
    // bitmap words
    const uint32_t per = (Qb.nwords + gridDim.x - 1) / gridDim.x;
    const uint32_t w0 = min(Qb.nwords, blockIdx.x * per), w1 = min(Qb.nwords, w0 + per);
    uint32_t c = 0;
    for (uint32_t w = w0 + threadIdx.x; w < w1; w += blockDim.x)
        c += (uint32_t)__popc(ld_cg(Qb.q + w) & ~ld_cg(Qb.done + w));
    const uint32_t cs = block_total(c, s_red);
    if (threadIdx.x == 0) st_cg(Qb.ccount + blockIdx.x, cs);
    if (!grid_sync(&S->bar, &S->err, barrier_ns)) return false;
    // pass 2: the CTA's offset, then its bricks in index order
    uint32_t before = 0, all = 0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
        const uint32_t v = ld_cg(Qb.ccount + i);
        all += v;
        if (i < blockIdx.x) before += v;
    }
    const uint32_t before_t = block_total(before, s_red);
    if (threadIdx.x == 0) s_off[0] = before_t;
    const uint32_t all_t = block_total(all, s_red);
    if (threadIdx.x == 0) s_off[1] = all_t;
    __syncthreads();
    uint32_t off = s_off[0];
    if (blockIdx.x == 0 && threadIdx.x == 0) *nsize = s_off[1];
    for (uint32_t base = w0; base < w1; base += blockDim.x) {
        const uint32_t w = base + threadIdx.x;
        uint32_t bits = 0;
        if (w < w1) {
            bits = ld_cg(Qb.q + w) & ~ld_cg(Qb.done + w);
            st_cg(Qb.q + w, 0u);
        }
        uint32_t total = 0;
        uint32_t pos = off + block_excl_scan((uint32_t)__popc(bits), s_scan, total);
        while (bits) {
            const uint32_t bit = (uint32_t)(__ffs(bits) - 1);
            bits &= bits - 1u;
            F[pos++] = w * 32u + bit;
        }
        off += total;
    }
    return grid_sync(&S->bar, &S->err, barrier_ns);
}

// MINB CTAs per SM: 1 for volumes whose labels mostly stay in L2 (a visit
// waits on L2 hits), 2 for larger ones (2x the warps to hide DRAM latency).
// BZ planes per brick.
template <bool IS3D, int BZ, int MINB>
__global__ void __launch_bounds__(kBT, MINB)
voronoi_bricks_kernel(uint32_t *lab, const uint8_t *__restrict__ seg, BGeo G,
                      const uint32_t *seeds, const uint32_t *d_seed_count, uint32_t *B0,
                      uint32_t *B1, uint32_t *Mv, uint32_t *Pf, uint32_t *bstep, BState *S, int *d_status,
                      uint32_t max_steps, uint64_t loop_ns, uint64_t barrier_ns,
                      const volatile int *cancel, unsigned long long *trace, BQueue Qb, int use_bitmap) {
    __shared__ uint32_t s_red[kWPB];
    __shared__ uint32_t s_scan[kWPB];
    __shared__ uint32_t s_off[2];
    const Geo &g = G.g;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    WarpAppender ap{&S->err, 0u};
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    constexpr int ZR = IS3D ? 1 : 0;

    // step 0's bricks: the brick neighbourhoods of the seeds (tag 1), one
    // seed per warp per round so a round queues at most 27 bricks per warp
    const uint32_t ns = __ldcg(d_seed_count);
    for (uint32_t base = blockIdx.x * kWPB; base < ns; base += gridDim.x * kWPB) {
        const uint32_t i = base + warp;
        if (i < ns) {
            uint32_t x, y, z;
            m2xyz(g, __ldcg(seeds + i), x, y, z);
            const bool want = lane < 27 && (IS3D || (lane / 9) == 1);
            if (use_bitmap) {
                uint32_t nb = 0;
                if (want && neighbour_brick(G, z / BZ, y / kBY, x / kBX, lane, nb))
                    atomicOr(Qb.q + (nb >> 5), 1u << (nb & 31u));
            } else {
                queue_neighbours(G, z / BZ, y / kBY, x / kBX, want, 1u, bstep, ap);
            }
        }
        if (!use_bitmap) ap.maybe_flush(B0, &S->sizes[0]);
    }
    if (!use_bitmap) ap.flush(B0, &S->sizes[0]);
    bool ok = grid_sync(&S->bar, &S->err, barrier_ns);
    // large volumes: step 0's list in brick order as well
    if (use_bitmap && ok) ok = compact_queue(Qb, B0, &S->sizes[0], S, barrier_ns, s_red, s_scan, s_off);

    const uint64_t t_start = global_ns();
    uint32_t t = 0;
    bool done = false, tail = false;
    while (ok && t < max_steps) {
        if (gtid == 0) {
            if (global_ns() - t_start > loop_ns) atomicExch(&S->err, (int)CLE_ERR_ITER_LIMIT);
            else if (cancel && *cancel) atomicExch(&S->err, (int)CLE_ERR_CANCELLED);
        }
        const uint32_t *F = (t & 1) ? B1 : B0;
        uint32_t *Fn = (t & 1) ? B0 : B1;
        const uint32_t nB = __ldcg(&S->sizes[t & 3]);
        if (!tail && nB <= kTailBricks) {
            tail = true;                      // uniform: nB was read after a barrier
            if (blockIdx.x != 0) break;       // CTA 0 finishes alone
        }
        // many bricks on a large volume: the next list goes through the
        // queue bitmap (brick order, two more barriers); otherwise appends
        const bool bitmap = use_bitmap && !tail && nB >= kBitmapBricks;
        const uint32_t wstride = tail ? kWPB : gridDim.x * kWPB;
        const uint32_t wbase = tail ? 0 : blockIdx.x * kWPB;
        const bool box = (t & 1) == 0;
        // ---- phase A ---------------------------------------------------
        uint32_t changed = 0;
        // the next round's list entry is loaded one round ahead, so a visit
        // waits for one memory latency (its rows) instead of two
        uint32_t bnext = (wbase + warp < nB) ? __ldcg(F + wbase + warp) : 0u;
        for (uint32_t base = wbase; base < nB; base += wstride) {
            const uint32_t idx = base + warp;
            const uint32_t b = bnext;
            bnext = (idx + wstride < nB) ? __ldcg(F + idx + wstride) : 0u;
            if (idx >= nB) continue;
            uint32_t zb, yb, xb;
            brick_zyx(G, b, zb, yb, xb);
            const int z0 = (int)(zb * BZ);
            const int xl = lane & (kBX - 1), yl = lane / kBX;
            const int x = (int)(xb * kBX) + xl, y = (int)(yb * kBY) + yl;
            const int xc = min(x, (int)g.W - 1), yc = min(y, (int)g.H - 1);
            const bool xyin = x < (int)g.W && y < (int)g.H;
            // per z plane: c the lane's voxel, and one voxel of the brick's halo
            // per lane (28 of them, clamped to the image): lanes 0-7 the row
            // y - 1, 8-15 the row y + 4, 16-19 the column x - 1, 20-23 the
            // column x + 8, 24-27 the corners; lanes that need a halo voxel
            // fetch it by shuffle.  Planes z0 - 1 .. z0 + BZ (clamped), all
            // loads issued before any is used.
            constexpr int K = BZ + 2 * ZR;
            const int x0b = (int)(xb * kBX), y0b = (int)(yb * kBY);
            int hx_ = x0b, hy_ = y0b;
            if (lane < 8) { hx_ = x0b + lane; hy_ = y0b - 1; }
            else if (lane < 16) { hx_ = x0b + lane - 8; hy_ = y0b + kBY; }
            else if (lane < 24) { hx_ = lane < 20 ? x0b - 1 : x0b + kBX; hy_ = y0b + (lane & 3); }
            else { hx_ = (lane & 1) ? x0b + kBX : x0b - 1; hy_ = (lane & 2) ? y0b + kBY : y0b - 1; }
            const uint32_t hoff = (uint32_t)clampi(hy_, 0, (int)g.H - 1) * g.W + (uint32_t)clampi(hx_, 0, (int)g.W - 1);
            const uint32_t coff = (uint32_t)yc * g.W + (uint32_t)xc;
            uint32_t c[K], hv[K];
            bool inm[BZ];
#pragma unroll
            for (int j = 0; j < BZ; ++j)
                inm[j] = xyin && z0 + j < (int)g.D &&
                         seg[(uint32_t)(z0 + j) * g.H * g.W + coff] != 0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const uint32_t zz = (uint32_t)clampi(z0 - ZR + k, 0, (int)g.D - 1);
                const uint32_t *P = lab + zz * g.H * g.W;
                c[k] = ld_cg(P + coff);
                hv[k] = lane < 28 ? ld_cg(P + hoff) : 0u;
            }
            bool remain = false, pl = false;
#pragma unroll
            for (int j = 0; j < BZ; ++j) {
                const int kc = j + ZR;              // the plane's index in c / hv
                const bool cand = inm[j] && c[kc] == 0u;
                uint32_t out = 0;
                if (__any_sync(0xffffffffu, cand)) {
                    // the halo voxels this lane needs: h its halo row's (first /
                    // last brick row), s its halo column's (first / last brick
                    // column), q the corner (both)
                    const int src_h = yl == 0 ? xl : 8 + xl;
                    const int src_s = (xl == 0 ? 16 : 20) + (yl & 3);
                    const int src_q = 24 + (yl == kBY - 1 ? 2 : 0) + (xl == kBX - 1 ? 1 : 0);
                    const bool x0 = xl == 0, x1 = xl == kBX - 1, y0 = yl == 0, y1 = yl == kBY - 1;
                    // box: the maximum over the planes, then over x - 1 .. x + 1 (the
                    // lane's row and its halo row), then over y - 1 .. y + 1
                    uint32_t cz = c[kc], hm = hv[kc];
                    if (ZR) {
                        cz = max(cz, max(c[kc - ZR], c[kc + ZR]));
                        hm = max(hm, max(hv[kc - ZR], hv[kc + ZR]));
                    }
                    const uint32_t hz = __shfl_sync(0xffffffffu, hm, src_h);
                    const uint32_t sz = __shfl_sync(0xffffffffu, hm, src_s);
                    const uint32_t qz = __shfl_sync(0xffffffffu, hm, src_q);
                    const uint32_t cl = __shfl_up_sync(0xffffffffu, cz, 1), cr = __shfl_down_sync(0xffffffffu, cz, 1);
                    const uint32_t hl = __shfl_up_sync(0xffffffffu, hz, 1), hr = __shfl_down_sync(0xffffffffu, hz, 1);
                    const uint32_t rx = max(cz, max(x0 ? sz : cl, x1 ? sz : cr));
                    const uint32_t hx = max(hz, max(x0 ? qz : hl, x1 ? qz : hr));
                    const uint32_t ru = __shfl_up_sync(0xffffffffu, rx, kBX), rd = __shfl_down_sync(0xffffffffu, rx, kBX);
                    const uint32_t bm = max(rx, max(y0 ? hx : ru, y1 ? hx : rd));
                    // face: the plane at x +- 1 and y +- 1, the planes z +- 1 at (x, y)
                    const uint32_t v = c[kc];
                    const uint32_t fl = __shfl_up_sync(0xffffffffu, v, 1), fr = __shfl_down_sync(0xffffffffu, v, 1);
                    const uint32_t fu = __shfl_up_sync(0xffffffffu, v, kBX), fd = __shfl_down_sync(0xffffffffu, v, kBX);
                    const uint32_t hc = __shfl_sync(0xffffffffu, hv[kc], src_h);
                    const uint32_t sc = __shfl_sync(0xffffffffu, hv[kc], src_s);
                    uint32_t dm = max(max(x0 ? sc : fl, x1 ? sc : fr), max(y0 ? hc : fu, y1 ? hc : fd));
                    if (ZR) dm = max(dm, max(c[kc - ZR], c[kc + ZR]));
                    if (cand) {
                        const uint32_t m = box ? bm : dm;
                        out = m;
                        pl |= m == 0u && bm != 0u;   // face stencil missed, the box stencil will hit
                        changed += (m != 0u);
                        remain |= (m == 0u);
                    }
                }
                Mv[((size_t)idx * BZ + j) * 32 + lane] = out;
            }
            const bool pend = __any_sync(0xffffffffu, pl);
            if (lane == 0) Pf[idx] = pend ? 1u : 0u;
            // no unlabelled mask voxel left after this step: never queue it again
            if (!__any_sync(0xffffffffu, remain) && lane == 0) {
                atomicExch(bstep + b, 0xFFFFFFFFu);
                atomicOr(Qb.done + (b >> 5), 1u << (b & 31u));
            }
        }
        const uint32_t bs = block_total(changed, s_red);
        if (threadIdx.x == 0 && bs) atomicAdd(&S->changes[t & 3], bs);
        if (!tail) ok = grid_sync(&S->bar, &S->err, barrier_ns);
        else { __syncthreads(); ok = *(volatile int *)&S->err == 0; }
        if (!ok) break;
        const uint32_t nchanged = __ldcg(&S->changes[t & 3]);
        if (trace && gtid == 0 && t < kTraceSteps) {
            trace[4 * t] = global_ns() - t_start;
            trace[4 * t + 1] = nB;
            trace[4 * t + 2] = nchanged;
        }
        if (nchanged == 0u) { done = true; break; }
        // ---- phase B ---------------------------------------------------
        if (gtid == 0) {
            S->changes[(t + 2) & 3] = 0u;
            S->sizes[(t + 2) & 3] = 0u;
        }
        uint32_t *nsize = &S->sizes[(t + 1) & 3];
        const uint32_t tag = t + 2;
        for (uint32_t base = wbase; base < nB; base += wstride) {
            const uint32_t idx = base + warp;
            if (idx < nB) {
                const uint32_t b = __ldcg(F + idx);
                uint32_t m[BZ];
#pragma unroll
                for (int j = 0; j < BZ; ++j) m[j] = Mv[((size_t)idx * BZ + j) * 32 + lane];
                const bool pend = __ldcg(Pf + idx) != 0u;
                uint32_t zb, yb, xb;
                brick_zyx(G, b, zb, yb, xb);
                const uint32_t x = xb * kBX + (uint32_t)(lane & (kBX - 1)), y = yb * kBY + (uint32_t)(lane / kBX);
                unsigned ch[BZ], chall = 0u;
#pragma unroll
                for (int j = 0; j < BZ; ++j) {
                    if (m[j]) st_cg(lab + ((zb * BZ + (uint32_t)j) * g.H + y) * g.W + x, m[j]);
                    ch[j] = __ballot_sync(0xffffffffu, m[j] != 0u);
                    chall |= ch[j];
                }
                bool want = false;
                if (lane < 27) {
                    const int dz = lane / 9 - 1, dyb = (lane / 3) % 3 - 1, dxb = lane % 3 - 1;
                    if (IS3D || dz == 0) {
                        // changed voxels next to brick (dz, dyb, dxb): the first / last
                        // plane, brick row and column
                        unsigned sel = dz < 0 ? ch[0] : (dz > 0 ? ch[BZ - 1] : chall);
                        if (dyb < 0) sel &= 0x000000FFu;
                        else if (dyb > 0) sel &= 0xFF000000u;
                        if (dxb < 0) sel &= 0x01010101u;
                        else if (dxb > 0) sel &= 0x80808080u;
                        want = sel != 0u;
                        if (pend && dz == 0 && dyb == 0 && dxb == 0) want = true;
                    }
                }
                if (bitmap) {
                    uint32_t nb = 0;
                    if (want && lane < 27 && neighbour_brick(G, zb, yb, xb, lane, nb))
                        atomicOr(Qb.q + (nb >> 5), 1u << (nb & 31u));
                } else {
                    queue_neighbours(G, zb, yb, xb, want, tag, bstep, ap);
                }
            }
            if (!bitmap) ap.maybe_flush(Fn, nsize);
        }
        if (!bitmap) ap.flush(Fn, nsize);
        if (!tail) ok = grid_sync(&S->bar, &S->err, barrier_ns);
        else { __syncthreads(); ok = *(volatile int *)&S->err == 0; }
        if (bitmap && ok) ok = compact_queue(Qb, Fn, nsize, S, barrier_ns, s_red, s_scan, s_off);
        if (trace && gtid == 0 && t < kTraceSteps) trace[4 * t + 3] = global_ns() - t_start;
        ++t;
    }
    if (gtid == 0) {
        S->steps = t + 1;
        S->done = done ? 1 : 0;
        const int e = *(volatile int *)&S->err;
        // the caller cleared the word; an earlier stage's error stays
        if (!done) *d_status = e ? e : (int)CLE_ERR_ITER_LIMIT;
    }
}

int brick_planes(const Img &im) { return im.ndim == 3 ? kBZ3 : 1; }
uint32_t bricks_x(const Img &im) { return (uint32_t)((im.W + kBX - 1) / kBX); }
uint32_t bricks_y(const Img &im) { return (uint32_t)((im.H + kBY - 1) / kBY); }
uint32_t bricks_z(const Img &im) { return (uint32_t)((im.D + brick_planes(im) - 1) / brick_planes(im)); }
uint32_t brick_count(const Img &im) { return bricks_z(im) * bricks_y(im) * bricks_x(im); }

}  // namespace

size_t voronoi_frontier_workspace_bytes(const Img &im) {
    const size_t nb = brick_count(im);
    Arena a(nullptr, 0);
    a.take<BState>(1);
    a.take<uint32_t>(nb);        // list 0
    a.take<uint32_t>(nb);        // list 1
    a.take<uint32_t>(nb);        // per-brick step tags
    a.take<uint32_t>(nb * 32 * (size_t)brick_planes(im));   // per-voxel phase-A results
    a.take<uint32_t>(nb);        // per-entry pending flags
    a.take<uint32_t>((nb + 31) / 32);   // queue bitmap
    a.take<uint32_t>((nb + 31) / 32);   // finished-brick bitmap
    a.take<uint32_t>(2048);             // per-CTA counts of the compaction
    return a.off;
}

int voronoi_frontier(const Img &im, uint32_t *lab, const uint8_t *seg, const uint32_t *seeds,
                     const uint32_t *d_seed_count, int *d_status, Arena &ws, cudaStream_t st,
                     const Limits &lim) {
    const size_t nb = brick_count(im);
    BState *S = ws.take<BState>(1);
    uint32_t *B0 = ws.take<uint32_t>(nb);
    uint32_t *B1 = ws.take<uint32_t>(nb);
    uint32_t *bstep = ws.take<uint32_t>(nb);
    uint32_t *Mv = ws.take<uint32_t>(nb * 32 * (size_t)brick_planes(im));
    uint32_t *Pf = ws.take<uint32_t>(nb);
    BQueue Qb;
    Qb.nwords = (uint32_t)((nb + 31) / 32);
    Qb.q = ws.take<uint32_t>(Qb.nwords);
    Qb.done = ws.take<uint32_t>(Qb.nwords);
    Qb.ccount = ws.take<uint32_t>(2048);
    if (!ws.ok()) { set_error("masked_voronoi_labeling: workspace too small"); return CLE_ERR_WORKSPACE; }
    CLE_CUDA(cudaMemsetAsync(Qb.q, 0, sizeof(uint32_t) * (size_t)Qb.nwords, st));
    CLE_CUDA(cudaMemsetAsync(Qb.done, 0, sizeof(uint32_t) * (size_t)Qb.nwords, st));
    CLE_CUDA(cudaMemsetAsync(S, 0, sizeof(BState), st));
    CLE_CUDA(cudaMemsetAsync(bstep, 0, sizeof(uint32_t) * nb, st));
    BGeo G;
    G.g = make_geo(im);
    G.WB = bricks_x(im);
    G.HB = bricks_y(im);
    G.DB = bricks_z(im);
    G.fWB = FastDiv(G.WB);
    G.fHB = FastDiv(G.HB);
    G.is3d = im.ndim == 3 ? 1 : 0;
    uint32_t max_steps = lim.steps_for(im.n());   // each step that changes labels >= 1 voxel
    uint64_t loop_ns = lim.loop_ns, barrier_ns = lim.barrier_ns;
    const volatile int *cancel = lim.cancel;
    // 3D (kBZ3-plane bricks, 64 registers): one CTA per SM, the measured best
    // (the 2-CTA form spills: light-sheet growth 6.98 vs 5.18 ms); 2D keeps
    // 2 CTAs per SM above kWideVoxels
    const int wide = (G.is3d == 0 && im.n() > kWideVoxels) ? 1 : 0;
    const void *kerns[2][2] = {
        {(const void *)voronoi_bricks_kernel<false, 1, 1>, (const void *)voronoi_bricks_kernel<false, 1, 2>},
        {(const void *)voronoi_bricks_kernel<true, kBZ3, 1>, (const void *)voronoi_bricks_kernel<true, kBZ3, 1>}};
    const void *kern = kerns[G.is3d][wide];
    // the sorted bitmap queue pays off where labels do not stay in L2 (on the
    // 33.5M-voxel nuclei volume the append queue is faster: 0.56 vs 0.69 ms)
    int use_bitmap = im.n() > kWideVoxels ? 1 : 0;
    // set on every call: the attribute belongs to the current device's context
    CLE_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBBufBytes));
    int dev = 0;
    CLE_CUDA(cudaGetDevice(&dev));
    int per_sm = 0;
    CLE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBT, kBBufBytes));
    if (per_sm < 1) { set_error("masked_voronoi_labeling: kernel does not fit on an SM"); return CLE_ERR_CUDA; }
    const int64_t want = std::max<int64_t>(1, (int64_t)(nb + 4 * kWPB - 1) / (4 * kWPB));
    const int grid = (int)std::min<int64_t>(std::min<int64_t>(want, (int64_t)per_sm * cooperative_ctas(dev, lim)), 2048);
    unsigned long long *trace =
        (unsigned long long *)profile_trace_buffer(4 * kTraceSteps * sizeof(unsigned long long), st);
    void *args[] = {&lab, (void *)&seg, &G, (void *)&seeds, (void *)&d_seed_count, &B0, &B1, &Mv, &Pf,
                    &bstep, &S, &d_status, &max_steps, &loop_ns, &barrier_ns, (void *)&cancel, &trace, &Qb,
                    &use_bitmap};
    CLE_CUDA(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kBT), args, kBBufBytes, st));
    count_launches(1);
    return CLE_OK;
}

}  // namespace cle
