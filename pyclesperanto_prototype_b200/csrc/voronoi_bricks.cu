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

// Exclusive prefix of v over the CTA (up to 1024 threads); total of the CTA in `total`.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *s_w, uint32_t &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (int)(blockDim.x >> 5);
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
        uint32_t w = lane < nw ? s_w[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) s_w[lane] = w;
    }
    __syncthreads();
    total = s_w[nw - 1];
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
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
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
template <typename St>
__device__ bool compact_queue(const BQueue &Qb, uint32_t *F, uint32_t *nsize, St *S, uint64_t barrier_ns,
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
                      const volatile int *cancel, unsigned long long *trace, BQueue Qb, int use_bitmap,
                      const int *gate) {
    __shared__ uint32_t s_red[kWPB];
    __shared__ uint32_t s_scan[kWPB];
    __shared__ uint32_t s_off[2];
    // after the key growth (below) this launch only runs when that kernel
    // handed the growth back (every CTA reads the same word)
    if (gate && *(const volatile int *)gate == 0) return;
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

// ---- growth by arrival keys ---------------------------------------------------
// The same labels as the Jacobi steps above, without a grid barrier per step.
// A voxel the growth labels has an arrival step A (the step that writes it)
// and a label; with s = A + 1 (seeds: s = 0) the reference's steps give
//   s(v) = min over labelled neighbours u of   s(u) + 1         for a face neighbour,
//                                              (s(u) + 1) | 1   for an edge / corner
//                                              neighbour (box steps only: odd s),
//   label(v) = the largest label among the neighbours that reach v at s(v).
// So v's key K = s << 24 | (0xFFFFFF - label) is the minimum over its
// neighbours of their keys sent through those two maps (the second map is
// applied to each neighbour before the minimum: it merges pairs of steps, so
// it does not commute with the minimum).  Re-evaluating voxels in any order
// reaches that fixpoint -- the s part only decreases, and the label part then
// settles in order of s -- so a warp relaxes its brick against the brick's
// halo until nothing changes within one visit, and a brick is visited again
// only when a neighbouring brick changes a voxel next to it.  Rounds of
// visits are separated by grid barriers; a round ends the growth when it
// queues nothing.
//
// The reference's loop stops at the first step that labels nothing: with S
// the smallest s >= 1 that no voxel holds, voxels of s > S stay unlabelled.
// Per-CTA counts of the voxels per s (kept up to date at every write) give S;
// only when some voxel holds an s above S does a last pass over the mask
// bytes set those labels back to 0.
//
// The label buffer holds plain labels throughout (0: unlabelled or outside
// the mask); a labelled voxel's s lives in its mask byte (bit 7: in the mask,
// bits 0-6: s, 127 while not yet known, as the seed passes write it), and
// its key is s << 24 | (label ^ 0xFFFFFF).  Labels above 2^24 - 1 or an s
// above kKeyMaxS do not fit: the kernel then leaves the labels as it found
// them (after an overflow it sets every grown voxel back to 0) and raises the
// gate word, and the brick kernel grows them instead.

constexpr uint32_t kKInf = 0xFFFFFFFFu;
constexpr uint32_t kKS1 = 0x01000000u;
constexpr uint32_t kKeyMaxS = 120;   // steps fit the mask byte's 7 bits (127 = not yet known)
constexpr int kKeyIters = 32;     // local iterations per visit; a brick still changing re-queues itself
#ifndef CLE_KEY_BT
#define CLE_KEY_BT 1024
#endif
constexpr int kKeyBT = CLE_KEY_BT; // threads per CTA of the key kernel (1024: 32 warps per SM, measured faster than 768 or 2 x 512)

struct KState {
    GridBarrier bar;
    int err;
    int gate;          // 1: the brick kernel grows the labels after this launch
    int overflow;      // an s above kKeyMaxS was reached
    uint32_t sizes[4];
    uint32_t rounds;   // diagnostics of the last launch: rounds run,
    uint32_t stop_s;   // S,
    uint32_t visits;   // brick visits
    int hist[256];     // grown voxels per s
};

// key of a voxel from its label p and mask byte sg (the arrival step in its
// low 7 bits once labelled; labels fit 24 bits).  A label read together with
// a step field still at 127 ("not yet known": the byte of a voxel another
// warp is labelling right now) counts as unlabelled -- a value that is never
// below the voxel's true key, and the writer queues this brick again.
__device__ __forceinline__ uint32_t key_of(uint32_t p, uint32_t sg) {
    return (p && (sg & 0x7Fu) != 0x7Fu) ? (((sg & 0x7Fu) << 24) | (p ^ 0x00FFFFFFu)) : kKInf;
}
// The two maps, with infinity kept: a real key's step is at most 127, so
// min(k, INF - S1) only changes infinity, which then maps to infinity again.
__device__ __forceinline__ uint32_t key_face(uint32_t k) { return min(k, kKInf - kKS1) + kKS1; }
__device__ __forceinline__ uint32_t key_diag(uint32_t k) { return (min(k, kKInf - kKS1) + kKS1) | kKS1; }

template <bool IS3D, int BZ, int KBT>
__global__ void __launch_bounds__(KBT, 1)
voronoi_keys_kernel(uint32_t *lab, uint8_t *seg, BGeo G, const uint32_t *seeds,
                    const uint32_t *d_seed_count, const uint32_t *d_max_label, uint32_t *B0, uint32_t *B1,
                    uint32_t *bstep, KState *S, int *d_status, uint32_t max_steps,
                    uint64_t loop_ns, uint64_t barrier_ns, const volatile int *cancel,
                    unsigned long long *trace, BQueue Qb, int use_bitmap) {
    constexpr int NW = KBT / 32;
    constexpr int ZR = IS3D ? 1 : 0;
    constexpr int K = BZ + 2 * ZR;
    __shared__ uint32_t s_red[NW];
    __shared__ uint32_t s_scan[NW];
    __shared__ uint32_t s_off[2];
    __shared__ int s_hist[256];
    const Geo &g = G.g;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    WarpAppender ap{&S->err, 0u};
    const uint64_t t_entry = global_ns();
    // labels that do not fit 24 bits: the brick kernel takes over (uniform)
    if (__ldcg(d_max_label) > 0x00FFFFFFu) {
        if (gtid == 0) S->gate = 1;
        return;
    }
    for (int i = threadIdx.x; i < 256; i += KBT) s_hist[i] = 0;

    // round 0: each seed's brick and the neighbouring bricks the seed touches
    // (a seed on a brick's face, edge or corner); the growth reaches every
    // other brick through a changed voxel next to it
    const uint32_t ns = __ldcg(d_seed_count);
    for (uint32_t base = blockIdx.x * NW; base < ns; base += gridDim.x * NW) {
        const uint32_t i = base + warp;
        if (i < ns) {
            const uint32_t m = __ldcg(seeds + i);
            if (lane == 0) seg[m] = 0x80u;   // in the mask, arrival step 0
            uint32_t x, y, z;
            m2xyz(g, m, x, y, z);
            const int dz = lane / 9 - 1, dyb = (lane / 3) % 3 - 1, dxb = lane % 3 - 1;
            const uint32_t xr = x % kBX, yr = y % kBY, zr = z % BZ;
            const bool touch = (dxb == 0 || (dxb < 0 ? xr == 0 : xr == kBX - 1)) &&
                               (dyb == 0 || (dyb < 0 ? yr == 0 : yr == kBY - 1)) &&
                               (dz == 0 || (dz < 0 ? zr == 0 : zr == (uint32_t)BZ - 1));
            const bool want = lane < 27 && (IS3D || dz == 0) && touch;
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
    if (use_bitmap && ok) ok = compact_queue(Qb, B0, &S->sizes[0], S, barrier_ns, s_red, s_scan, s_off);

    // the lane's column and halo voxel (as in the brick kernel)
    const int xl = lane & (kBX - 1), yl = lane / kBX;
    const bool x0 = xl == 0, x1 = xl == kBX - 1, y0 = yl == 0, y1 = yl == kBY - 1;
    const int src_h = yl == 0 ? xl : 8 + xl;
    const int src_s = (xl == 0 ? 16 : 20) + (yl & 3);
    const int src_q = 24 + (yl == kBY - 1 ? 2 : 0) + (xl == kBX - 1 ? 1 : 0);
    // the neighbouring brick lane d < 27 stands for in the queueing and the
    // presence test: its offset, the brick voxels (as ballot bits) that face
    // it, and the halo lanes that lie in it -- fixed for the whole launch
    const int qdz = lane / 9 - 1, qdy = (lane / 3) % 3 - 1, qdx = lane % 3 - 1;
    const bool qself = qdz == 0 && qdy == 0 && qdx == 0;
    const bool qlive = lane < 27 && (IS3D || qdz == 0);
    const unsigned qmask = (qdy < 0 ? 0x000000FFu : qdy > 0 ? 0xFF000000u : 0xFFFFFFFFu) &
                           (qdx < 0 ? 0x01010101u : qdx > 0 ? 0x80808080u : 0xFFFFFFFFu);
    const unsigned qhsel = qdy == 0 ? (qdx < 0 ? 0x000F0000u : 0x00F00000u)
                         : qdx == 0 ? (qdy < 0 ? 0x000000FFu : 0x0000FF00u)
                         : (1u << (24 + (qdy > 0 ? 2 : 0) + (qdx > 0 ? 1 : 0)));

    const uint64_t t_start = global_ns();
    // trace: the last two rows hold the set-up (round 0's queue) and the
    // finish (counts, S, conversion) times
    if (trace && gtid == 0) trace[4 * (kTraceSteps - 2)] = t_start - t_entry;
    const uint32_t max_rounds = max_steps > 0x0FFFFFFFu ? 0xFFFFFFFFu : 4u * max_steps + 64u;
    uint32_t r = 0, visits = 0;
    bool done = false;
    while (ok && r < max_rounds) {
        uint32_t iters = 0;
        if (gtid == 0) {
            if (global_ns() - t_start > loop_ns) atomicExch(&S->err, (int)CLE_ERR_ITER_LIMIT);
            else if (cancel && *cancel) atomicExch(&S->err, (int)CLE_ERR_CANCELLED);
        }
        const uint32_t *F = (r & 1) ? B1 : B0;
        uint32_t *Fn = (r & 1) ? B0 : B1;
        const uint32_t nB = __ldcg(&S->sizes[r & 3]);
        if (nB == 0u) { done = true; break; }
        if (*(volatile int *)&S->overflow) break;
        if (trace && gtid == 0 && r < kTraceSteps) {
            trace[4 * r] = global_ns() - t_start;
            trace[4 * r + 1] = nB;
        }
        if (gtid == 0) S->sizes[(r + 2) & 3] = 0u;
        uint32_t *nsize = &S->sizes[(r + 1) & 3];
        const bool bitmap = use_bitmap && nB >= kBitmapBricks;
        const uint32_t tag = r + 2;
        const uint32_t wstride = gridDim.x * NW, wbase = blockIdx.x * NW;
        // odd rounds walk the list (brick order) backwards: a brick visited
        // later in a round sees what earlier visits wrote, so alternating the
        // direction lets fronts in every direction cross several bricks per
        // round, as the plane sweeps do inside a brick
        const bool rev = (r & 1u) != 0u;
        auto entry = [&](uint32_t i) { return __ldcg(F + (rev ? nB - 1u - i : i)); };
        uint32_t bnext = (wbase + warp < nB) ? entry(wbase + warp) : 0u;
        for (uint32_t base = wbase; base < nB; base += wstride) {
            const uint32_t idx = base + warp;
            const uint32_t b = bnext;
            bnext = (idx + wstride < nB) ? entry(idx + wstride) : 0u;
            if (idx < nB) {
                if (lane == 0) ++visits;
                uint32_t zb, yb, xb;
                brick_zyx(G, b, zb, yb, xb);
                const int z0 = (int)(zb * BZ);
                const int x0b = (int)(xb * kBX), y0b = (int)(yb * kBY);
                const int x = x0b + xl, y = y0b + yl;
                const bool xyin = x < (int)g.W && y < (int)g.H;
                int hx_ = x0b, hy_ = y0b;
                if (lane < 8) { hx_ = x0b + lane; hy_ = y0b - 1; }
                else if (lane < 16) { hx_ = x0b + lane - 8; hy_ = y0b + kBY; }
                else if (lane < 24) { hx_ = lane < 20 ? x0b - 1 : x0b + kBX; hy_ = y0b + (lane & 3); }
                else { hx_ = (lane & 1) ? x0b + kBX : x0b - 1; hy_ = (lane & 2) ? y0b + kBY : y0b - 1; }
                const bool hin = lane < 28 && hx_ >= 0 && hy_ >= 0 && hx_ < (int)g.W && hy_ < (int)g.H;
                const uint32_t hoff = (uint32_t)clampi(hy_, 0, (int)g.H - 1) * g.W + (uint32_t)clampi(hx_, 0, (int)g.W - 1);
                const uint32_t coff = (uint32_t)min(y, (int)g.H - 1) * g.W + (uint32_t)min(x, (int)g.W - 1);
                // keys of planes z0 - 1 .. z0 + BZ; voxels outside the image are
                // no neighbour (key infinity), as the reference skips them
                uint32_t k[K], h[K];
                bool cm[K], hm[K];   // mask voxels: the lane's column, its halo voxel
                // a brick whose halo lies inside the image (most of them) needs
                // no clamps and no validity tests (warp-uniform)
                const bool inner = z0 >= ZR && z0 + BZ + ZR <= (int)g.D && x0b >= 1 && x0b + kBX < (int)g.W &&
                                   y0b >= 1 && y0b + kBY < (int)g.H;
                if (inner) {
                    const uint32_t HWp = g.H * g.W;
#pragma unroll
                    for (int q = 0; q < K; ++q) {
                        const uint32_t zo = (uint32_t)(z0 - ZR + q) * HWp;
                        const uint32_t kp = ld_cg(lab + zo + coff);
                        const uint32_t hp = lane < 28 ? ld_cg(lab + zo + hoff) : 0u;
                        const uint32_t ks = __ldcg(seg + zo + coff);
                        const uint32_t hs = lane < 28 ? (uint32_t)__ldcg(seg + zo + hoff) : 0u;
                        cm[q] = ks != 0u;
                        hm[q] = hs != 0u;
                        k[q] = key_of(kp, ks);
                        h[q] = key_of(hp, hs);   // lanes 28..31: label 0, infinity
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < K; ++q) {
                        const int zq = z0 - ZR + q;
                        const bool zin = zq >= 0 && zq < (int)g.D;
                        const uint32_t zo = (uint32_t)clampi(zq, 0, (int)g.D - 1) * g.H * g.W;
                        const uint32_t kp = ld_cg(lab + zo + coff);
                        const uint32_t hp = lane < 28 ? ld_cg(lab + zo + hoff) : 0u;
                        const uint32_t ks = __ldcg(seg + zo + coff);
                        const uint32_t hs = lane < 28 ? (uint32_t)__ldcg(seg + zo + hoff) : 0u;
                        cm[q] = zin && xyin && ks != 0u;
                        hm[q] = zin && hin && hs != 0u;
                        k[q] = (zin && xyin) ? key_of(kp, ks) : kKInf;
                        h[q] = (zin && hin) ? key_of(hp, hs) : kKInf;
                    }
                }
                // candidates: mask voxels that are not seeds (seeds have s = 0)
                bool cand[BZ];
                bool anyc = false;
#pragma unroll
                for (int j = 0; j < BZ; ++j) {
                    cand[j] = cm[j + ZR] && (k[j + ZR] >> 24) != 0u;
                    anyc |= cand[j];
                }
                // lane d < 27: does neighbouring brick d hold a candidate next to
                // this brick (in its halo)?  If not, nothing this brick writes can
                // change that brick, and it is not queued for it
                bool present = false;
                {
                    unsigned pres = 0u;
#pragma unroll
                    for (int q = 0; q < K; ++q) {
                        const unsigned cb = __ballot_sync(0xffffffffu, cm[q] && (k[q] >> 24) != 0u);
                        const unsigned hb = __ballot_sync(0xffffffffu, hm[q] && (h[q] >> 24) != 0u);
                        const bool inP = qdz < 0 ? q == 0 : (qdz > 0 ? q == K - 1 : (q >= ZR && q < ZR + BZ));
                        if (inP) pres |= (qdy == 0 && qdx == 0) ? cb : (hb & qhsel);
                    }
                    present = lane < 27 && pres != 0u;
                }
                if (!__any_sync(0xffffffffu, anyc)) {
                    // nothing here can change: never queue it again
                    if (lane == 0) {
                        atomicExch(bstep + b, 0xFFFFFFFFu);
                        atomicOr(Qb.done + (b >> 5), 1u << (b & 31u));
                    }
                    continue;
                }
                // halo terms, fixed during the visit: per plane the halo row's
                // x-minimum (y edge) and the halo column's value (x edge) of the
                // box term, and the face term's halo row / column voxels
                uint32_t HX[BZ], SZ[BZ], HC[BZ], SC[BZ];
                {
                    uint32_t dh[K];
#pragma unroll
                    for (int q = 0; q < K; ++q) dh[q] = key_diag(h[q]);
#pragma unroll
                    for (int j = 0; j < BZ; ++j) {
                        const int kc = j + ZR;
                        uint32_t dhm = dh[kc];
                        if (ZR) dhm = min(dhm, min(dh[kc - ZR], dh[kc + ZR]));
                        const uint32_t hz = __shfl_sync(0xffffffffu, dhm, src_h);
                        const uint32_t sz = __shfl_sync(0xffffffffu, dhm, src_s);
                        const uint32_t qz = __shfl_sync(0xffffffffu, dhm, src_q);
                        const uint32_t hl = __shfl_up_sync(0xffffffffu, hz, 1), hr = __shfl_down_sync(0xffffffffu, hz, 1);
                        const uint32_t hc = __shfl_sync(0xffffffffu, h[kc], src_h);
                        const uint32_t sc = __shfl_sync(0xffffffffu, h[kc], src_s);
                        // only the brick's edge lanes see the halo; elsewhere
                        // infinity, the minimum's neutral value
                        HX[j] = (y0 || y1) ? min(hz, min(x0 ? qz : hl, x1 ? qz : hr)) : kKInf;
                        SZ[j] = (x0 || x1) ? sz : kKInf;
                        HC[j] = (y0 || y1) ? hc : kKInf;
                        SC[j] = (x0 || x1) ? sc : kKInf;
                    }
                }
                uint32_t k0[BZ], dk[K];
#pragma unroll
                for (int j = 0; j < BZ; ++j) k0[j] = k[j + ZR];
#pragma unroll
                for (int q = 0; q < K; ++q) dk[q] = key_diag(k[q]);
                // Gauss-Seidel over the planes (upward on even iterations,
                // downward on odd ones); a plane is evaluated again only after
                // it or a plane next to it changed
                unsigned cmask = 0u;
#pragma unroll
                for (int j = 0; j < BZ; ++j)
                    if (__any_sync(0xffffffffu, cand[j])) cmask |= 1u << j;
                unsigned act = cmask, nxt = 0u;
                auto relax = [&](auto J) {
                    constexpr int j = decltype(J)::value;
                    if constexpr (j < BZ) {
                        constexpr int kc = j + ZR;
                        if ((act >> j) & 1u) {
                            // box term over the map-2 keys: planes, then x, then y.
                            // Shuffles within a row (width 8) and across the
                            // brick's rows give an edge lane its own value, which
                            // a minimum may include (a voxel's own key never
                            // beats its true candidates); the halo enters through
                            // SZ / HX, infinity on interior lanes.
                            uint32_t dz = dk[kc];
                            if constexpr (ZR > 0) dz = min(dz, min(dk[kc - 1], dk[kc + 1]));
                            const uint32_t cl = __shfl_up_sync(0xffffffffu, dz, 1, kBX);
                            const uint32_t cr = __shfl_down_sync(0xffffffffu, dz, 1, kBX);
                            const uint32_t rx = min(min(dz, SZ[j]), min(cl, cr));
                            const uint32_t ru = __shfl_up_sync(0xffffffffu, rx, kBX), rd = __shfl_down_sync(0xffffffffu, rx, kBX);
                            const uint32_t bm = min(min(rx, HX[j]), min(ru, rd));
                            // face term over the raw keys (the same edge rule)
                            const uint32_t v = k[kc];
                            const uint32_t fl = __shfl_up_sync(0xffffffffu, v, 1, kBX), fr = __shfl_down_sync(0xffffffffu, v, 1, kBX);
                            const uint32_t fu = __shfl_up_sync(0xffffffffu, v, kBX), fd = __shfl_down_sync(0xffffffffu, v, kBX);
                            uint32_t fm = min(min(min(fl, fr), min(fu, fd)), min(SC[j], HC[j]));
                            if constexpr (ZR > 0) fm = min(fm, min(k[kc - 1], k[kc + 1]));
                            const uint32_t nk = cand[j] ? min(key_face(fm), bm) : v;
                            const bool c = nk != v;
                            k[kc] = nk;                  // unchanged lanes store their own value
                            dk[kc] = key_diag(nk);
                            if (__any_sync(0xffffffffu, c)) {
                                const unsigned nb3 = ((7u << j) >> 1) & cmask;   // planes j-1 .. j+1
                                nxt |= nb3;
                                act |= nb3;   // the plane the sweep reaches next sees it now
                            }
                        }
                    }
                };
                using I0 = std::integral_constant<int, 0>;
                using I1 = std::integral_constant<int, 1>;
                using I2 = std::integral_constant<int, 2>;
                using I3 = std::integral_constant<int, 3>;
                static_assert(BZ <= 4, "the plane sweep is unrolled for up to 4 planes");
                bool conv = false;
                int it = 0;
                for (; it < kKeyIters; ++it) {
                    nxt = 0u;
                    if (it & 1) { relax(I3{}); relax(I2{}); relax(I1{}); relax(I0{}); }
                    else        { relax(I0{}); relax(I1{}); relax(I2{}); relax(I3{}); }
                    act = nxt;
                    if (!act) { conv = true; break; }
                }
                if (lane == 0) iters += (uint32_t)it + 1u;
                // write the changed voxels, keep the per-s counts, queue the
                // bricks next to changed voxels (and this one if still changing)
                unsigned chb[BZ], chall = 0u;
                bool over = false;
#pragma unroll
                for (int j = 0; j < BZ; ++j) {
                    const uint32_t kn = k[j + ZR];
                    const bool c = kn != k0[j];
                    if (c) {
                        const uint32_t m = ((uint32_t)(z0 + j) * g.H + (uint32_t)y) * g.W + (uint32_t)x;
                        // steps above kKeyMaxS raise the overflow below; the
                        // clamp keeps such a step from wrapping into a seed's 0
                        __stcg(seg + m, (uint8_t)(0x80u | min(kn >> 24, 126u)));
                        st_cg(lab + m, (kn & 0x00FFFFFFu) ^ 0x00FFFFFFu);
                        if (k0[j] != kKInf) atomicSub(&s_hist[k0[j] >> 24], 1);
                        atomicAdd(&s_hist[kn >> 24], 1);
                        over |= (kn >> 24) > kKeyMaxS;
                    }
                    chb[j] = __ballot_sync(0xffffffffu, c);
                    chall |= chb[j];
                }
                if (over) atomicExch(&S->overflow, 1);
                // this brick again if it is still changing, a neighbour when a
                // changed voxel faces it and it holds a candidate next to them
                bool want = false;
                if (qlive) {
                    const unsigned sel = (qdz < 0 ? chb[0] : (qdz > 0 ? chb[BZ - 1] : chall)) & qmask;
                    want = qself ? !conv : (sel != 0u && present);
                }
                if (bitmap) {
                    const uint32_t zz = zb + (uint32_t)qdz, yy = yb + (uint32_t)qdy, xx = xb + (uint32_t)qdx;
                    if (want && zz < G.DB && yy < G.HB && xx < G.WB)   // unsigned: -1 wraps above
                        atomicOr(Qb.q + (((zz * G.HB + yy) * G.WB + xx) >> 5), 1u << (((zz * G.HB + yy) * G.WB + xx) & 31u));
                } else {
                    queue_neighbours(G, zb, yb, xb, want, tag, bstep, ap);
                }
            }
            if (!bitmap) ap.maybe_flush(Fn, nsize);
        }
        if (!bitmap) ap.flush(Fn, nsize);
        if (trace) {
            const uint32_t is = block_total(iters, s_red);
            if (threadIdx.x == 0 && r < kTraceSteps && is) atomicAdd(trace + 4 * r + 2, (unsigned long long)is);
        }
        ok = grid_sync(&S->bar, &S->err, barrier_ns);
        if (bitmap && ok) ok = compact_queue(Qb, Fn, nsize, S, barrier_ns, s_red, s_scan, s_off);
        if (trace && gtid == 0 && r < kTraceSteps) trace[4 * r + 3] = global_ns() - t_start;
        ++r;
    }
    // ---- finish: S from the counts, the cut of voxels that arrived after S ----
    if (trace && gtid == 0) trace[4 * (kTraceSteps - 1)] = global_ns() - t_start;
    const uint32_t vs = block_total(visits, s_red);
    if (threadIdx.x == 0 && vs) atomicAdd(&S->visits, vs);
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += KBT)
        if (s_hist[i]) atomicAdd(&S->hist[i], s_hist[i]);
    if (ok) ok = grid_sync(&S->bar, &S->err, barrier_ns);
    const bool overflow = *(volatile int *)&S->overflow != 0;
    if (ok && !done && !overflow) ok = false;   // round bound reached
    if (!ok && !overflow) {
        if (gtid == 0) {
            const int e = *(volatile int *)&S->err;
            *d_status = e ? e : (int)CLE_ERR_ITER_LIMIT;
            S->rounds = r;
        }
        return;
    }
    // S = the smallest s >= 1 that no voxel holds, and whether any voxel holds
    // a larger s (warp 0 of each CTA)
    if (warp == 0) {
        uint32_t stop = 128u;
        for (int c = 0; c < 4 && stop == 128u; ++c) {
            const int sidx = 32 * c + lane;
            const unsigned empty = __ballot_sync(0xffffffffu, sidx >= 1 && __ldcg(&S->hist[sidx]) == 0);
            if (empty) stop = (uint32_t)(32 * c + __ffs(empty) - 1);
        }
        bool beyond = false;
        for (int c = 0; c < 4; ++c) {
            const int sidx = 32 * c + lane;
            beyond |= sidx > (int)stop && __ldcg(&S->hist[sidx]) != 0;
        }
        beyond = __any_sync(0xffffffffu, beyond);
        if (lane == 0) {
            s_off[0] = overflow ? 0u : stop;         // 0: keep no grown voxel
            s_off[1] = (overflow || beyond) ? 1u : 0u;
        }
    }
    __syncthreads();
    const uint32_t stop = s_off[0];
    const bool cut = s_off[1] != 0u;
    if (cut) {
        // labels of voxels that arrived after step S (or, after an overflow,
        // of every grown voxel) go back to 0: a pass over the mask bytes
        const int64_t nvox = (int64_t)g.D * g.H * g.W;
        for (int64_t m = (int64_t)blockIdx.x * KBT + threadIdx.x; m < nvox; m += (int64_t)gridDim.x * KBT) {
            const uint32_t sg = (uint32_t)__ldcg(seg + m);
            if (sg != 0u && (sg & 0x7Fu) > stop && (sg & 0x7Fu) != 0x7Fu && ld_cg(lab + m) != 0u) st_cg(lab + (size_t)m, 0u);
        }
    }
    if (trace) {
        __syncthreads();
        if (threadIdx.x == 0) atomicMax(trace + 4 * (kTraceSteps - 1) + 3, (unsigned long long)(global_ns() - t_start));
    }
    if (gtid == 0) {
        S->rounds = r;
        S->stop_s = stop;
        if (overflow) S->gate = 1;                          // labels restored; the brick kernel grows them
        else if (stop > max_steps) *d_status = (int)CLE_ERR_ITER_LIMIT;   // the reference needs S steps
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
                     const Limits &lim, const int *gate) {
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
    // behind the key kernel (gate set) the trace stays that kernel's
    unsigned long long *trace = gate ? nullptr
        : (unsigned long long *)profile_trace_buffer(4 * kTraceSteps * sizeof(unsigned long long), st);
    void *args[] = {&lab, (void *)&seg, &G, (void *)&seeds, (void *)&d_seed_count, &B0, &B1, &Mv, &Pf,
                    &bstep, &S, &d_status, &max_steps, &loop_ns, &barrier_ns, (void *)&cancel, &trace, &Qb,
                    &use_bitmap, (void *)&gate};
    CLE_CUDA(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kBT), args, kBBufBytes, st));
    count_launches(1);
    return CLE_OK;
}

namespace {

size_t keys_part_bytes(const Img &im) {
    const size_t nb = brick_count(im);
    Arena a(nullptr, 0);
    a.take<KState>(1);
    a.take<uint32_t>(nb);               // list 0
    a.take<uint32_t>(nb);               // list 1
    a.take<uint32_t>(nb);               // per-brick round tags
    a.take<uint32_t>((nb + 31) / 32);   // queue bitmap
    a.take<uint32_t>((nb + 31) / 32);   // bricks without candidates
    a.take<uint32_t>(2048);             // per-CTA counts of the compaction
    return a.off;
}

}  // namespace

size_t voronoi_grow_workspace_bytes(const Img &im) {
    return voronoi_frontier_workspace_bytes(im) + keys_part_bytes(im);
}

int voronoi_grow(const Img &im, uint32_t *lab, uint8_t *seg, const uint32_t *seeds,
                 const uint32_t *d_seed_count, const uint32_t *d_max_label, int *d_status, Arena &ws,
                 cudaStream_t st, const Limits &lim) {
    // the key kernel's state sits behind the brick kernel's workspace, so the
    // gate word survives that kernel's set-up
    const size_t off0 = ws.off;
    ws.off = off0 + voronoi_frontier_workspace_bytes(im);
    const size_t nb = brick_count(im);
    KState *S = ws.take<KState>(1);
    uint32_t *B0 = ws.take<uint32_t>(nb);
    uint32_t *B1 = ws.take<uint32_t>(nb);
    uint32_t *bstep = ws.take<uint32_t>(nb);
    BQueue Qb;
    Qb.nwords = (uint32_t)((nb + 31) / 32);
    Qb.q = ws.take<uint32_t>(Qb.nwords);
    Qb.done = ws.take<uint32_t>(Qb.nwords);
    Qb.ccount = ws.take<uint32_t>(2048);
    if (!ws.ok()) { set_error("masked_voronoi_labeling: workspace too small"); return CLE_ERR_WORKSPACE; }
    CLE_CUDA(cudaMemsetAsync(S, 0, sizeof(KState), st));
    CLE_CUDA(cudaMemsetAsync(bstep, 0, sizeof(uint32_t) * nb, st));
    // q and done are adjacent: one clear
    CLE_CUDA(cudaMemsetAsync(Qb.q, 0, (size_t)((char *)(Qb.done + Qb.nwords) - (char *)Qb.q), st));
    BGeo G;
    G.g = make_geo(im);
    G.WB = bricks_x(im);
    G.HB = bricks_y(im);
    G.DB = bricks_z(im);
    G.fWB = FastDiv(G.WB);
    G.fHB = FastDiv(G.HB);
    G.is3d = im.ndim == 3 ? 1 : 0;
    uint32_t max_steps = lim.steps_for(im.n());
    uint64_t loop_ns = lim.loop_ns, barrier_ns = lim.barrier_ns;
    const volatile int *cancel = lim.cancel;
    const void *kern = G.is3d ? (const void *)voronoi_keys_kernel<true, kBZ3, kKeyBT>
                              : (const void *)voronoi_keys_kernel<false, 1, kKeyBT>;
    const size_t smem = sizeof(uint32_t) * kSlice * (kKeyBT / 32);
    CLE_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0;
    CLE_CUDA(cudaGetDevice(&dev));
    int per_sm = 0;
    CLE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kKeyBT, smem));
    if (per_sm < 1) { set_error("masked_voronoi_labeling: kernel does not fit on an SM"); return CLE_ERR_CUDA; }
    const int64_t want = std::max<int64_t>(1, (int64_t)(nb + 4 * (kKeyBT / 32) - 1) / (4 * (kKeyBT / 32)));
    const int grid = (int)std::min<int64_t>(std::min<int64_t>(want, (int64_t)per_sm * cooperative_ctas(dev, lim)), 2048);
    unsigned long long *trace =
        (unsigned long long *)profile_trace_buffer(4 * kTraceSteps * sizeof(unsigned long long), st);
    int use_bitmap = im.n() > kWideVoxels ? 1 : 0;
    void *args[] = {&lab, (void *)&seg, &G, (void *)&seeds, (void *)&d_seed_count, (void *)&d_max_label,
                    &B0, &B1, &bstep, &S, &d_status, &max_steps, &loop_ns, &barrier_ns,
                    (void *)&cancel, &trace, &Qb, &use_bitmap};
    CLE_CUDA(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kKeyBT), args, smem, st));
    count_launches(1);
    // the brick kernel, which returns at once unless the gate was raised
    ws.off = off0;
    return voronoi_frontier(im, lab, seg, seeds, d_seed_count, d_status, ws, st, lim, &S->gate);
}

}  // namespace cle
