// batch.cu -- the batched form of voronoi_otsu_labeling behind the C ABI
// (cle_vol_batch_plan / cle_vol_batch_launch).
//
// The reference runs each tile as its own host-driven sequence
// (_tier9/_voronoi_otsu_labeling.py:57-71).  Here a plan fixes a set of tiles
// (shapes and dtypes), the sigmas and the loop options once; a launch then
// runs every tile's pipeline on the plan's lanes -- CUDA streams forked from
// the caller's stream with an event and joined back into it -- so a whole
// batch is ordered on the caller's stream, with no host work per tile beyond
// the launches, and can be captured into one CUDA graph by the caller.
//
// Tiles go to lanes longest first (greedy on voxel count); a lane's tiles run
// one after another on one workspace slice sized for its largest tile.  While
// several lanes run, each lane's cooperative growth launch is capped at its
// share of the SMs (passed with every call).  The lane count comes from the
// caller, or, with lanes = 0, from the tuned table in batch_tuning.h (written
// by pyclesperanto_prototype_b200/autotune.py from measurements).  A status
// word on the device collects the maximum of every tile's loop status.
#include <algorithm>
#include <cstdio>
#include <new>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "batch_tuning.h"

struct cle_vol_batch {
    int device = 0;
    double spot = 2.0, outline = 2.0;
    cle::Limits lim;
    std::vector<cle::Img> tiles;              // shapes and dtypes (data unused)
    std::vector<std::vector<int>> lane_tiles;
    std::vector<size_t> lane_off;             // workspace slice of each lane
    size_t ws_bytes = 0;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> join;
    cudaEvent_t fork = nullptr;
};

namespace cle {

namespace {

__global__ void status_max_kernel(const int *__restrict__ word, int *__restrict__ out) {
    const int v = *word;
    if (v) atomicMax(out, v);
}

// Lanes for a batch from the tuned table: the entry of the batch's mean tile
// size class, capped by the tile count.
int tuned_lanes(const std::vector<Img> &tiles) {
    double mean = 0.0;
    for (const Img &t : tiles) mean += (double)t.n();
    mean /= (double)std::max<size_t>(tiles.size(), 1);
    int lanes = kBatchTuning[0].lanes;
    for (const BatchTuning &e : kBatchTuning)
        if (mean >= e.min_mean_voxels) lanes = e.lanes;
    return std::max(1, std::min<int>(lanes, (int)tiles.size()));
}

void release(cle_vol_batch *p) {
    for (cudaStream_t s : p->streams) cudaStreamDestroy(s);
    for (cudaEvent_t e : p->join) cudaEventDestroy(e);
    if (p->fork) cudaEventDestroy(p->fork);
    delete p;
}

}  // namespace

}  // namespace cle

using namespace cle;

extern "C" {

int cle_vol_batch_plan(const cle_tensor *tiles, int n_tiles, double spot_sigma, double outline_sigma,
                       int lanes, const cle_call_options *options, cle_vol_batch **plan) {
    if (!plan) { set_error("vol_batch_plan: null plan pointer"); return CLE_ERR_ARG; }
    *plan = nullptr;
    if (!tiles || n_tiles < 1) { set_error("vol_batch_plan: no tiles"); return CLE_ERR_ARG; }
    if (lanes < 0 || lanes > 64) { set_error("vol_batch_plan: lanes must be 0 (tuned) .. 64, got %d", lanes); return CLE_ERR_ARG; }
    Limits lim;
    CLE_TRY(limits_from(options, lim));
    cle_vol_batch *p = new (std::nothrow) cle_vol_batch();
    if (!p) { set_error("vol_batch_plan: out of host memory"); return CLE_ERR_ARG; }
    p->spot = spot_sigma;
    p->outline = outline_sigma;
    p->tiles.resize((size_t)n_tiles);
    for (int i = 0; i < n_tiles; ++i) {
        char name[32];
        snprintf(name, sizeof(name), "tiles[%d]", i);
        Img im;
        int s = to_img(&tiles[i], im, name);
        if (s == CLE_OK && im.dtype != CLE_U8 && im.dtype != CLE_U16 && im.dtype != CLE_F32) {
            set_error("vol_batch_plan: %s must be uint8, uint16 or float32", name);
            s = CLE_ERR_DTYPE;
        }
        if (s != CLE_OK) { release(p); return s; }
        if (i > 0 && tiles[i].device != tiles[0].device) {
            set_error("vol_batch_plan: all tiles must be on one device");
            release(p);
            return CLE_ERR_ARG;
        }
        p->tiles[(size_t)i] = im;
    }
    p->device = tiles[0].device;
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess || (p->device >= 0 && p->device != cur && cudaSetDevice(p->device) != cudaSuccess)) {
        set_error("vol_batch_plan: cannot use device %d", p->device);
        release(p);
        return CLE_ERR_CUDA;
    }
    if (p->device < 0) p->device = cur;
    const int L = lanes ? std::min(lanes, n_tiles) : tuned_lanes(p->tiles);
    // longest first, each tile to the lane with the fewest voxels so far
    std::vector<int> order((size_t)n_tiles);
    for (int i = 0; i < n_tiles; ++i) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return p->tiles[(size_t)a].n() > p->tiles[(size_t)b].n(); });
    std::vector<int64_t> load((size_t)L, 0);
    p->lane_tiles.assign((size_t)L, {});
    for (int i : order) {
        const size_t k = (size_t)(std::min_element(load.begin(), load.end()) - load.begin());
        p->lane_tiles[k].push_back(i);
        load[k] += p->tiles[(size_t)i].n();
    }
    size_t off = 0;
    for (int k = 0; k < L; ++k) {
        size_t need = 0;
        for (int i : p->lane_tiles[(size_t)k]) need = std::max(need, vol_workspace_bytes(p->tiles[(size_t)i]));
        p->lane_off.push_back(off);
        off += (need + 255) & ~size_t(255);
    }
    p->ws_bytes = off;
    p->lim = lim;
    if (L > 1 && lim.coop_ctas == 0) p->lim.coop_ctas = std::max(1, num_sms(p->device) / L);
    cudaError_t e = cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming);
    for (int k = 0; k < L && e == cudaSuccess; ++k) {
        cudaStream_t s = nullptr;
        cudaEvent_t j = nullptr;
        e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e == cudaSuccess) p->streams.push_back(s);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&j, cudaEventDisableTiming);
        if (e == cudaSuccess) p->join.push_back(j);
    }
    if (cur != p->device) cudaSetDevice(cur);
    if (e != cudaSuccess) {
        const int s = cuda_error(e, "vol_batch_plan streams");
        release(p);
        return s;
    }
    *plan = p;
    return CLE_OK;
}

size_t cle_vol_batch_workspace_bytes(const cle_vol_batch *plan) { return plan ? plan->ws_bytes : 0; }

int cle_vol_batch_lanes(const cle_vol_batch *plan) { return plan ? (int)plan->streams.size() : 0; }

int cle_vol_batch_launch(const cle_vol_batch *p, const cle_tensor *tiles, const cle_tensor *labels,
                         void *workspace, size_t workspace_bytes, int32_t *d_status, void *stream) {
    if (!p) { set_error("vol_batch_launch: null plan"); return CLE_ERR_ARG; }
    if (!tiles || !labels || !d_status) { set_error("vol_batch_launch: null tiles, labels or status"); return CLE_ERR_ARG; }
    if (p->ws_bytes && (!workspace || workspace_bytes < p->ws_bytes)) {
        set_error("vol_batch_launch: workspace of %zu bytes needed, %zu given", p->ws_bytes, workspace ? workspace_bytes : (size_t)0);
        return CLE_ERR_WORKSPACE;
    }
    if (reinterpret_cast<uintptr_t>(workspace) & 255) { set_error("vol_batch_launch: workspace must be 256-byte aligned"); return CLE_ERR_WORKSPACE; }
    const size_t n = p->tiles.size();
    std::vector<Img> src(n), dst(n);
    for (size_t i = 0; i < n; ++i) {
        char name[32];
        snprintf(name, sizeof(name), "tiles[%zu]", i);
        CLE_TRY(to_img(&tiles[i], src[i], name));
        snprintf(name, sizeof(name), "labels[%zu]", i);
        CLE_TRY(to_img(&labels[i], dst[i], name));
        const Img &t = p->tiles[i];
        if (src[i].D != t.D || src[i].H != t.H || src[i].W != t.W || src[i].dtype != t.dtype || src[i].ndim != t.ndim) {
            set_error("vol_batch_launch: tiles[%zu] differs from the planned shape or dtype", i);
            return CLE_ERR_SHAPE;
        }
    }
    int cur = 0;
    CLE_CUDA(cudaGetDevice(&cur));
    if (cur != p->device) CLE_CUDA(cudaSetDevice(p->device));
    cudaStream_t main = reinterpret_cast<cudaStream_t>(stream);
    int rc = CLE_OK;
    do {
        if (cudaMemsetAsync(d_status, 0, sizeof(int32_t), main) != cudaSuccess) { rc = cuda_error(cudaGetLastError(), "status reset"); break; }
        if (cudaEventRecord(p->fork, main) != cudaSuccess) { rc = cuda_error(cudaGetLastError(), "fork"); break; }
        for (size_t k = 0; k < p->streams.size() && rc == CLE_OK; ++k) {
            cudaStream_t s = p->streams[k];
            if (cudaStreamWaitEvent(s, p->fork, 0) != cudaSuccess) { rc = cuda_error(cudaGetLastError(), "lane wait"); break; }
            char *ws = (char *)workspace + p->lane_off[k];
            const size_t cap = (k + 1 < p->lane_off.size() ? p->lane_off[k + 1] : p->ws_bytes) - p->lane_off[k];
            for (int i : p->lane_tiles[k]) {
                Arena ar(ws, cap);
                rc = voronoi_otsu_labeling(src[(size_t)i], dst[(size_t)i], p->spot, p->outline, ar, s, p->lim);
                if (rc != CLE_OK) break;
                status_max_kernel<<<1, 1, 0, s>>>(workspace_status_ptr(ws), d_status);
                count_launches(1);
                if (cudaGetLastError() != cudaSuccess) { rc = cuda_error(cudaGetLastError(), "status max"); break; }
            }
        }
        // join every lane that was forked, also after an error, so the
        // caller's stream (and a capture on it) stays consistent
        for (size_t k = 0; k < p->streams.size(); ++k) {
            cudaEventRecord(p->join[k], p->streams[k]);
            cudaStreamWaitEvent(main, p->join[k], 0);
        }
    } while (0);
    if (cur != p->device) cudaSetDevice(cur);
    return rc;
}

void cle_vol_batch_free(cle_vol_batch *plan) {
    if (plan) release(plan);
}

}  // extern "C"
