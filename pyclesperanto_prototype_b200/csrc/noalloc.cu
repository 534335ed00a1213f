// noalloc.cu -- threshold_otsu for callers that cannot allocate device memory.
//
// cle_threshold_otsu takes its scratch (per-row histogram partials, min/max
// partials, the histogram and the threshold) from a workspace the caller
// allocates.  Some callers can hand over the input and output buffers but
// cannot allocate anything themselves: a host application that owns a fixed
// device-memory budget and forbids allocation inside its processing loop, or
// a plugin that only passes through the buffers its host gives it.  For them
// cle_threshold_otsu_noalloc uses a scratch array compiled into the library
// instead: a file-scope __device__ array of kScratchBytes, which every GPU
// that loads the library holds until the process exits.
//
// Host code never uses the array's name as a pointer (on the host it only
// stands for the symbol): every call, with the call's device current,
// resolves the array's device address with cudaGetSymbolAddress.  The first
// call on a device also loads the library's code onto it (set-up), so that
// first call should come before any stream capture; later look-ups are cheap.
// Nothing is cached, so a device reset (which reloads the code at a new
// address) leaves no stale pointer behind.  All calls share the one array and each call rewrites every part
// of it it reads (the row partials are cleared on the stream first), so a
// call sees nothing of the previous one; calls that overlap on the GPU (other
// streams, other host threads) race on it and must be serialised by the
// caller.  No allocation happens here: no cudaMalloc, no cudaFree, no
// allocating library routine.
#include "common.cuh"
#include "kernels.cuh"

namespace cle {

namespace {

// 4 MiB of row partials (4096 rows x 256 bins x 4 B) plus 64 KiB for the
// min/max partials, the histogram and the threshold.
constexpr size_t kScratchBytes = (size_t(4) << 20) + (size_t(64) << 10);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of the scratch array on the current device, looked up on
// each call (the first look-up on a device is its set-up).
int scratch_address(void **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(noalloc scratch)");
    if (!p || (reinterpret_cast<uintptr_t>(p) & 255)) {
        set_error("threshold_otsu_noalloc: scratch array address is not 256-byte aligned");
        return CLE_ERR_CUDA;
    }
    *out = p;
    return CLE_OK;
}

}  // namespace

size_t threshold_otsu_noalloc_capacity() { return kScratchBytes; }

int threshold_otsu_noalloc(const Img &a, const Img &b, cudaStream_t st) {
    CLE_TRY(same_shape(a, b, "source", "destination"));
    // same carve-up as cle_threshold_otsu: {min,max,thr32}, histogram, threshold, then the
    // min/max partials and the row partials
    Arena probe(nullptr, 0);
    probe.take<float>(64);
    probe.take<float>(256);
    probe.take<double>(4);
    const size_t need = probe.off + minmax_workspace_bytes(a) + histogram_workspace_bytes(a, 256);
    if (need > kScratchBytes) {
        set_error("threshold_otsu_noalloc: this image needs %zu bytes of scratch but the built-in "
                  "array holds %zu (images with up to 4096 rows fit); use cle_threshold_otsu with a "
                  "workspace", need, kScratchBytes);
        return CLE_ERR_TOO_LARGE;
    }
    void *scratch = nullptr;
    CLE_TRY(scratch_address(&scratch));
    Arena ar(scratch, kScratchBytes);
    float *mm = ar.take<float>(64);
    float *hist = ar.take<float>(256);
    double *thr = ar.take<double>(4);
    CLE_TRY(minmax(a, mm, ar, st));
    CLE_TRY(histogram(a, 256, mm, hist, ar, st));   // clears its row partials first
    CLE_TRY(otsu(hist, mm, thr, mm + 2, st));
    return greater_constant(a, b, 0.0f, mm + 2, st);
}

}  // namespace cle
