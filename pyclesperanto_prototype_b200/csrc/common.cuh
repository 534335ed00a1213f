// common.cuh -- shared helpers of libcle_b200 (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <type_traits>

#include "../../include/cle_b200.h"

namespace cle {

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
void set_error(const char *fmt, ...);
const char *last_error();
void count_launches(int n);
unsigned long long launches_issued();
// Optional stage events (cle_profile_enable): the composite records one event
// per stage boundary on its stream; a no-op unless enabled on this thread.
void stage_mark(int i, cudaStream_t st);
int stage_ms(float *out, int max);
int profile_enable(int flags);
// Device buffer for per-step traces of device loops while profiling is
// enabled (null otherwise); cle_profile_trace() copies it out.
void *profile_trace_buffer(size_t bytes, cudaStream_t st);
int profile_trace_read(void *host, size_t bytes);
int cuda_error(cudaError_t e, const char *where);

#define CLE_CUDA(call)                                                        \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) return ::cle::cuda_error(e_, #call);           \
    } while (0)

// Checks the launch(es) just issued and counts them (kernel launches issued
// by this library, reported by cle_kernel_launches()).
#define CLE_LAUNCH_CHECK_N(name, nlaunch)                                     \
    do {                                                                      \
        ::cle::count_launches(nlaunch);                                       \
        cudaError_t e_ = cudaGetLastError();                                  \
        if (e_ != cudaSuccess) return ::cle::cuda_error(e_, name);            \
    } while (0)
#define CLE_LAUNCH_CHECK(name) CLE_LAUNCH_CHECK_N(name, 1)

#define CLE_TRY(expr)                                                         \
    do {                                                                      \
        int s_ = (expr);                                                      \
        if (s_ != CLE_OK) return s_;                                          \
    } while (0)

// ---------------------------------------------------------------------------
// Images
// ---------------------------------------------------------------------------
struct Img {
    void *data = nullptr;
    int ndim = 0;        // reference dimensionality (2 or 3)
    int dtype = 0;
    int64_t D = 1, H = 1, W = 1;
    int64_t n() const { return D * H * W; }
};

// Validates a 2D/3D C-contiguous tensor and fills an Img.
int to_img(const cle_tensor *t, Img &out, const char *name);
int same_shape(const Img &a, const Img &b, const char *an, const char *bn);
int dtype_size(int dtype);

// ---------------------------------------------------------------------------
// Workspace: a bump allocator over caller memory.  Every carve is 256-byte
// aligned.  size() on a null-based arena measures what a call needs.
// ---------------------------------------------------------------------------
struct Arena {
    char *base;
    size_t cap;
    size_t off = 0;
    bool measuring;
    Arena(void *b, size_t c) : base((char *)b), cap(c), measuring(b == nullptr) {}
    template <typename T>
    T *take(size_t count) {
        size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
        T *p = measuring ? nullptr : (T *)(base + off);
        off += bytes;
        return p;
    }
    bool ok() const { return measuring || off <= cap; }
};

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
static constexpr uint32_t kMarkBit = 0x80000000u;
// Mask byte of a voxel inside the segmentation, as the seed passes write it
// (0 outside).  The key growth keeps a voxel's arrival step in the low 7 bits
// once the voxel is labelled; all ones there stands for "not yet known".
static constexpr uint8_t kMaskByte = 0xFF;
static constexpr int kMaxTaps = 1025;

struct Taps {
    int n;            // 2r+1
    float w[kMaxTaps];
};

int make_gauss_taps(double sigma, Taps &t);
int sigma_to_kernel_size(double sigma);

template <typename T>
__device__ __forceinline__ float to_f32(T v) { return (float)v; }

__device__ __forceinline__ int64_t clamp64(int64_t v, int64_t lo, int64_t hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}
__device__ __forceinline__ int clampi(int v, int lo, int hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

// Order-preserving float <-> int mapping for atomicMin/atomicMax on floats.
__device__ __forceinline__ int f2ord(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float ord2f(int i) {
    return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF);
}

// L2-coherent loads/stores for data that other SMs update during a kernel.
__device__ __forceinline__ uint32_t ld_cg(const uint32_t *p) { return __ldcg(p); }
__device__ __forceinline__ void st_cg(uint32_t *p, uint32_t v) { __stcg(p, v); }

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Fast unsigned division by a runtime-constant divisor (round-up method):
// q = (umulhi(n, m) + n) >> s, exact for every 32-bit n.
struct FastDiv {
    uint32_t d, m, s;
    __host__ __device__ FastDiv() : d(1), m(1), s(0) {}
    __host__ FastDiv(uint32_t div) : d(div) {
        s = 0;
        while ((1ull << s) < div) ++s;
        m = (uint32_t)((((1ull << 32) * ((1ull << s) - div)) / div) + 1);
    }
    __device__ __forceinline__ uint32_t div(uint32_t n) const {
        return (uint32_t)(((uint64_t)__umulhi(n, m) + n) >> s);
    }
};

// Voxel index helpers: memory index m = (z*H + y)*W + x; reference label key
// K = (x*H + y)*D + z (x most significant, tests/test_set_nonzero_pixels_to_pixelindex.py).
struct Geo {
    uint32_t D, H, W;
    FastDiv fW, fH, fD, fHD;
};
Geo make_geo(const Img &im);

__device__ __forceinline__ void m2xyz(const Geo &g, uint32_t m, uint32_t &x, uint32_t &y,
                                      uint32_t &z) {
    uint32_t zy = g.fW.div(m);
    x = m - zy * g.W;
    z = g.fH.div(zy);
    y = zy - z * g.H;
}
__device__ __forceinline__ uint32_t xyz2m(const Geo &g, uint32_t x, uint32_t y, uint32_t z) {
    return (z * g.H + y) * g.W + x;
}
__device__ __forceinline__ uint32_t xyz2k(const Geo &g, uint32_t x, uint32_t y, uint32_t z) {
    return (x * g.H + y) * g.D + z;
}
__device__ __forceinline__ uint32_t k2m(const Geo &g, uint32_t k) {
    uint32_t x = g.fHD.div(k);
    uint32_t r = k - x * g.H * g.D;
    uint32_t y = g.fD.div(r);
    uint32_t z = r - y * g.D;
    return xyz2m(g, x, y, z);
}

// Dense index of an integer-valued float32 key f >= 1: f itself below 2^24,
// above it the count of integer floats (every float >= 2^23 is an integer,
// so consecutive bit patterns are consecutive integers).  Monotonic.
__host__ __device__ __forceinline__ uint32_t fkey_index(float f) {
    if (f < 16777216.0f) return (uint32_t)f;
#ifdef __CUDA_ARCH__
    uint32_t b = __float_as_uint(f);
#else
    uint32_t b;
    memcpy(&b, &f, 4);
#endif
    return (b - (151u << 23)) + 16777216u;
}
uint32_t fkey_bits_for(int64_t n);  // bitmap size covering keys 1..n

// ---------------------------------------------------------------------------
// Grid-wide barrier for cooperative launches with a wall-clock limit: a
// block that waits longer than limit_ns records CLE_ERR_ITER_LIMIT in *err
// and returns; callers check the returned flag and leave their loops.
// ---------------------------------------------------------------------------
struct GridBarrier {
    unsigned int count;
    unsigned int gen;
};

__device__ __forceinline__ bool grid_sync(GridBarrier *b, int *err, uint64_t limit_ns) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int *vgen = &b->gen;
        unsigned int g = *vgen;
        __threadfence();
        unsigned int arrived = atomicAdd(&b->count, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(&b->count, 0u);
            __threadfence();
            atomicAdd(&b->gen, 1u);
        } else {
            uint64_t t0 = global_ns();
            uint32_t spins = 0;
            while (*vgen == g) {
                if ((++spins & 1023u) == 0u && global_ns() - t0 > limit_ns) {
                    atomicExch(err, (int)CLE_ERR_ITER_LIMIT);
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int *)err == 0;
}

// Per-call limits of the device loops (cle_call_options); a value, passed
// down each call, never stored between calls.
struct Limits {
    uint32_t max_steps = 0;                     // 0: voxels + 16
    uint64_t loop_ns = 20000000000ull;          // wall-clock bound of one loop launch
    uint64_t barrier_ns = 4000000000ull;        // bound of one grid-barrier wait
    int coop_ctas = 0;                          // 0: one CTA per SM
    const volatile int *cancel = nullptr;       // device view of the caller's cancel word
    // step bound of a loop over n voxels
    uint32_t steps_for(int64_t n) const {
        const uint64_t dflt = (uint64_t)n + 16u;
        const uint64_t s = max_steps ? std::min<uint64_t>(max_steps, dflt) : dflt;
        return (uint32_t)std::min<uint64_t>(s, 0xFFFFFFF0ull);
    }
};
// Validates options (NULL = defaults) into a Limits.
int limits_from(const cle_call_options *o, Limits &out);

// Launch helpers
int num_sms(int device);
// CTAs one cooperative launch may use on `device` under lim (one per SM
// unless lim caps it).
int cooperative_ctas(int device, const Limits &lim);
int launch_blocks(int64_t items, int threads, int max_blocks_per_sm = 8);

}  // namespace cle
