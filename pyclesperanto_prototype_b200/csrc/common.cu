// common.cu -- error state, tensor validation, workspace and launch helpers.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <atomic>
#include <mutex>

#include "common.cuh"

namespace cle {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

const char *last_error() { return g_err; }

static std::atomic<unsigned long long> g_launches{0};
void count_launches(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }
unsigned long long launches_issued() { return g_launches.load(std::memory_order_relaxed); }

static constexpr int kMaxStages = 16;
static thread_local cudaEvent_t g_ev[kMaxStages];
static thread_local bool g_prof = false;
static thread_local int g_marks = 0;
static thread_local unsigned g_recorded = 0;   // bit i: event i recorded since the last mark 0

static thread_local void *g_trace = nullptr;
static thread_local size_t g_trace_bytes = 0;
static constexpr size_t kTraceBytes = 1 << 16;

// Trace buffer of the current profiling session (allocated when tracing is
// enabled, never on a compute call); cleared on the caller's stream.
void *profile_trace_buffer(size_t bytes, cudaStream_t st) {
    if (!g_trace || bytes > g_trace_bytes) return nullptr;
    cudaMemsetAsync(g_trace, 0, bytes, st);
    return g_trace;
}

int profile_trace_read(void *host, size_t bytes) {
    if (!g_trace) return 0;
    if (bytes > g_trace_bytes) bytes = g_trace_bytes;
    cudaError_t e = cudaMemcpy(host, g_trace, bytes, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return -cuda_error(e, "trace copy");
    return (int)bytes;
}

// flags: bit 0 stage events, bit 1 per-step loop trace; 0 turns both off.
int profile_enable(int flags) {
    const bool on = flags != 0;
    if (on && !g_prof) {
        for (int i = 0; i < kMaxStages; ++i) {
            cudaError_t e = cudaEventCreate(&g_ev[i]);
            if (e != cudaSuccess) return cuda_error(e, "cudaEventCreate");
        }
        g_prof = true;
    }
    if ((flags & 2) && !g_trace) {
        cudaError_t e = cudaMalloc(&g_trace, kTraceBytes);
        if (e != cudaSuccess) return cuda_error(e, "trace buffer");
        g_trace_bytes = kTraceBytes;
    }
    if (!(flags & 2) && g_trace) {
        cudaFree(g_trace);
        g_trace = nullptr;
        g_trace_bytes = 0;
    }
    if (!on && g_prof) {
        for (int i = 0; i < kMaxStages; ++i) cudaEventDestroy(g_ev[i]);
        g_prof = false;
    }
    return CLE_OK;
}

void stage_mark(int i, cudaStream_t st) {
    if (!g_prof || i < 0 || i >= kMaxStages) return;
    cudaEventRecord(g_ev[i], st);
    if (i == 0) { g_marks = 1; g_recorded = 1u; }
    else {
        if (i + 1 > g_marks) g_marks = i + 1;
        g_recorded |= 1u << i;
    }
}

// Interval i-1 -> i in ms for every mark pair recorded (0 where either mark
// was not recorded, e.g. a call that runs only some of the stages).
int stage_ms(float *out, int max) {
    if (!g_prof || g_marks < 2) return 0;
    cudaError_t e = cudaEventSynchronize(g_ev[g_marks - 1]);
    if (e != cudaSuccess) return -cuda_error(e, "cudaEventSynchronize");
    int n = 0;
    for (int i = 1; i < g_marks && n < max; ++i, ++n) {
        float ms = 0.f;
        const unsigned pair = (1u << (i - 1)) | (1u << i);
        if ((g_recorded & pair) == pair && cudaEventElapsedTime(&ms, g_ev[i - 1], g_ev[i]) != cudaSuccess) {
            (void)cudaGetLastError();   // leave no error behind for the next launch check
            ms = 0.f;
        }
        out[n] = ms;
    }
    return n;
}

int cuda_error(cudaError_t e, const char *where) {
    set_error("CUDA error %d (%s) in %s", (int)e, cudaGetErrorString(e), where);
    return CLE_ERR_CUDA;
}

int dtype_size(int dtype) {
    switch (dtype) {
        case CLE_U8: return 1;
        case CLE_U16: return 2;
        case CLE_U32: return 4;
        case CLE_I32: return 4;
        case CLE_F32: return 4;
        default: return 0;
    }
}

int to_img(const cle_tensor *t, Img &out, const char *name) {
    if (!t) {
        set_error("%s: null tensor", name);
        return CLE_ERR_ARG;
    }
    if (dtype_size(t->dtype) == 0) {
        set_error("%s: unsupported dtype code %d", name, t->dtype);
        return CLE_ERR_DTYPE;
    }
    if (t->ndim < 1 || t->ndim > 3) {
        set_error("%s: expected a 1D, 2D or 3D image, got ndim=%d", name, t->ndim);
        return CLE_ERR_SHAPE;
    }
    int64_t expect = 1;
    for (int i = t->ndim - 1; i >= 0; --i) {
        if (t->shape[i] < 1) {
            set_error("%s: empty dimension %d (shape[%d]=%lld)", name, i, i, (long long)t->shape[i]);
            return CLE_ERR_SHAPE;
        }
        if (t->shape[i] > 1 && t->strides[i] != expect) {
            set_error("%s: not C-contiguous (dim %d stride %lld, expected %lld)", name, i,
                      (long long)t->strides[i], (long long)expect);
            return CLE_ERR_SHAPE;
        }
        expect *= t->shape[i];
    }
    out.data = t->data;
    out.dtype = t->dtype;
    out.ndim = t->ndim;
    if (t->ndim == 3) {
        out.D = t->shape[0]; out.H = t->shape[1]; out.W = t->shape[2];
    } else if (t->ndim == 2) {
        out.D = 1; out.H = t->shape[0]; out.W = t->shape[1];
    } else {
        out.D = 1; out.H = 1; out.W = t->shape[0];
        out.ndim = 2;
    }
    if (out.n() > (int64_t)0x7FFFFFFE) {
        set_error("%s: %lld voxels exceed the supported 2^31-2", name, (long long)out.n());
        return CLE_ERR_TOO_LARGE;
    }
    if (!t->data && out.n() > 0) {
        set_error("%s: null data pointer", name);
        return CLE_ERR_ARG;
    }
    return CLE_OK;
}

int same_shape(const Img &a, const Img &b, const char *an, const char *bn) {
    if (a.D != b.D || a.H != b.H || a.W != b.W) {
        set_error("shape mismatch: %s is (%lld,%lld,%lld) but %s is (%lld,%lld,%lld)", an,
                  (long long)a.D, (long long)a.H, (long long)a.W, bn, (long long)b.D,
                  (long long)b.H, (long long)b.W);
        return CLE_ERR_SHAPE;
    }
    return CLE_OK;
}

// _tier0/_sigma_to_kernel_size.py:1-4
int sigma_to_kernel_size(double sigma) {
    int n = (int)(sigma * 8.0);
    if (n % 2 == 0) n += 1;
    return n;
}

// Normalised sampled Gaussian; float32 sigma as the reference kernel receives
// it ("s": float(sigma), _tier1/_execute_separable_kernel.py:25-29).
int make_gauss_taps(double sigma, Taps &t) {
    int n = sigma_to_kernel_size(sigma);
    if (n > kMaxTaps) {
        set_error("gaussian_blur: sigma %g needs %d taps (max %d)", sigma, n, kMaxTaps);
        return CLE_ERR_ARG;
    }
    const int r = (n - 1) / 2;
    const double s = (double)(float)sigma;
    double sum = 0.0;
    for (int i = -r; i <= r; ++i) sum += std::exp(-(double)(i * i) / (2.0 * s * s));
    for (int i = -r; i <= r; ++i)
        t.w[i + r] = (float)(std::exp(-(double)(i * i) / (2.0 * s * s)) / sum);
    t.n = n;
    return CLE_OK;
}

Geo make_geo(const Img &im) {
    Geo g;
    g.D = (uint32_t)im.D;
    g.H = (uint32_t)im.H;
    g.W = (uint32_t)im.W;
    g.fW = FastDiv(g.W);
    g.fH = FastDiv(g.H);
    g.fD = FastDiv(g.D);
    g.fHD = FastDiv(g.H * g.D);
    return g;
}

uint32_t fkey_bits_for(int64_t n) {
    float f = (float)(n + 1);
    return fkey_index(f) + 2;
}

int num_sms(int device) {
    static int cache[64] = {0};
    if (device < 0 || device >= 64) device = 0;
    if (cache[device] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
            v <= 0)
            v = 148;
        cache[device] = v;
    }
    return cache[device];
}

int limits_from(const cle_call_options *o, Limits &out) {
    out = Limits();
    if (!o) return CLE_OK;
    if (o->struct_bytes != 0 && o->struct_bytes < sizeof(cle_call_options)) {
        set_error("call options: struct_bytes %u is smaller than this library's %zu", o->struct_bytes,
                  sizeof(cle_call_options));
        return CLE_ERR_ARG;
    }
    if (o->cooperative_ctas < 0 || o->reserved != 0) {
        set_error("call options: cooperative_ctas must be >= 0 and reserved 0 (got %d, %d)",
                  o->cooperative_ctas, o->reserved);
        return CLE_ERR_ARG;
    }
    out.max_steps = o->max_loop_steps;
    if (o->loop_time_limit_ms) out.loop_ns = (uint64_t)o->loop_time_limit_ms * 1000000ull;
    if (o->barrier_time_limit_ms) out.barrier_ns = (uint64_t)o->barrier_time_limit_ms * 1000000ull;
    out.coop_ctas = o->cooperative_ctas;
    if (o->cancel) {
        // the word must be page-locked host memory the device can read
        void *dptr = nullptr;
        cudaError_t e = cudaHostGetDevicePointer(&dptr, (void *)o->cancel, 0);
        if (e != cudaSuccess || !dptr) {
            (void)cudaGetLastError();
            set_error("call options: the cancel word is not page-locked host memory the device can map");
            return CLE_ERR_ARG;
        }
        out.cancel = (const volatile int *)dptr;
    }
    return CLE_OK;
}

int cooperative_ctas(int device, const Limits &lim) {
    const int sms = num_sms(device);
    return (lim.coop_ctas > 0 && lim.coop_ctas < sms) ? lim.coop_ctas : sms;
}

int launch_blocks(int64_t items, int threads, int max_blocks_per_sm) {
    int dev = 0;
    cudaGetDevice(&dev);
    int64_t need = (items + threads - 1) / threads;
    int64_t cap = (int64_t)num_sms(dev) * max_blocks_per_sm;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
}

}  // namespace cle
