/*
 * cle_oracle.c -- CPU restatement of pyclesperanto_prototype's
 * voronoi_otsu_labeling + statistics_of_labelled_pixels path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * library and the timed CPU baseline.  Only tests/, __graft_entry__.smoke()
 * and bench.py (cpu_baseline leg and --impl reference) may load it.  The
 * product path never calls into it.
 *
 * Arrays are C-order (z, y, x) with extents D, H, W (D = 1 for 2D images);
 * "ndim" is the reference array's dimensionality (2 or 3) because several
 * kernels behave differently for 2D and 3D inputs.
 *
 * Parity pins: see the citations on each function.  Where the reference
 * kernel source is absent (un-vendored clij-opencl-kernels submodule) the
 * semantics are reconstructed from the reference's call sites and tests; the
 * floating-point operation order chosen here is the one the CUDA kernels use.
 *
 * Build: oracle/Makefile  (gcc -O2 -ffp-contract=off -fopenmp, no -ffast-math:
 * every multiply-add below is either an explicit fmaf() or a separately
 * rounded multiply and add).
 */
#include <math.h>
#include <float.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define IDX(z, y, x) ((((int64_t)(z)) * H + (y)) * W + (x))

static inline int64_t clampi(int64_t v, int64_t lo, int64_t hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------ */
/* A2: kernel size.  _tier0/_sigma_to_kernel_size.py:1-4               */
/* n = int(8*sigma); n += 1 if n is even.                              */
/* ------------------------------------------------------------------ */
int orc_sigma_to_kernel_size(double sigma) {
    int n = (int)(sigma * 8.0);
    if (n % 2 == 0) n += 1;
    return n;
}

/* Normalised sampled Gaussian: h_i = exp(-i^2 / (2 s^2)) in double with s
 * the float32 sigma the reference hands to its kernel
 * (_tier1/_execute_separable_kernel.py:25-29 passes "s": float(sigma)),
 * w_i = float32(h_i / sum_j h_j), sum accumulated from -r to r. */
void orc_gauss_weights(double sigma, int n, float *w) {
    const int r = (n - 1) / 2;
    const double s = (double)(float)sigma;
    double sum = 0.0;
    for (int i = -r; i <= r; ++i) sum += exp(-(double)(i * i) / (2.0 * s * s));
    for (int i = -r; i <= r; ++i)
        w[i + r] = (float)(exp(-(double)(i * i) / (2.0 * s * s)) / sum);
}

/* One separable pass along `axis` (0 = z, 1 = y, 2 = x), clamp-to-edge reads
 * (_tier0/preamble.cl:33-195), accumulation acc = fmaf(w_i, v_i, acc) for
 * i = -r..r ascending starting from acc = 0. */
static void blur_pass(const float *in, float *out, int64_t D, int64_t H, int64_t W,
                      int axis, const float *w, int r) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t z = 0; z < D; ++z)
        for (int64_t y = 0; y < H; ++y)
            for (int64_t x = 0; x < W; ++x) {
                float acc = 0.0f;
                for (int i = -r; i <= r; ++i) {
                    int64_t zz = z, yy = y, xx = x;
                    if (axis == 0) zz = clampi(z + i, 0, D - 1);
                    else if (axis == 1) yy = clampi(y + i, 0, H - 1);
                    else xx = clampi(x + i, 0, W - 1);
                    acc = fmaf(w[i + r], in[IDX(zz, yy, xx)], acc);
                }
                out[IDX(z, y, x)] = acc;
            }
}

/* A3 gaussian_blur: _tier1/_gaussian_blur.py:39-56 and
 * _tier1/_execute_separable_kernel.py:7-76.  Passes x, then y, then z (3D
 * only); a pass with sigma <= 0 is a copy.  In 2D sigma_z is ignored. */
void orc_gaussian_blur(const float *src, float *dst, int64_t D, int64_t H, int64_t W,
                       int ndim, double sx, double sy, double sz) {
    const int64_t n = D * H * W;
    float *t1 = (float *)malloc(sizeof(float) * n);
    float *t2 = (float *)malloc(sizeof(float) * n);
    double sig[3] = {sx, sy, sz};
    const float *cur = src;
    float *bufs[2] = {t1, t2};
    int which = 0;
    int passes = (ndim == 3) ? 3 : 2;
    for (int p = 0; p < passes; ++p) {
        float *o = (p == passes - 1) ? dst : bufs[which];
        if (sig[p] > 0) {
            int ks = orc_sigma_to_kernel_size(sig[p]);
            float *w = (float *)malloc(sizeof(float) * ks);
            orc_gauss_weights(sig[p], ks, w);
            blur_pass(cur, o, D, H, W, 2 - p, w, (ks - 1) / 2);
            free(w);
        } else {
            memcpy(o, cur, sizeof(float) * n);
        }
        cur = o;
        which ^= 1;
    }
    free(t1);
    free(t2);
}

/* ------------------------------------------------------------------ */
/* A4 detect_maxima (radius 1):  _tier1/detect_maxima_3d_x.cl:8-48,    */
/* _tier1/detect_maxima_2d_x.cl:8-34.  Literal emulation of the loop:  */
/* localMax starts at v(p) - 1 (float32), positions with a negative    */
/* coordinate are skipped, reads clamp to the edge, strict '>' update, */
/* loop order x (outer), y, z (inner).  out = 1 iff the arg-max        */
/* position is p itself.                                               */
/* ------------------------------------------------------------------ */
void orc_detect_maxima(const float *src, uint8_t *dst, int64_t D, int64_t H, int64_t W,
                       int ndim) {
    const int zr = (ndim == 3) ? 1 : 0;
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t z = 0; z < D; ++z)
        for (int64_t y = 0; y < H; ++y)
            for (int64_t x = 0; x < W; ++x) {
                float lm = src[IDX(z, y, x)] - 1.0f;
                int64_t px = x, py = y, pz = z;
                for (int dx = -1; dx <= 1; ++dx)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dz = -zr; dz <= zr; ++dz) {
                            int64_t lx = x + dx, ly = y + dy, lz = z + dz;
                            if (lx >= 0 && ly >= 0 && lz >= 0) {
                                float v = src[IDX(clampi(lz, 0, D - 1), clampi(ly, 0, H - 1),
                                                  clampi(lx, 0, W - 1))];
                                if (v > lm) {
                                    lm = v;
                                    px = lx; py = ly; pz = lz;
                                }
                            }
                        }
                dst[IDX(z, y, x)] = (px == x && py == y && pz == z) ? 1 : 0;
            }
}

/* A5: exact float32 min / max over all voxels
 * (_tier2/_minimum_of_all_pixels.py:7-60, _tier2/_maximum_of_all_pixels.py). */
void orc_minmax(const float *src, int64_t n, float *mn, float *mx) {
    float a = INFINITY, b = -INFINITY;
    for (int64_t i = 0; i < n; ++i) {
        float v = src[i];
        if (v < a) a = v;
        if (v > b) b = v;
    }
    *mn = a;
    *mx = b;
}

/* OpenCL convert_uint_sat(float): NaN -> 0, saturate, truncate toward 0. */
static inline uint32_t cvt_uint_sat(float t) {
    if (!(t > 0.0f)) return 0u;          /* NaN, zero and negatives */
    if (t >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)t;
}

/* Histogram bin of v (rule C, numpy restatement of the missing
 * histogram_3d_x.cl): t = ((v - min) * (bins - 1)) / range in float32,
 * then convert_uint_sat(t + 0.5f).  Returns -1 for an out-of-range bin
 * (only possible with a caller-supplied min/max narrower than the data). */
static inline int64_t hist_bin(float v, float mn, float range, int bins) {
    float t = ((v - mn) * (float)(bins - 1)) / range;
    uint32_t b = cvt_uint_sat(t + 0.5f);
    return (b < (uint32_t)bins) ? (int64_t)b : -1;
}

/* A6 histogram: _tier3/_histogram.py:85-128.  One partial histogram per
 * y row (exact integer counts over all z and x of that row, stored as
 * float32), then sum_z_projection: a float32 running sum over rows
 * y = 0 .. H-1 in order. */
void orc_histogram(const float *src, int64_t D, int64_t H, int64_t W, int bins, float mn,
                   float mx, float *hist) {
    const float range = mx - mn;
    uint32_t *part = (uint32_t *)calloc((size_t)H * bins, sizeof(uint32_t));
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < H; ++y) {
        uint32_t *row = part + y * bins;
        for (int64_t z = 0; z < D; ++z)
            for (int64_t x = 0; x < W; ++x) {
                int64_t b = hist_bin(src[IDX(z, y, x)], mn, range, bins);
                if (b >= 0) row[b]++;
            }
    }
    for (int b = 0; b < bins; ++b) {
        float acc = 0.0f;
        for (int64_t y = 0; y < H; ++y) acc = acc + (float)part[y * bins + b];
        hist[b] = acc;
    }
    free(part);
}

/* A7 Otsu: _tier9/_threshold_otsu.py:38-49 (bin centres) and :64-106
 * (scikit-image's threshold_otsu on a given histogram), float64, numpy's
 * sequential cumsum, x**2 == x*x, first-occurrence argmax where NaN counts
 * as the maximum (numpy.argmax).  Returns the float64 threshold. */
double orc_otsu_threshold(const float *hist, int bins, float mn, float mx) {
    const float range32 = mx - mn;
    double *bc = (double *)malloc(sizeof(double) * bins);
    double *w1 = (double *)malloc(sizeof(double) * bins);
    double *w2 = (double *)malloc(sizeof(double) * bins);
    double *m1 = (double *)malloc(sizeof(double) * bins);
    double *m2 = (double *)malloc(sizeof(double) * bins);
    for (int i = 0; i < bins; ++i) bc[i] = ((double)i * (double)range32) / 255.0 + (double)mn;
    double acc = 0.0, accm = 0.0;
    for (int i = 0; i < bins; ++i) {
        double c = (double)hist[i];
        acc = acc + c;
        accm = accm + c * bc[i];
        w1[i] = acc;
        m1[i] = accm / acc;
    }
    acc = 0.0;
    accm = 0.0;
    for (int i = bins - 1; i >= 0; --i) {
        double c = (double)hist[i];
        acc = acc + c;
        accm = accm + c * bc[i];
        w2[i] = acc;
        m2[i] = accm / acc;
    }
    int idx = 0;
    double best = 0.0;
    for (int i = 0; i < bins - 1; ++i) {
        double d = m1[i] - m2[i + 1];
        double v = (w1[i] * w2[i + 1]) * (d * d);
        if (isnan(v)) { idx = i; break; }
        if (i == 0 || v > best) { best = v; idx = i; }
    }
    double t = bc[idx];
    free(bc); free(w1); free(w2); free(m1); free(m2);
    return t;
}

/* A8: greater_constant(source, dest, float(threshold)):
 * _tier1/_greater_constant.py (scalar passed as float32). */
void orc_greater_constant(const float *src, uint8_t *dst, int64_t n, float c) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) dst[i] = src[i] > c ? 1 : 0;
}

/* A9: binary_and -- (a != 0 && b != 0). */
void orc_binary_and(const uint8_t *a, const uint8_t *b, uint8_t *dst, int64_t n) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) dst[i] = (a[i] != 0 && b[i] != 0) ? 1 : 0;
}

/* threshold_otsu (A5-A8) end to end on a float32 image. */
double orc_threshold_otsu(const float *src, uint8_t *dst, int64_t D, int64_t H, int64_t W) {
    float mn, mx, hist[256];
    orc_minmax(src, D * H * W, &mn, &mx);
    orc_histogram(src, D, H, W, 256, mn, mx, hist);
    double t = orc_otsu_threshold(hist, 256, mn, mx);
    orc_greater_constant(src, dst, D * H * W, (float)t);
    return t;
}

/* ------------------------------------------------------------------ */
/* A10 connected_components_labeling_box + relabel_sequential.         */
/* _tier4/_connected_components_labeling_box.py:39-64,                 */
/* _tier1/_set_non_zero_pixels_to_pixel_index.py (offset 1),           */
/* tests/test_set_nonzero_pixels_to_pixelindex.py pins 2D key x*H+y+1; */
/* 3D key assumed x*H*D + y*D + z + 1 (x most significant).  Keys live */
/* in float32, so every component's value is float32(min key); the     */
/* relabel (_tier3/_relabel_sequential.py:42-57) ranks distinct values */
/* and components whose float32 keys collide share one label.          */
/* ------------------------------------------------------------------ */
static int64_t uf_find(int64_t *par, int64_t a) {
    while (par[a] != a) {
        par[a] = par[par[a]];
        a = par[a];
    }
    return a;
}

static int cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return (x > y) - (x < y);
}

/* fg: nonzero = foreground.  labels: output uint32.  Returns the number of
 * labels. */
static int64_t ccl_conn(const uint8_t *fg, uint32_t *labels, int64_t D, int64_t H, int64_t W,
                        int diamond);

int64_t orc_ccl_box(const uint8_t *fg, uint32_t *labels, int64_t D, int64_t H, int64_t W) {
    return ccl_conn(fg, labels, D, H, W, 0);
}

/* connected_components_labeling_diamond: _tier5/_connected_components_labeling_diamond.py:
 * 39 -- the box labelling with nonzero_minimum_diamond as the propagation
 * filter, i.e. face connectivity; keys and relabel as for the box form. */
int64_t orc_ccl_diamond(const uint8_t *fg, uint32_t *labels, int64_t D, int64_t H, int64_t W) {
    return ccl_conn(fg, labels, D, H, W, 1);
}

static int64_t ccl_conn(const uint8_t *fg, uint32_t *labels, int64_t D, int64_t H, int64_t W,
                        int diamond) {
    const int64_t n = D * H * W;
    int64_t *par = (int64_t *)malloc(sizeof(int64_t) * n);
    for (int64_t i = 0; i < n; ++i) par[i] = fg[i] ? i : -1;
    /* union with the 13 neighbours that precede in memory order */
    for (int64_t z = 0; z < D; ++z)
        for (int64_t y = 0; y < H; ++y)
            for (int64_t x = 0; x < W; ++x) {
                int64_t p = IDX(z, y, x);
                if (!fg[p]) continue;
                for (int dz = -1; dz <= 0; ++dz)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx) {
                            if (dz == 0 && (dy > 0 || (dy == 0 && dx >= 0))) continue;
                            if (diamond && (abs(dx) + abs(dy) + abs(dz)) > 1) continue;
                            int64_t qz = z + dz, qy = y + dy, qx = x + dx;
                            if (qz < 0 || qy < 0 || qy >= H || qx < 0 || qx >= W) continue;
                            int64_t q = IDX(qz, qy, qx);
                            if (!fg[q]) continue;
                            int64_t a = uf_find(par, p), b = uf_find(par, q);
                            if (a != b) {
                                if (a < b) par[b] = a; else par[a] = b;
                            }
                        }
            }
    /* per root: minimum x-major key K = (x*H + y)*D + z */
    uint32_t *rootkey = (uint32_t *)malloc(sizeof(uint32_t) * n);
    for (int64_t i = 0; i < n; ++i) rootkey[i] = 0xFFFFFFFFu;
    for (int64_t z = 0; z < D; ++z)
        for (int64_t y = 0; y < H; ++y)
            for (int64_t x = 0; x < W; ++x) {
                int64_t p = IDX(z, y, x);
                if (!fg[p]) continue;
                int64_t r = uf_find(par, p);
                uint32_t k = (uint32_t)((x * H + y) * D + z);
                if (k < rootkey[r]) rootkey[r] = k;
            }
    /* float32 key of each component, as its bit pattern (positive floats
     * order like their bit patterns) */
    int64_t nroots = 0;
    for (int64_t i = 0; i < n; ++i)
        if (fg[i] && par[i] == i) nroots++;
    uint32_t *keys = (uint32_t *)malloc(sizeof(uint32_t) * (nroots ? nroots : 1));
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i)
        if (fg[i] && par[i] == i) {
            float f = (float)((int64_t)rootkey[i] + 1);
            memcpy(&keys[k++], &f, 4);
        }
    qsort(keys, nroots, sizeof(uint32_t), cmp_u32);
    int64_t nuniq = 0;
    for (int64_t i = 0; i < nroots; ++i)
        if (i == 0 || keys[i] != keys[i - 1]) keys[nuniq++] = keys[i];
    for (int64_t i = 0; i < n; ++i) {
        if (!fg[i]) { labels[i] = 0; continue; }
        int64_t r = uf_find(par, i);
        float f = (float)((int64_t)rootkey[r] + 1);
        uint32_t kb;
        memcpy(&kb, &f, 4);
        int64_t lo = 0, hi = nuniq - 1;
        while (lo < hi) {
            int64_t mid = (lo + hi) / 2;
            if (keys[mid] < kb) lo = mid + 1; else hi = mid;
        }
        labels[i] = (uint32_t)(lo + 1);
    }
    free(par); free(rootkey); free(keys);
    return nuniq;
}

/* relabel_sequential (_tier3/_relabel_sequential.py:12-58): dense ranks of
 * the distinct nonzero values, order preserving, background stays 0.
 * Values are taken as (int) of the float (flag_existing_intensities /
 * replace_intensities index by the truncated value). */
void orc_relabel_sequential(const uint32_t *src, uint32_t *dst, int64_t n) {
    uint32_t mx = 0;
    for (int64_t i = 0; i < n; ++i) if (src[i] > mx) mx = src[i];
    uint32_t *map = (uint32_t *)calloc((size_t)mx + 1, sizeof(uint32_t));
    for (int64_t i = 0; i < n; ++i) map[src[i]] = 1;
    map[0] = 0;
    uint32_t c = 0;
    for (uint64_t v = 0; v <= mx; ++v) if (map[v]) map[v] = ++c;
    for (int64_t i = 0; i < n; ++i) dst[i] = map[src[i]];
    free(map);
}

/* ------------------------------------------------------------------ */
/* A11 masked_voronoi_labeling: _tier5/_masked_voronoi_labeling.py:44-76*/
/* flup = mask - 1; flop = CCL(seeds); flip = flup + flop (float32);   */
/* Jacobi steps of onlyzero_overwrite_maximum, box (26/8 neighbours)   */
/* on even steps and diamond (6/4) on odd steps, until a step changes  */
/* nothing; then mask(result, mask).  A voxel is overwritten only while*/
/* it is 0, with the maximum over the stencil including itself.        */
/* Returns the number of steps run (including the final no-change one).*/
/* out_f32 may be NULL; out_u32 (clij_convert_uint_sat of the masked   */
/* result, preamble.cl:548-556) may be NULL.                           */
/* ------------------------------------------------------------------ */
static inline uint32_t cvt_uint_sat_clij(float v) {
    if (v > 4294967295.0f) return 0xFFFFFFFFu;
    if (v < 0.0f) return 0u;
    if (v != v) return 0u;
    return (uint32_t)v;
}

int64_t orc_masked_voronoi(const uint8_t *seeds, const float *mask, float *out_f32,
                           uint32_t *out_u32, int64_t D, int64_t H, int64_t W, int ndim) {
    const int64_t n = D * H * W;
    uint32_t *cc = (uint32_t *)malloc(sizeof(uint32_t) * n);
    orc_ccl_box(seeds, cc, D, H, W);
    float *a = (float *)malloc(sizeof(float) * n);
    float *b = (float *)malloc(sizeof(float) * n);
    for (int64_t i = 0; i < n; ++i) a[i] = (mask[i] - 1.0f) + (float)cc[i];
    free(cc);
    const int zr = (ndim == 3) ? 1 : 0;
    int64_t step = 0;
    for (;;) {
        const int box = (step % 2) == 0;
        int64_t changed = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : changed)
        for (int64_t z = 0; z < D; ++z)
            for (int64_t y = 0; y < H; ++y)
                for (int64_t x = 0; x < W; ++x) {
                    const int64_t p = IDX(z, y, x);
                    float v = a[p];
                    if (v != 0.0f) { b[p] = v; continue; }
                    float m = v;
                    for (int dz = -zr; dz <= zr; ++dz)
                        for (int dy = -1; dy <= 1; ++dy)
                            for (int dx = -1; dx <= 1; ++dx) {
                                if (!box && (abs(dx) + abs(dy) + abs(dz)) > 1) continue;
                                int64_t qz = z + dz, qy = y + dy, qx = x + dx;
                                if (qz < 0 || qz >= D || qy < 0 || qy >= H || qx < 0 || qx >= W)
                                    continue;
                                float q = a[IDX(qz, qy, qx)];
                                if (q > m) m = q;
                            }
                    b[p] = m;
                    if (m != v) changed++;
                }
        float *t = a; a = b; b = t;
        step++;
        if (changed == 0) break;
    }
    for (int64_t i = 0; i < n; ++i) {
        float r = (mask[i] != 0.0f) ? a[i] : 0.0f;
        if (out_f32) out_f32[i] = r;
        if (out_u32) out_u32[i] = cvt_uint_sat_clij(r);
    }
    free(a); free(b);
    return step;
}

/* ------------------------------------------------------------------ */
/* erode_box: _tier1/_erode_box.py:6-47 (erode_box_{2,3}d_x.cl, absent  */
/* from the checkout).  out = 1 iff v(p) != 0 and v(q) != 0 for every q */
/* of the 3x3(x3) box around p.  Reads clamp to the edge, and a clamped */
/* read lands on a voxel of the same box, so out-of-range neighbours    */
/* are skipped.  Pinned by tests/test_erode_box.py (2D 5x5).           */
/* ------------------------------------------------------------------ */
static void erode_u8(const uint8_t *src, uint8_t *dst, int64_t D, int64_t H, int64_t W,
                     int ndim) {
    const int zr = (ndim == 3) ? 1 : 0;
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t z = 0; z < D; ++z)
        for (int64_t y = 0; y < H; ++y)
            for (int64_t x = 0; x < W; ++x) {
                uint8_t o = src[IDX(z, y, x)] != 0;
                for (int dz = -zr; dz <= zr && o; ++dz)
                    for (int dy = -1; dy <= 1 && o; ++dy)
                        for (int dx = -1; dx <= 1 && o; ++dx) {
                            const int64_t qz = z + dz, qy = y + dy, qx = x + dx;
                            if (qz < 0 || qz >= D || qy < 0 || qy >= H || qx < 0 || qx >= W)
                                continue;
                            if (src[IDX(qz, qy, qx)] == 0) o = 0;
                        }
                dst[IDX(z, y, x)] = o;
            }
}

void orc_erode_box(const float *src, uint8_t *dst, int64_t D, int64_t H, int64_t W, int ndim) {
    const int64_t n = D * H * W;
    uint8_t *nz = (uint8_t *)malloc(n);
    for (int64_t i = 0; i < n; ++i) nz[i] = src[i] != 0.0f;
    erode_u8(nz, dst, D, H, W, ndim);
    free(nz);
}

/* minimum_box / maximum_box: _tier1/_minimum_box.py:6-55 with             */
/* _tier1/_execute_separable_kernel.py:7-76 -- passes x, y, z (3D); each     */
/* the min (max) over i = -c..c, c = (N-1)/2, N = int(2*radius + 1), reads   */
/* clamped to the edge; radius <= 0 copies.  top_hat_box: _tier2/            */
/* _top_hat_box.py:37-43, source - maximum_box(minimum_box(source)).          */
static void minmax_line_pass(const float *src, float *dst, int64_t D, int64_t H, int64_t W,
                             int axis, int c, int is_max) {
    const int64_t n = D * H * W;
    if (c <= 0) { memcpy(dst, src, sizeof(float) * n); return; }
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t z = 0; z < D; ++z)
        for (int64_t y = 0; y < H; ++y)
            for (int64_t x = 0; x < W; ++x) {
                float m = src[IDX(z, y, x)];
                for (int i = -c; i <= c; ++i) {
                    int64_t qz = z, qy = y, qx = x;
                    if (axis == 0) qx = clampi(x + i, 0, W - 1);
                    else if (axis == 1) qy = clampi(y + i, 0, H - 1);
                    else qz = clampi(z + i, 0, D - 1);
                    const float v = src[IDX(qz, qy, qx)];
                    m = is_max ? (v > m ? v : m) : (v < m ? v : m);
                }
                dst[IDX(z, y, x)] = m;
            }
}

static int box_radius(double r) {
    if (!(r > 0)) return 0;
    const int64_t n = (int64_t)(r * 2 + 1);
    return (int)((n - 1) / 2);
}

void orc_minmax_box(const float *src, float *dst, int64_t D, int64_t H, int64_t W, int ndim,
                    double rx, double ry, double rz, int is_max) {
    const int64_t n = D * H * W;
    float *t = (float *)malloc(sizeof(float) * n);
    float *u = (float *)malloc(sizeof(float) * n);
    minmax_line_pass(src, t, D, H, W, 0, box_radius(rx), is_max);
    minmax_line_pass(t, ndim == 3 ? u : dst, D, H, W, 1, box_radius(ry), is_max);
    if (ndim == 3) minmax_line_pass(u, dst, D, H, W, 2, box_radius(rz), is_max);
    free(t); free(u);
}

void orc_top_hat_box(const float *src, float *dst, int64_t D, int64_t H, int64_t W, int ndim,
                     double rx, double ry, double rz) {
    const int64_t n = D * H * W;
    float *mn = (float *)malloc(sizeof(float) * n);
    float *op = (float *)malloc(sizeof(float) * n);
    orc_minmax_box(src, mn, D, H, W, ndim, rx, ry, rz, 0);
    orc_minmax_box(mn, op, D, H, W, ndim, rx, ry, rz, 1);
    for (int64_t i = 0; i < n; ++i) dst[i] = src[i] - op[i];
    free(mn); free(op);
}

/* gauss_otsu_labeling: _tier9/_gauss_otsu_labeling.py:36-45 -- blur with */
/* outline_sigma on every axis, threshold_otsu, connected components    */
/* (box).  Returns the number of labels.                                */
int64_t orc_gauss_otsu_labeling(const float *src, uint32_t *labels, int64_t D, int64_t H,
                                int64_t W, int ndim, double outline_sigma) {
    const int64_t n = D * H * W;
    float *tmp = (float *)malloc(sizeof(float) * n);
    uint8_t *seg = (uint8_t *)malloc(n);
    orc_gaussian_blur(src, tmp, D, H, W, ndim, outline_sigma, outline_sigma, outline_sigma);
    orc_threshold_otsu(tmp, seg, D, H, W);
    const int64_t nl = orc_ccl_box(seg, labels, D, H, W);
    free(tmp);
    free(seg);
    return nl;
}

/* eroded_otsu_labeling: _tier9/_eroded_otsu_labeling.py:46-62 -- blur, */
/* threshold_otsu, number_of_erosions box erosions of the binary image  */
/* (int() of the argument, none when it is <= 0), then                  */
/* masked_voronoi_labeling(eroded, binary).  Returns the Voronoi steps.  */
int64_t orc_eroded_otsu_labeling(const float *src, uint32_t *labels, int64_t D, int64_t H,
                                 int64_t W, int ndim, int number_of_erosions,
                                 double outline_sigma) {
    const int64_t n = D * H * W;
    float *tmp = (float *)malloc(sizeof(float) * n);
    uint8_t *binary = (uint8_t *)malloc(n);
    uint8_t *e0 = (uint8_t *)malloc(n);
    uint8_t *e1 = (uint8_t *)malloc(n);
    orc_gaussian_blur(src, tmp, D, H, W, ndim, outline_sigma, outline_sigma, outline_sigma);
    orc_threshold_otsu(tmp, binary, D, H, W);
    memcpy(e0, binary, n);
    for (int i = 0; i < number_of_erosions; ++i) {
        erode_u8(e0, e1, D, H, W, ndim);
        uint8_t *t = e0; e0 = e1; e1 = t;
    }
    for (int64_t i = 0; i < n; ++i) tmp[i] = (float)binary[i];
    const int64_t steps = orc_masked_voronoi(e0, tmp, NULL, labels, D, H, W, ndim);
    free(tmp); free(binary); free(e0); free(e1);
    return steps;
}

/* ------------------------------------------------------------------ */
/* extend_labeling_via_voronoi: _tier4/_extend_labeling_via_voronoi.py:*/
/* 30-56.  uint32 state (flip/flop are uint32 label images): every 0   */
/* voxel takes the maximum over the box (even steps) or the face       */
/* neighbours (odd steps) including itself; stop after the first step  */
/* that changes nothing.  Returns the number of steps.                 */
/* ------------------------------------------------------------------ */
int64_t orc_extend_labeling_via_voronoi(const uint32_t *src, uint32_t *out, int64_t D,
                                        int64_t H, int64_t W, int ndim) {
    const int64_t n = D * H * W;
    uint32_t *a = (uint32_t *)malloc(sizeof(uint32_t) * n);
    uint32_t *b = (uint32_t *)malloc(sizeof(uint32_t) * n);
    memcpy(a, src, sizeof(uint32_t) * n);
    const int zr = (ndim == 3) ? 1 : 0;
    int64_t step = 0;
    for (;;) {
        const int box = (step % 2) == 0;
        int64_t changed = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : changed)
        for (int64_t z = 0; z < D; ++z)
            for (int64_t y = 0; y < H; ++y)
                for (int64_t x = 0; x < W; ++x) {
                    const int64_t p = IDX(z, y, x);
                    const uint32_t v = a[p];
                    if (v != 0) { b[p] = v; continue; }
                    uint32_t m = 0;
                    for (int dz = -zr; dz <= zr; ++dz)
                        for (int dy = -1; dy <= 1; ++dy)
                            for (int dx = -1; dx <= 1; ++dx) {
                                if (!box && (abs(dx) + abs(dy) + abs(dz)) > 1) continue;
                                const int64_t qz = z + dz, qy = y + dy, qx = x + dx;
                                if (qz < 0 || qz >= D || qy < 0 || qy >= H || qx < 0 || qx >= W)
                                    continue;
                                const uint32_t q = a[IDX(qz, qy, qx)];
                                if (q > m) m = q;
                            }
                    b[p] = m;
                    if (m != 0) changed++;
                }
        uint32_t *t = a; a = b; b = t;
        step++;
        if (changed == 0) break;
    }
    memcpy(out, a, sizeof(uint32_t) * n);
    free(a); free(b);
    return step;
}

/* voronoi_labeling: _tier5/_voronoi_labeling.py:36-40 -- connected       */
/* components (box), then extend_labeling_via_voronoi.                    */
int64_t orc_voronoi_labeling(const uint8_t *fg, uint32_t *out, int64_t D, int64_t H, int64_t W,
                             int ndim) {
    const int64_t n = D * H * W;
    uint32_t *cc = (uint32_t *)malloc(sizeof(uint32_t) * n);
    orc_ccl_box(fg, cc, D, H, W);
    const int64_t steps = orc_extend_labeling_via_voronoi(cc, out, D, H, W, ndim);
    free(cc);
    return steps;
}

/* ------------------------------------------------------------------ */
/* A1-A12 voronoi_otsu_labeling: _tier9/_voronoi_otsu_labeling.py:57-71*/
/* Optional debug outputs (may be NULL): spots (u8), seg (u8),         */
/* threshold (double).                                                 */
/* ------------------------------------------------------------------ */
int64_t orc_voronoi_otsu_labeling(const float *src, uint32_t *labels, int64_t D, int64_t H,
                                  int64_t W, int ndim, double spot_sigma, double outline_sigma,
                                  uint8_t *spots_out, uint8_t *seg_out, double *thr_out) {
    const int64_t n = D * H * W;
    float *tmp = (float *)malloc(sizeof(float) * n);
    uint8_t *spots = (uint8_t *)malloc(n);
    uint8_t *seg = (uint8_t *)malloc(n);
    float *segf = (float *)malloc(sizeof(float) * n);
    orc_gaussian_blur(src, tmp, D, H, W, ndim, spot_sigma, spot_sigma, spot_sigma);
    orc_detect_maxima(tmp, spots, D, H, W, ndim);
    orc_gaussian_blur(src, tmp, D, H, W, ndim, outline_sigma, outline_sigma, outline_sigma);
    double t = orc_threshold_otsu(tmp, seg, D, H, W);
    orc_binary_and(spots, seg, spots, n);
    for (int64_t i = 0; i < n; ++i) segf[i] = (float)seg[i];
    int64_t steps = orc_masked_voronoi(spots, segf, NULL, labels, D, H, W, ndim);
    if (spots_out) memcpy(spots_out, spots, n);
    if (seg_out) memcpy(seg_out, seg, n);
    if (thr_out) *thr_out = t;
    free(tmp); free(spots); free(seg); free(segf);
    return steps;
}

/* ------------------------------------------------------------------ */
/* A13 statistics_of_labelled_pixels:                                  */
/* _tier9/_statistics_of_labelled_pixels.py:56-291,                    */
/* _tier9/statistics_per_label_x.cl, standard_deviation_per_label_x.cl */
/* Labels 1..L where L = int(max label).  Accumulation in float64      */
/* (the reference accumulates float32 per row; agreement is checked at */
/* 1e-5 relative), every derived column computed from float32 values   */
/* exactly as the reference combines its float32 columns.  Labels      */
/* absent from the image keep the reference's sentinels: min/bbox-min  */
/* FLT_MAX, max/bbox-max -FLT_MAX, sums 0, 0/0 = NaN means.            */
/* out: ORC_NCOLS x L float32, columns in the reference's dict order   */
/* after 'label' and 'original_label'.                                 */
/* ------------------------------------------------------------------ */
enum {
    C_BBOX_MIN_X, C_BBOX_MIN_Y, C_BBOX_MIN_Z, C_BBOX_MAX_X, C_BBOX_MAX_Y, C_BBOX_MAX_Z,
    C_BBOX_W, C_BBOX_H, C_BBOX_D, C_MIN_I, C_MAX_I, C_SUM_I, C_AREA, C_MEAN_I,
    C_SUM_IX, C_MASS_X, C_SUM_IY, C_MASS_Y, C_SUM_IZ, C_MASS_Z,
    C_SUM_X, C_CEN_X, C_SUM_Y, C_CEN_Y, C_SUM_Z, C_CEN_Z,
    C_SUM_DC, C_MEAN_DC, C_SUM_DM, C_MEAN_DM, C_STD_I, C_MAX_DC, C_MAX_DM,
    C_RATIO_C, C_RATIO_M, ORC_NCOLS
};

int orc_stats_ncols(void) { return ORC_NCOLS; }

void orc_statistics(const float *inten, const uint32_t *lab, int64_t D, int64_t H, int64_t W,
                    int64_t L, float *out) {
    double *acc = (double *)calloc((size_t)L * 8, sizeof(double));
    float *mnmx = (float *)malloc(sizeof(float) * L * 8);
    for (int64_t l = 0; l < L; ++l) {
        mnmx[l * 8 + 0] = FLT_MAX;  mnmx[l * 8 + 1] = -FLT_MAX;   /* intensity */
        mnmx[l * 8 + 2] = FLT_MAX;  mnmx[l * 8 + 3] = -FLT_MAX;   /* x */
        mnmx[l * 8 + 4] = FLT_MAX;  mnmx[l * 8 + 5] = -FLT_MAX;   /* y */
        mnmx[l * 8 + 6] = FLT_MAX;  mnmx[l * 8 + 7] = -FLT_MAX;   /* z */
    }
    for (int64_t z = 0; z < D; ++z)
        for (int64_t y = 0; y < H; ++y)
            for (int64_t x = 0; x < W; ++x) {
                uint32_t l = lab[IDX(z, y, x)];
                if (l == 0 || l > (uint32_t)L) continue;
                double v = inten[IDX(z, y, x)];
                double *a = acc + (l - 1) * 8;
                float *m = mnmx + (l - 1) * 8;
                a[0] += x; a[1] += y; a[2] += z; a[3] += 1.0;
                a[4] += v * x; a[5] += v * y; a[6] += v * z; a[7] += v;
                float fv = (float)v;
                if (fv < m[0]) m[0] = fv;
                if (fv > m[1]) m[1] = fv;
                if ((float)x < m[2]) m[2] = (float)x;
                if ((float)x > m[3]) m[3] = (float)x;
                if ((float)y < m[4]) m[4] = (float)y;
                if ((float)y > m[5]) m[5] = (float)y;
                if ((float)z < m[6]) m[6] = (float)z;
                if ((float)z > m[7]) m[7] = (float)z;
            }
#define O(c, l) out[(int64_t)(c) * L + (l)]
    for (int64_t l = 0; l < L; ++l) {
        double *a = acc + l * 8;
        float *m = mnmx + l * 8;
        float area = (float)a[3];
        float sum_i = (float)a[7];
        O(C_BBOX_MIN_X, l) = m[2]; O(C_BBOX_MIN_Y, l) = m[4]; O(C_BBOX_MIN_Z, l) = m[6];
        O(C_BBOX_MAX_X, l) = m[3]; O(C_BBOX_MAX_Y, l) = m[5]; O(C_BBOX_MAX_Z, l) = m[7];
        O(C_BBOX_W, l) = (m[3] - m[2]) + 1.0f;
        O(C_BBOX_H, l) = (m[5] - m[4]) + 1.0f;
        O(C_BBOX_D, l) = (m[7] - m[6]) + 1.0f;
        O(C_MIN_I, l) = m[0];
        O(C_MAX_I, l) = m[1];
        O(C_SUM_I, l) = sum_i;
        O(C_AREA, l) = area;
        O(C_MEAN_I, l) = sum_i / area;
        O(C_SUM_IX, l) = (float)a[4]; O(C_MASS_X, l) = (float)a[4] / sum_i;
        O(C_SUM_IY, l) = (float)a[5]; O(C_MASS_Y, l) = (float)a[5] / sum_i;
        O(C_SUM_IZ, l) = (float)a[6]; O(C_MASS_Z, l) = (float)a[6] / sum_i;
        O(C_SUM_X, l) = (float)a[0]; O(C_CEN_X, l) = (float)a[0] / area;
        O(C_SUM_Y, l) = (float)a[1]; O(C_CEN_Y, l) = (float)a[1] / area;
        O(C_SUM_Z, l) = (float)a[2]; O(C_CEN_Z, l) = (float)a[2] / area;
    }
    /* second pass: distances and squared intensity deviations using the
     * float32 centroid / mass centre / mean / area */
    double *acc2 = (double *)calloc((size_t)L * 3, sizeof(double));
    double *mx2 = (double *)calloc((size_t)L * 2, sizeof(double));
    for (int64_t z = 0; z < D; ++z)
        for (int64_t y = 0; y < H; ++y)
            for (int64_t x = 0; x < W; ++x) {
                uint32_t l = lab[IDX(z, y, x)];
                if (l == 0 || l > (uint32_t)L) continue;
                int64_t i = l - 1;
                double v = inten[IDX(z, y, x)];
                double cx = O(C_CEN_X, i), cy = O(C_CEN_Y, i), cz = O(C_CEN_Z, i);
                double mxc = O(C_MASS_X, i), myc = O(C_MASS_Y, i), mzc = O(C_MASS_Z, i);
                double dc = sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz));
                double dm = sqrt((x - mxc) * (x - mxc) + (y - myc) * (y - myc) +
                                 (z - mzc) * (z - mzc));
                double dv = v - (double)O(C_MEAN_I, i);
                acc2[i * 3 + 0] += dc;
                acc2[i * 3 + 1] += dm;
                acc2[i * 3 + 2] += dv * dv / (double)O(C_AREA, i);
                if (dc > mx2[i * 2 + 0]) mx2[i * 2 + 0] = dc;
                if (dm > mx2[i * 2 + 1]) mx2[i * 2 + 1] = dm;
            }
    for (int64_t l = 0; l < L; ++l) {
        float area = O(C_AREA, l);
        float sdc = (float)acc2[l * 3 + 0], sdm = (float)acc2[l * 3 + 1];
        float mdc = sdc / area, mdm = sdm / area;
        float xdc = (float)mx2[l * 2 + 0], xdm = (float)mx2[l * 2 + 1];
        O(C_SUM_DC, l) = sdc; O(C_MEAN_DC, l) = mdc;
        O(C_SUM_DM, l) = sdm; O(C_MEAN_DM, l) = mdm;
        O(C_STD_I, l) = (float)sqrt(acc2[l * 3 + 2]);
        O(C_MAX_DC, l) = xdc; O(C_MAX_DM, l) = xdm;
        O(C_RATIO_C, l) = xdc / mdc;
        O(C_RATIO_M, l) = xdm / mdm;
    }
#undef O
    free(acc); free(mnmx); free(acc2); free(mx2);
}
