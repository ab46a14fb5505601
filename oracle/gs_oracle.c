/*
 * gs_oracle.c -- CPU oracle for the Gaussian-splat training step.  TEST INFRASTRUCTURE
 * ONLY: tests, the smoke check and the CPU-baseline arm of bench.py call it as the
 * checker; the product never links or calls it.
 *
 * Two independent restatements:
 *
 *  orc32_*  FP32, the reference's WGSL kernels of barakatiass-alt/home-measure-privacy
 *           (trainer/gpu.js) restated in C with the same operation order and AoS data:
 *           PREPROCESS/projectShape (:20-60, :64-88), BIN + SORT (:616-685; per-tile depth
 *           order with the splat-index tie-break of :673 and the TILE_CAP of :614),
 *           tileLists (:450-481), alphaAt + FORWARD (:91-137), SSIM_COEF + LOSS_GRAD
 *           (:336-409), BACKWARD (:139-202), SHAPE by f32 central differences
 *           (:297-328) and ADAM (:411-443).  Compiled with -ffp-contract=off so every
 *           operation rounds like WGSL's f32 arithmetic; the projection's exp is the
 *           specified exp of the product (same reduction, polynomial and rounding
 *           steps), so projected records and tile keys match the CUDA path bit for bit.
 *           OpenMP parallelises the same work items the WGSL dispatches over; the
 *           backward's float atomics are OpenMP atomics.  This is also the timed CPU
 *           baseline.
 *
 *  d64_*    FP64 forward (same rules: near cull, 0.3 dilation, integer radius, alpha
 *           cap/floor, T stop) and its analytic adjoint, written from the mathematics
 *           with its own SH constants computed from the normalisation formula.  The
 *           tests pin it with central finite differences of d64_render (h = 1e-4) and
 *           use it as the gradient truth for the CUDA path.
 *
 * SH degree >= 1 and the 11-tap Gaussian SSIM window are extensions the reference does
 * not have (its colour is raw RGB, :87; its SSIM window a 7x7 box, :352): the colour is
 * rgb = dc + sum_{k>=1} Y_k(d) c_k with d = normalize(mean - camera centre).
 *
 * Golden vectors: the reference's only stored check is trainer/ssim-test.html (loss
 * gradient vs FP64 finite differences, W=20, H=14, lambda=0.2, Park-Miller LCG seed 7);
 * tests/golden holds that case.  Raster, binning, backward and Adam have no golden
 * outputs in the reference (it runs only under WebGPU in a browser): for those, parity
 * is pinned by the FP64 finite-difference check, not by outputs of the reference.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EXPORT __attribute__((visibility("default")))

typedef struct OrcCamera {
    float view[12];
    float fx, fy, cx, cy;
    int32_t width, height;
} OrcCamera;

static int nk_of(int degree) { return (degree + 1) * (degree + 1) - 1; }
EXPORT int orc_stride(int degree) { return 14 + 3 * nk_of(degree); }

/* ============================== FP32 restatement ================================== */

static float bits_float(uint32_t b) {
    float f;
    memcpy(&f, &b, 4);
    return f;
}
static uint32_t float_bits(float f) {
    uint32_t b;
    memcpy(&b, &f, 4);
    return b;
}

/* The product's specified single-precision exp: x = k ln2 + r (k = rint(x / ln2), ln2
 * split 0x3f317200 + tail), e^r by the degree-7 Taylor polynomial in Horner form, times
 * 2^k; one rounding per operation. */
static float spec_expf(float x) {
    if (!(x > -87.0f)) return (x != x) ? x : 0.0f;
    if (x > 88.0f) return bits_float(0x7f800000u);
    const float k = rintf(x * 1.44269502162933349609375f);
    const float r = (x - k * 0.693145751953125f) - k * 1.428606765330187045e-06f;
    float p = 1.98412698412698412698e-04f;
    p = p * r + 1.38888888888888888889e-03f;
    p = p * r + 8.33333333333333333333e-03f;
    p = p * r + 4.16666666666666666667e-02f;
    p = p * r + 1.66666666666666666667e-01f;
    p = p * r + 0.5f;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    return p * bits_float((uint32_t)(((int)k + 127) << 23));
}

typedef struct {
    int ok;
    float u, v, a, b, c, radius, depth;
} Proj32;

/* projectShape (trainer/gpu.js:30-60). q: mean.xyz, logScale.xyz, rotation.wxyz. */
static Proj32 project32(const OrcCamera* cam, const float q[10], float near, float dil) {
    Proj32 o;
    memset(&o, 0, sizeof o);
    const float* m = cam->view;
    const float r0[4] = {m[0], m[1], m[2], m[3]}, r1[4] = {m[4], m[5], m[6], m[7]}, r2[4] = {m[8], m[9], m[10], m[11]};
    const float px = ((r0[0] * q[0] + r0[1] * q[1]) + r0[2] * q[2]) + r0[3];
    const float py = ((r1[0] * q[0] + r1[1] * q[1]) + r1[2] * q[2]) + r1[3];
    const float pz = ((r2[0] * q[0] + r2[1] * q[1]) + r2[2] * q[2]) + r2[3];
    o.depth = pz;
    if (pz < near) return o;
    const float s[3] = {spec_expf(q[3]), spec_expf(q[4]), spec_expf(q[5])};
    /* quatToMat (:20-27) */
    const float len = sqrtf(((q[6] * q[6] + q[7] * q[7]) + q[8] * q[8]) + q[9] * q[9]);
    const float dd = len > 1e-12f ? len : 1e-12f;
    const float w = q[6] / dd, x = q[7] / dd, y = q[8] / dd, z = q[9] / dd;
    float R[3][3];
    R[0][0] = 1.0f - 2.0f * (y * y + z * z);
    R[1][0] = 2.0f * (x * y + w * z);
    R[2][0] = 2.0f * (x * z - w * y);
    R[0][1] = 2.0f * (x * y - w * z);
    R[1][1] = 1.0f - 2.0f * (x * x + z * z);
    R[2][1] = 2.0f * (y * z + w * x);
    R[0][2] = 2.0f * (x * z + w * y);
    R[1][2] = 2.0f * (y * z - w * x);
    R[2][2] = 1.0f - 2.0f * (x * x + y * y);
    float M[3][3], S[3][3], W[3][3], A[3][3], C[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) M[i][j] = R[i][j] * s[j];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) S[i][j] = (M[i][0] * M[j][0] + M[i][1] * M[j][1]) + M[i][2] * M[j][2];
    for (int j = 0; j < 3; j++) {
        W[0][j] = r0[j];
        W[1][j] = r1[j];
        W[2][j] = r2[j];
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) A[i][j] = (W[i][0] * S[0][j] + W[i][1] * S[1][j]) + W[i][2] * S[2][j];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) C[i][j] = (A[i][0] * W[j][0] + A[i][1] * W[j][1]) + A[i][2] * W[j][2];
    const float fx = cam->fx, fy = cam->fy;
    const float zz = pz * pz;
    const float j00 = fx / pz, j02 = (-fx * px) / zz;
    const float j11 = fy / pz, j12 = (-fy * py) / zz;
    const float cj0_0 = C[0][0] * j00 + C[0][2] * j02;
    const float cj0_2 = C[2][0] * j00 + C[2][2] * j02;
    const float cj1_0 = C[0][1] * j11 + C[0][2] * j12;
    const float cj1_1 = C[1][1] * j11 + C[1][2] * j12;
    const float cj1_2 = C[2][1] * j11 + C[2][2] * j12;
    const float a = (j00 * cj0_0 + j02 * cj0_2) + dil;
    const float b = j00 * cj1_0 + j02 * cj1_2;
    const float c = (j11 * cj1_1 + j12 * cj1_2) + dil;
    const float det = a * c - b * b;
    if (!(det > 0.0f)) return o;
    const float mid = (a + c) * 0.5f;
    o.ok = 1;
    o.u = fx * (px / pz) + cam->cx;
    o.v = fy * (py / pz) + cam->cy;
    o.a = c / det;
    o.b = -b / det;
    o.c = a / det;
    const float inner = mid * mid - det;
    o.radius = ceilf(3.0f * sqrtf(mid + sqrtf(inner > 0.1f ? inner : 0.1f)));
    return o;
}

/* SH basis constants (float), coefficient order k = l^2 + l + m, k >= 1. */
static void sh32(int degree, float x, float y, float z, float* Y) {
    if (degree < 1) return;
    const float c1 = 0.48860251190291992f;
    Y[0] = -c1 * y;
    Y[1] = c1 * z;
    Y[2] = -c1 * x;
    if (degree < 2) return;
    const float xx = x * x, yy = y * y, zz = z * z;
    Y[3] = 1.0925484305920792f * x * y;
    Y[4] = -1.0925484305920792f * y * z;
    Y[5] = 0.31539156525252005f * (2.0f * zz - xx - yy);
    Y[6] = -1.0925484305920792f * x * z;
    Y[7] = 0.54627421529603959f * (xx - yy);
    if (degree < 3) return;
    Y[8] = -0.59004358992664352f * y * (3.0f * xx - yy);
    Y[9] = 2.8906114426405538f * x * y * z;
    Y[10] = -0.45704579946446572f * y * (4.0f * zz - xx - yy);
    Y[11] = 0.37317633259011540f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
    Y[12] = -0.45704579946446572f * x * (4.0f * zz - xx - yy);
    Y[13] = 1.4453057213202769f * z * (xx - yy);
    Y[14] = -0.59004358992664352f * x * (xx - 3.0f * yy);
}

static void shape_of(const float* rec, float q[10]) {
    q[0] = rec[0]; q[1] = rec[1]; q[2] = rec[2];
    q[3] = rec[3]; q[4] = rec[4]; q[5] = rec[5];
    q[6] = rec[6]; q[7] = rec[7]; q[8] = rec[8]; q[9] = rec[9];
}

/* PREPROCESS (trainer/gpu.js:64-88): 12-float splat records. params: host records
 * (mean3, logScale3, rot4, opacityLogit, colour3, SH rest). */
EXPORT void orc32_preprocess(const OrcCamera* cam, const float* params, int n, int degree, float near, float dil,
                             float* splats) {
    const int S = orc_stride(degree), NK = nk_of(degree);
    const float* m = cam->view;
    float campos[3];
    for (int j = 0; j < 3; j++) campos[j] = -(m[0 + j] * m[3] + m[4 + j] * m[7] + m[8 + j] * m[11]);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        const float* g = params + (size_t)i * S;
        float* o = splats + (size_t)i * 12;
        float q[10];
        shape_of(g, q);
        const Proj32 p = project32(cam, q, near, dil);
        memset(o, 0, 12 * sizeof(float));
        o[11] = p.ok ? 1.0f : 0.0f;
        if (!p.ok) continue;
        o[0] = p.u; o[1] = p.v; o[2] = p.a; o[3] = p.b; o[4] = p.c;
        o[5] = 1.0f / (1.0f + spec_expf(-g[10]));
        o[6] = p.radius;
        o[7] = p.depth;
        float rgb[3] = {g[11], g[12], g[13]};
        if (degree > 0) {
            float dx = g[0] - campos[0], dy = g[1] - campos[1], dz = g[2] - campos[2];
            const float inv = 1.0f / sqrtf(dx * dx + dy * dy + dz * dz);
            dx *= inv; dy *= inv; dz *= inv;
            float Y[15];
            sh32(degree, dx, dy, dz, Y);
            for (int c = 0; c < 3; c++)
                for (int k = 0; k < NK; k++) rgb[c] += Y[k] * g[14 + c * NK + k];
        }
        o[8] = rgb[0]; o[9] = rgb[1]; o[10] = rgb[2];
    }
}

/* Tile rectangle, half-open.  mode 0: BIN (trainer/gpu.js:632-635, f32); mode 1:
 * tileLists (:456-461, f64 like JS). */
static void rect32(float u, float v, float r, int tx, int ty, int mode, int* x0, int* x1, int* y0, int* y1) {
    if (mode == 0) {
        float fx0 = floorf(((u - r) - 0.5f) / 16.0f), fx1 = floorf(((u + r) - 0.5f) / 16.0f);
        float fy0 = floorf(((v - r) - 0.5f) / 16.0f), fy1 = floorf(((v + r) - 0.5f) / 16.0f);
        fx0 = fminf(fmaxf(fx0, 0.0f), (float)(tx - 1));
        fx1 = fminf(fmaxf(fx1, -1.0f), (float)(tx - 1));
        fy0 = fminf(fmaxf(fy0, 0.0f), (float)(ty - 1));
        fy1 = fminf(fmaxf(fy1, -1.0f), (float)(ty - 1));
        *x0 = (int)fx0; *x1 = (int)(fx1 + 1.0f);
        *y0 = (int)fy0; *y1 = (int)(fy1 + 1.0f);
    } else {
        const double du = u, dv = v, dr = r;
        double a0 = floor((du - dr - 0.5) / 16.0), a1 = floor((du + dr - 0.5) / 16.0);
        double b0 = floor((dv - dr - 0.5) / 16.0), b1 = floor((dv + dr - 0.5) / 16.0);
        *x0 = (int)fmax(0.0, a0); *x1 = (int)fmin((double)(tx - 1), a1) + 1;
        *y0 = (int)fmax(0.0, b0); *y1 = (int)fmin((double)(ty - 1), b1) + 1;
    }
    if (*x1 < *x0) *x1 = *x0;
    if (*y1 < *y0) *y1 = *y0;
}

typedef struct {
    float depth;
    uint32_t idx;
} DepthIdx;

static int cmp_depth_idx(const void* pa, const void* pb) {
    const DepthIdx* a = (const DepthIdx*)pa;
    const DepthIdx* b = (const DepthIdx*)pb;
    if (a->depth < b->depth) return -1;
    if (a->depth > b->depth) return 1;
    return (a->idx > b->idx) - (a->idx < b->idx);
}

/* Per-tile buckets of BIN + SORT: each tile's entries (depth, splat index), first filled
 * in splat-index order, then the first min(count, cap) of them sorted by (depth, index).
 * The rectangles and the per-tile sorts run in parallel; the fill is sequential, so the
 * bucket order (and with it which entries a cap keeps) does not depend on threads. */
typedef struct {
    DepthIdx* buf;
    int64_t* start;
    int64_t* count;   /* entries kept per tile (capped) */
    int64_t total;    /* sum of count */
    int tiles;
} Bins;

static void bins_build(Bins* b, const float* splats, int n, int W, int H, int rect_mode, int cap) {
    const int tx = (W + 15) / 16, ty = (H + 15) / 16, tiles = tx * ty;
    int32_t* rect = (int32_t*)malloc(sizeof(int32_t) * 4 * (size_t)(n > 0 ? n : 1));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        const float* s = splats + (size_t)i * 12;
        int32_t* r = rect + (size_t)i * 4;
        if (s[11] < 0.5f) {
            r[0] = r[1] = r[2] = r[3] = 0;
            continue;
        }
        int x0, x1, y0, y1;
        rect32(s[0], s[1], s[6], tx, ty, rect_mode, &x0, &x1, &y0, &y1);
        r[0] = x0; r[1] = x1; r[2] = y0; r[3] = y1;
    }
    int64_t* all = (int64_t*)calloc((size_t)tiles + 1, sizeof(int64_t));
    for (int i = 0; i < n; i++) {
        const int32_t* r = rect + (size_t)i * 4;
        for (int y = r[2]; y < r[3]; y++)
            for (int x = r[0]; x < r[1]; x++) all[y * tx + x]++;
    }
    b->tiles = tiles;
    b->start = (int64_t*)calloc((size_t)tiles + 1, sizeof(int64_t));
    b->count = (int64_t*)calloc((size_t)tiles + 1, sizeof(int64_t));
    int64_t run = 0;
    b->total = 0;
    for (int t = 0; t < tiles; t++) {
        b->start[t] = run;
        run += all[t];
        b->count[t] = (cap > 0 && all[t] > cap) ? cap : all[t];
        b->total += b->count[t];
    }
    b->buf = (DepthIdx*)malloc(sizeof(DepthIdx) * (size_t)(run > 0 ? run : 1));
    memset(all, 0, sizeof(int64_t) * ((size_t)tiles + 1));
    for (int i = 0; i < n; i++) {
        const int32_t* r = rect + (size_t)i * 4;
        const DepthIdx e = {splats[(size_t)i * 12 + 7], (uint32_t)i};
        for (int y = r[2]; y < r[3]; y++)
            for (int x = r[0]; x < r[1]; x++) {
                const int t = y * tx + x;
                b->buf[b->start[t] + all[t]++] = e;
            }
    }
#pragma omp parallel for schedule(dynamic, 8)
    for (int t = 0; t < tiles; t++) qsort(b->buf + b->start[t], (size_t)b->count[t], sizeof(DepthIdx), cmp_depth_idx);
    free(all);
    free(rect);
}

static void bins_free(Bins* b) {
    free(b->buf);
    free(b->start);
    free(b->count);
}

/* Compact list, [start, end) per tile and (optional) keys tile << 32 | depth bits. */
static void bins_write(const Bins* b, uint32_t* list_out, uint32_t* ranges_out, uint64_t* keys_out) {
    int64_t pos = 0;
    for (int t = 0; t < b->tiles; t++) {
        ranges_out[2 * t] = (uint32_t)pos;
        pos += b->count[t];
        ranges_out[2 * t + 1] = (uint32_t)pos;
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int t = 0; t < b->tiles; t++) {
        int64_t o = ranges_out[2 * t];
        for (int64_t k = 0; k < b->count[t]; k++, o++) {
            const DepthIdx e = b->buf[b->start[t] + k];
            if (list_out) list_out[o] = e.idx;
            if (keys_out) keys_out[o] = ((uint64_t)t << 32) | float_bits(e.depth);
        }
    }
}

/* BIN + SORT (trainer/gpu.js:616-685) or tileLists (:450-481): per tile, the valid splats
 * whose rectangle covers it, in (depth, splat index) order.  cap > 0 keeps the first
 * `cap` splats of a tile in splat-index order (the reference keeps the first `cap` to
 * win its atomic counter, an order that is not deterministic).  Writes the compact list
 * and [start, end) per tile; keys_out (optional) gets tile << 32 | depth bits.  Returns
 * the entry count, or -(needed) when list_cap is too small. */
EXPORT int64_t orc32_bin(const float* splats, int n, int W, int H, int rect_mode, int cap, uint32_t* list_out,
                         uint32_t* ranges_out, uint64_t* keys_out, int64_t list_cap) {
    Bins b;
    bins_build(&b, splats, n, W, H, rect_mode, cap);
    const int64_t total = b.total;
    if (total > list_cap) {
        bins_free(&b);
        return -total;
    }
    bins_write(&b, list_out, ranges_out, keys_out);
    bins_free(&b);
    return total;
}

/* alphaAt (trainer/gpu.js:91-103).  Returns alpha, or 0 when the splat is skipped.
 * WGSL leaves exp's last bits to the implementation (a few ulp); this restatement uses
 * the specified exp (spec_expf) that the CUDA path also uses wherever alpha decides a
 * skip, so that the two agree even when alpha is within an ulp of 1/255. */
static inline float alpha_at(const float* s, float px, float py, float amax, float amin, float* dxo, float* dyo) {
    const float dx = px - s[0], dy = py - s[1];
    const float r = s[6];
    if (fabsf(dx) > r || fabsf(dy) > r) return 0.0f;
    const float power = -0.5f * (s[2] * dx * dx + s[4] * dy * dy) - s[3] * dx * dy;
    if (power > 0.0f) return 0.0f;
    float alpha = s[5] * spec_expf(power);
    if (alpha > amax) alpha = amax;
    if (alpha < amin) return 0.0f;
    *dxo = dx;
    *dyo = dy;
    return alpha;
}

/* FORWARD (trainer/gpu.js:105-137).  state: final T and last (counted from the tile's
 * start, as a float). */
EXPORT void orc32_forward(const float* splats, const uint32_t* list, const uint32_t* ranges, int W, int H, float amax,
                          float amin, float tmin, float* image, float* state) {
    const int tx = (W + 15) / 16;
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const float px = (float)x + 0.5f, py = (float)y + 0.5f;
            const int tile = (y / 16) * tx + x / 16;
            const uint32_t start = ranges[2 * tile], end = ranges[2 * tile + 1];
            float T = 1.0f, r = 0.f, g = 0.f, b = 0.f;
            uint32_t last = start;
            for (uint32_t k = start; k < end; k++) {
                if (T <= tmin) break;
                const float* s = splats + (size_t)list[k] * 12;
                float dx, dy;
                const float alpha = alpha_at(s, px, py, amax, amin, &dx, &dy);
                if (alpha == 0.0f) continue;
                r += s[8] * alpha * T;
                g += s[9] * alpha * T;
                b += s[10] * alpha * T;
                T *= 1.0f - alpha;
                last = k + 1;
            }
            const size_t p = (size_t)y * W + x;
            image[p * 3] = r;
            image[p * 3 + 1] = g;
            image[p * 3 + 2] = b;
            state[p * 2] = T;
            state[p * 2 + 1] = (float)(last - start);
        }
}

/* SSIM_COEF + LOSS_GRAD (trainer/gpu.js:336-409); window 0 = 7x7 box (the reference),
 * window 1 = 11-tap Gaussian sigma 1.5 with the same fully-inside rule.  loss_out
 * (optional): (1 - lambda) L1 + lambda (1 - mean SSIM). */
EXPORT void orc32_loss_grad(const float* image, const float* target, int W, int H, float lambda, int window,
                            float* grad, double* loss_out) {
    const int R = window == 0 ? 3 : 5, K = 2 * R + 1;
    float w2[11 * 11];
    if (window == 0) {
        for (int k = 0; k < 49; k++) w2[k] = 1.0f / 49.0f;
    } else {
        double g[11], s = 0.0;
        for (int k = 0; k < 11; k++) {
            g[k] = exp(-(double)(k - 5) * (k - 5) / (2.0 * 1.5 * 1.5));
            s += g[k];
        }
        for (int a = 0; a < 11; a++)
            for (int b = 0; b < 11; b++) w2[a * 11 + b] = (float)(g[a] / s * g[b] / s);
    }
    const size_t npx = (size_t)W * H;
    float* coef = (float*)calloc(npx * 9, sizeof(float));
    const float n = (float)(npx * 3);
    const int wx = W - 2 * R, wy = H - 2 * R;
    const float windows = (wx > 0 && wy > 0) ? (float)wx * (float)wy * 3.0f : 0.0f;
    double ssim_total = 0.0, l1_total = 0.0;
    if (lambda > 0.0f && windows > 0.0f) {
#pragma omp parallel for schedule(static) reduction(+ : ssim_total)
        for (int y = R; y < H - R; y++)
            for (int x = R; x < W - R; x++)
                for (int c = 0; c < 3; c++) {
                    float mx = 0.f, my = 0.f, sxx = 0.f, syy = 0.f, sxy = 0.f;
                    for (int dy = 0; dy < K; dy++)
                        for (int dx = 0; dx < K; dx++) {
                            const size_t q = ((size_t)(y + dy - R) * W + (x + dx - R)) * 3 + c;
                            const float xv = image[q], yv = target[q], w = w2[dy * K + dx];
                            if (window == 0) {
                                mx += xv; my += yv; sxx += xv * xv; syy += yv * yv; sxy += xv * yv;
                            } else {
                                mx += w * xv; my += w * yv; sxx += w * xv * xv; syy += w * yv * yv; sxy += w * xv * yv;
                            }
                        }
                    if (window == 0) {
                        mx /= 49.0f; my /= 49.0f; sxx /= 49.0f; syy /= 49.0f; sxy /= 49.0f;
                    }
                    const float c1 = 0.0001f, c2 = 0.0009f;
                    const float a1 = 2.0f * mx * my + c1;
                    const float a2 = 2.0f * (sxy - mx * my) + c2;
                    const float b1 = mx * mx + my * my + c1;
                    const float b2 = (sxx - mx * mx) + (syy - my * my) + c2;
                    const float ssim = a1 * a2 / (b1 * b2);
                    ssim_total += ssim;
                    float* o = coef + ((size_t)y * W + x) * 9 + c * 3;
                    o[0] = ssim * (2.0f * my / a1 - 2.0f * my / a2 - 2.0f * mx / b1 + 2.0f * mx / b2);
                    o[1] = -ssim / b2;
                    o[2] = 2.0f * ssim / a2;
                }
    }
#pragma omp parallel for schedule(static) reduction(+ : l1_total)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            for (int c = 0; c < 3; c++) {
                const size_t q = ((size_t)y * W + x) * 3 + c;
                const float xv = image[q], yv = target[q];
                const float d = xv - yv;
                l1_total += fabs((double)d);
                float g = (1.0f - lambda) * (float)((d > 0.0f) - (d < 0.0f)) / n;
                if (lambda > 0.0f && windows > 0.0f) {
                    float sa = 0.f, sb = 0.f, sd = 0.f;
                    for (int dy = -R; dy <= R; dy++)
                        for (int dx = -R; dx <= R; dx++) {
                            const int cx = x + dx, cy = y + dy;
                            if (cx < 0 || cy < 0 || cx >= W || cy >= H) continue;
                            const float* k = coef + ((size_t)cy * W + cx) * 9 + c * 3;
                            /* The window centred at (cx, cy) weighs this pixel by w(-dx,-dy). */
                            const float w = window == 0 ? 1.0f : w2[(R - dy) * K + (R - dx)];
                            sa += w * k[0];
                            sb += w * k[1];
                            sd += w * k[2];
                        }
                    const float dssim = window == 0 ? (sa + 2.0f * xv * sb + yv * sd) / 49.0f / windows
                                                    : (sa + 2.0f * xv * sb + yv * sd) / windows;
                    g -= lambda * dssim;
                }
                grad[q] = g;
            }
    if (loss_out) {
        const double l1 = l1_total / (double)(npx * 3);
        const double ssim = windows > 0.0f ? ssim_total / windows : 1.0;
        *loss_out = (1.0 - lambda) * l1 + (lambda > 0.0f ? lambda * (1.0 - ssim) : 0.0);
    }
    free(coef);
}

/* BACKWARD (trainer/gpu.js:139-202), per pixel, back to front from `last`.  grads16
 * accumulates (0-2 colour, 3 opacity logit, 4-8 u, v, A, B, C) with float atomics. */
EXPORT void orc32_backward(const float* splats, const uint32_t* list, const uint32_t* ranges, const float* state,
                           const float* dl, int W, int H, float amax, float amin, float* grads16) {
    const int tx = (W + 15) / 16;
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const size_t p = (size_t)y * W + x;
            const float px = (float)x + 0.5f, py = (float)y + 0.5f;
            const int tile = (y / 16) * tx + x / 16;
            const uint32_t start = ranges[2 * tile];
            const float dL[3] = {dl[p * 3], dl[p * 3 + 1], dl[p * 3 + 2]};
            float T = state[p * 2];
            uint32_t k = start + (uint32_t)state[p * 2 + 1];
            float behind[3] = {0.f, 0.f, 0.f};
            while (k > start) {
                k--;
                const uint32_t gi = list[k];
                const float* s = splats + (size_t)gi * 12;
                float dx, dy;
                const float alpha = alpha_at(s, px, py, amax, amin, &dx, &dy);
                if (alpha == 0.0f) continue;
                const float Tk = T / (1.0f - alpha);
                float* g = grads16 + (size_t)gi * 16;
                const float c[3] = {s[8], s[9], s[10]};
                float v[9] = {0.f};
                v[0] = dL[0] * alpha * Tk;
                v[1] = dL[1] * alpha * Tk;
                v[2] = dL[2] * alpha * Tk;
                const float dA = dL[0] * (Tk * c[0] - behind[0] / (1.0f - alpha)) +
                                 dL[1] * (Tk * c[1] - behind[1] / (1.0f - alpha)) +
                                 dL[2] * (Tk * c[2] - behind[2] / (1.0f - alpha));
                for (int j = 0; j < 3; j++) behind[j] += c[j] * alpha * Tk;
                T = Tk;
                if (alpha < amax) {
                    const float op = s[5];
                    v[3] = dA * (alpha / op) * op * (1.0f - op);
                    const float dP = dA * alpha;
                    const float A = s[2], B = s[3], C = s[4];
                    v[4] = dP * (A * dx + B * dy);
                    v[5] = dP * (C * dy + B * dx);
                    v[6] = dP * -0.5f * dx * dx;
                    v[7] = dP * -dx * dy;
                    v[8] = dP * -0.5f * dy * dy;
                }
                for (int j = 0; j < 9; j++)
                    if (v[j] != 0.0f) {
#pragma omp atomic
                        g[j] += v[j];
                    }
            }
        }
}

/* SHAPE (trainer/gpu.js:297-328): screen gradients chained to mean, logScale, rotation
 * by f32 central differences of projectShape (h = 1e-3, 2e-3 for the rotation). */
EXPORT void orc32_shape_fd(const OrcCamera* cam, const float* params, int n, int degree, float near, float dil,
                           const float* grads16, float* shape10) {
    const int S = orc_stride(degree);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        const float* gg = grads16 + (size_t)i * 16;
        const float sg[5] = {gg[4], gg[5], gg[6], gg[7], gg[8]};
        float base[10];
        shape_of(params + (size_t)i * S, base);
        for (int k = 0; k < 10; k++) {
            const float h = k >= 6 ? 2e-3f : 1e-3f;
            float up[10], down[10];
            memcpy(up, base, sizeof up);
            memcpy(down, base, sizeof down);
            up[k] = base[k] + h;
            down[k] = base[k] - h;
            const Proj32 a = project32(cam, up, near, dil);
            const Proj32 b = project32(cam, down, near, dil);
            float d = 0.0f;
            if (a.ok && b.ok)
                d = (sg[0] * (a.u - b.u) + sg[1] * (a.v - b.v) + sg[2] * (a.a - b.a) + sg[3] * (a.b - b.b) +
                     sg[4] * (a.c - b.c)) /
                    (2.0f * h);
            shape10[(size_t)i * 10 + k] = d;
        }
    }
}

/* ADAM (trainer/gpu.js:411-443) over the host records: grads in record layout, moments
 * m and v in record layout.  lr[6]: colour, opacity, mean, scale, rotation, SH. */
EXPORT void orc32_adam(float* params, const float* grads, float* m, float* v, int n, int degree, int t, const float* lr,
                       float beta1, float beta2, float eps) {
    const int S = orc_stride(degree);
    const float bc1 = 1.0f - powf(beta1, (float)t), bc2 = 1.0f - powf(beta2, (float)t);
    const float omb1 = 1.0f - beta1, omb2 = 1.0f - beta2;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        float* p = params + (size_t)i * S;
        for (int k = 0; k < S; k++) {
            const size_t idx = (size_t)i * S + k;
            const float g = grads[idx];
            float l;
            if (k < 3) l = lr[2];
            else if (k < 6) l = lr[3];
            else if (k < 10) l = lr[4];
            else if (k == 10) l = lr[1];
            else if (k < 14) l = lr[0];
            else l = lr[5];
            m[idx] = beta1 * m[idx] + omb1 * g;
            v[idx] = beta2 * v[idx] + omb2 * g * g;
            p[k] -= l * (m[idx] / bc1) / (sqrtf(v[idx] / bc2) + eps);
        }
        for (int c = 11; c < 14; c++) p[c] = fminf(fmaxf(p[c], 0.0f), 1.0f);
        const float nrm = sqrtf(p[6] * p[6] + p[7] * p[7] + p[8] * p[8] + p[9] * p[9]);
        const float d = nrm > 1e-12f ? nrm : 1e-12f;
        for (int k = 6; k < 10; k++) p[k] /= d;
    }
}

/* Buffers of the per-view step, sized for the largest view and reused across steps
 * (the reference keeps its step buffers in a scratch pool, trainer/gpu.js:764-772). */
typedef struct {
    float *splats, *image, *state, *dl, *g16, *shape, *grads, *target;
    size_t npx_cap;
} StepWork;

static void work_init(StepWork* w, int n, int S, size_t npx) {
    w->splats = (float*)malloc(sizeof(float) * 12 * (size_t)n);
    w->g16 = (float*)malloc(sizeof(float) * 16 * (size_t)n);
    w->shape = (float*)malloc(sizeof(float) * 10 * (size_t)n);
    w->grads = (float*)malloc(sizeof(float) * (size_t)S * n);
    w->image = (float*)malloc(sizeof(float) * npx * 3);
    w->state = (float*)malloc(sizeof(float) * npx * 2);
    w->dl = (float*)malloc(sizeof(float) * npx * 3);
    w->target = (float*)malloc(sizeof(float) * npx * 3);
    w->npx_cap = npx;
}

static void work_free(StepWork* w) {
    free(w->splats); free(w->g16); free(w->shape); free(w->grads);
    free(w->image); free(w->state); free(w->dl); free(w->target);
}

/* One step of trainScene on one view (trainer/gpu.js:915-933): PREPROCESS, BIN + SORT
 * (cap as given), FORWARD, loss gradient, BACKWARD, SHAPE by finite differences, STATS
 * (optional, :484-497) and ADAM at step t.  Colour grads of SH bands >= 1 come from the
 * colour grad and the basis (the extension above).  target: RGB floats. */
static double step_view(StepWork* w, const OrcCamera* cam, float* params, float* m, float* v, float* stats, int n,
                        int degree, const float* target, float lambda, int window, int t, const float* lr, float near,
                        int cap) {
    const int W = cam->width, H = cam->height, S = orc_stride(degree), NK = nk_of(degree);
    orc32_preprocess(cam, params, n, degree, near, 0.3f, w->splats);
    Bins b;
    bins_build(&b, w->splats, n, W, H, 0, cap);
    uint32_t* ranges = (uint32_t*)malloc(sizeof(uint32_t) * 2 * (size_t)b.tiles);
    uint32_t* list = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(b.total > 0 ? b.total : 1));
    bins_write(&b, list, ranges, NULL);
    bins_free(&b);
    orc32_forward(w->splats, list, ranges, W, H, 0.99f, 1.0f / 255.0f, 1e-4f, w->image, w->state);
    double loss = 0.0;
    orc32_loss_grad(w->image, target, W, H, lambda, window, w->dl, &loss);
    memset(w->g16, 0, sizeof(float) * 16 * (size_t)n);
    orc32_backward(w->splats, list, ranges, w->state, w->dl, W, H, 0.99f, 1.0f / 255.0f, w->g16);
    orc32_shape_fd(cam, params, n, degree, near, 0.3f, w->g16, w->shape);
    const float* vm = cam->view;
    float campos[3];
    for (int j = 0; j < 3; j++) campos[j] = -(vm[0 + j] * vm[3] + vm[4 + j] * vm[7] + vm[8 + j] * vm[11]);
    float* grads = w->grads;
    const float* g16 = w->g16;
    const float* shape = w->shape;
    const float* splats = w->splats;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        float* g = grads + (size_t)i * S;
        for (int k = 0; k < 10; k++) g[k] = shape[(size_t)i * 10 + k];
        g[10] = g16[(size_t)i * 16 + 3];
        for (int c = 0; c < 3; c++) g[11 + c] = g16[(size_t)i * 16 + c];
        if (degree > 0) {
            const float* p = params + (size_t)i * S;
            float dx = p[0] - campos[0], dy = p[1] - campos[1], dz = p[2] - campos[2];
            const float inv = 1.0f / sqrtf(dx * dx + dy * dy + dz * dz);
            float Y[15];
            sh32(degree, dx * inv, dy * inv, dz * inv, Y);
            for (int c = 0; c < 3; c++)
                for (int k = 0; k < NK; k++) g[14 + c * NK + k] = Y[k] * g16[(size_t)i * 16 + c];
        }
        if (stats && splats[(size_t)i * 12 + 11] >= 0.5f) {
            const float gu = g16[(size_t)i * 16 + 4], gv = g16[(size_t)i * 16 + 5];
            stats[(size_t)i * 2] += sqrtf(gu * gu + gv * gv);
            stats[(size_t)i * 2 + 1] += 1.0f;
        }
    }
    orc32_adam(params, grads, m, v, n, degree, t, lr, 0.9f, 0.999f, 1e-8f);
    free(list);
    free(ranges);
    return loss;
}

/* One training step of the reference's trainScene for one view (in place on params, m,
 * v); returns the step's loss.  target: RGB floats. */
EXPORT double orc32_step(const OrcCamera* cam, float* params, float* m, float* v, int n, int degree, const float* target,
                         float lambda, int window, int t, const float* lr, float near, int cap) {
    StepWork w;
    work_init(&w, n, orc_stride(degree), (size_t)cam->width * cam->height);
    const double loss = step_view(&w, cam, params, m, v, NULL, n, degree, target, lambda, window, t, lr, near, cap);
    work_free(&w);
    return loss;
}

/* trainScene (trainer/gpu.js:894-933) over `nviews` views in the given order, one
 * reference step per view (steps t0, t0 + 1, ...): each step converts the view's RGB
 * bytes to floats (v / 255, :921), then runs the per-view step above with STATS into
 * `stats` (n x 2, optional).  targets_u8: the views' photos concatenated.  losses_out
 * (optional) gets each step's loss, seconds_out (optional) each step's wall time.  Buffers
 * are allocated once for all the steps. */
EXPORT void orc32_train_views(const OrcCamera* cams, int nviews, const uint8_t* targets_u8, float* params, float* m,
                              float* v, float* stats, int n, int degree, float lambda, int window, int t0,
                              const float* lr, float near, int cap, double* losses_out, double* seconds_out) {
    size_t npx_max = 0;
    for (int k = 0; k < nviews; k++) {
        const size_t npx = (size_t)cams[k].width * cams[k].height;
        if (npx > npx_max) npx_max = npx;
    }
    StepWork w;
    work_init(&w, n, orc_stride(degree), npx_max > 0 ? npx_max : 1);
    size_t off = 0;
    for (int k = 0; k < nviews; k++) {
        const size_t cnt = (size_t)cams[k].width * cams[k].height * 3;
#ifdef _OPENMP
        const double t_start = omp_get_wtime();
#endif
        const uint8_t* src = targets_u8 + off;
        float* dst = w.target;
#pragma omp parallel for schedule(static)
        for (long long j = 0; j < (long long)cnt; j++) dst[j] = (float)((double)src[j] / 255.0);  /* JS: f64, then f32 */
        const double loss =
            step_view(&w, &cams[k], params, m, v, stats, n, degree, w.target, lambda, window, t0 + k, lr, near, cap);
        if (losses_out) losses_out[k] = loss;
#ifdef _OPENMP
        if (seconds_out) seconds_out[k] = omp_get_wtime() - t_start;
#else
        if (seconds_out) seconds_out[k] = 0.0;
#endif
        off += cnt;
    }
    work_free(&w);
}

EXPORT int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

EXPORT void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ============================== FP64 forward + adjoint ============================ */

typedef struct {
    int ok;
    double p[3];          /* camera-space point */
    double u, v, a, b, c; /* screen position, 2D covariance (dilated) */
    double A, B, C;       /* conic */
    double radius, depth;
    double opacity;
    double rgb[3];
    double dir[3], dnorm; /* view direction (unit) and |mean - centre| */
    double Y[15];
} P64;

static void sh64_consts(double* K) {
    /* K_l^m = sqrt((2l+1)/(4 pi) (l-|m|)!/(l+|m|)!), times sqrt(2) for m != 0, times the
     * associated Legendre polynomial's leading factor; signs of the Condon-Shortley phase. */
    const double pi = 3.14159265358979323846;
    K[0] = -sqrt(3.0 / (4.0 * pi));           /* -y */
    K[1] = sqrt(3.0 / (4.0 * pi));            /*  z */
    K[2] = -sqrt(3.0 / (4.0 * pi));           /* -x */
    K[3] = 0.5 * sqrt(15.0 / pi);             /* xy */
    K[4] = -0.5 * sqrt(15.0 / pi);            /* yz */
    K[5] = 0.25 * sqrt(5.0 / pi);             /* 3z^2 - 1 = 2z^2 - x^2 - y^2 */
    K[6] = -0.5 * sqrt(15.0 / pi);            /* xz */
    K[7] = 0.25 * sqrt(15.0 / pi);            /* x^2 - y^2 */
    K[8] = -0.25 * sqrt(35.0 / (2.0 * pi));   /* y (3x^2 - y^2) */
    K[9] = 0.5 * sqrt(105.0 / pi);            /* xyz */
    K[10] = -0.25 * sqrt(21.0 / (2.0 * pi));  /* y (4z^2 - x^2 - y^2) */
    K[11] = 0.25 * sqrt(7.0 / pi);            /* z (2z^2 - 3x^2 - 3y^2) */
    K[12] = -0.25 * sqrt(21.0 / (2.0 * pi));  /* x (4z^2 - x^2 - y^2) */
    K[13] = 0.25 * sqrt(105.0 / pi);          /* z (x^2 - y^2) */
    K[14] = -0.25 * sqrt(35.0 / (2.0 * pi));  /* x (x^2 - 3y^2) */
}

EXPORT void d64_sh_constants(double* out15) { sh64_consts(out15); }

static void sh64(int degree, const double d[3], double* Y, double* dY /* 15x3 or NULL */) {
    double K[15];
    sh64_consts(K);
    const double x = d[0], y = d[1], z = d[2];
    double P[15], G[15][3];
    memset(G, 0, sizeof G);
    P[0] = y;  G[0][1] = 1;
    P[1] = z;  G[1][2] = 1;
    P[2] = x;  G[2][0] = 1;
    P[3] = x * y;  G[3][0] = y; G[3][1] = x;
    P[4] = y * z;  G[4][1] = z; G[4][2] = y;
    P[5] = 2 * z * z - x * x - y * y;  G[5][0] = -2 * x; G[5][1] = -2 * y; G[5][2] = 4 * z;
    P[6] = x * z;  G[6][0] = z; G[6][2] = x;
    P[7] = x * x - y * y;  G[7][0] = 2 * x; G[7][1] = -2 * y;
    P[8] = y * (3 * x * x - y * y);  G[8][0] = 6 * x * y; G[8][1] = 3 * x * x - 3 * y * y;
    P[9] = x * y * z;  G[9][0] = y * z; G[9][1] = x * z; G[9][2] = x * y;
    P[10] = y * (4 * z * z - x * x - y * y);
    G[10][0] = -2 * x * y; G[10][1] = 4 * z * z - x * x - 3 * y * y; G[10][2] = 8 * y * z;
    P[11] = z * (2 * z * z - 3 * x * x - 3 * y * y);
    G[11][0] = -6 * x * z; G[11][1] = -6 * y * z; G[11][2] = 6 * z * z - 3 * x * x - 3 * y * y;
    P[12] = x * (4 * z * z - x * x - y * y);
    G[12][0] = 4 * z * z - 3 * x * x - y * y; G[12][1] = -2 * x * y; G[12][2] = 8 * x * z;
    P[13] = z * (x * x - y * y);  G[13][0] = 2 * x * z; G[13][1] = -2 * y * z; G[13][2] = x * x - y * y;
    P[14] = x * (x * x - 3 * y * y);  G[14][0] = 3 * x * x - 3 * y * y; G[14][1] = -6 * x * y;
    const int nk = nk_of(degree);
    for (int k = 0; k < nk; k++) {
        Y[k] = K[k] * P[k];
        if (dY)
            for (int j = 0; j < 3; j++) dY[k * 3 + j] = K[k] * G[k][j];
    }
}

static void rot64(const double q[4], double R[3][3], double* qn, double* qlen) {
    const double len = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const double d = len > 1e-12 ? len : 1e-12;
    const double w = q[0] / d, x = q[1] / d, y = q[2] / d, z = q[3] / d;
    qn[0] = w; qn[1] = x; qn[2] = y; qn[3] = z;
    *qlen = d;
    R[0][0] = 1 - 2 * (y * y + z * z); R[0][1] = 2 * (x * y - w * z); R[0][2] = 2 * (x * z + w * y);
    R[1][0] = 2 * (x * y + w * z); R[1][1] = 1 - 2 * (x * x + z * z); R[1][2] = 2 * (y * z - w * x);
    R[2][0] = 2 * (x * z - w * y); R[2][1] = 2 * (y * z + w * x); R[2][2] = 1 - 2 * (x * x + y * y);
}

static void cam64(const OrcCamera* cam, double W[3][3], double t[3], double cpos[3]) {
    const float* m = cam->view;
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) W[i][j] = m[i * 4 + j];
        t[i] = m[i * 4 + 3];
    }
    for (int j = 0; j < 3; j++) cpos[j] = -(W[0][j] * t[0] + W[1][j] * t[1] + W[2][j] * t[2]);
}

static P64 project64(const OrcCamera* cam, const double* g, int degree, double near, double dil) {
    P64 o;
    memset(&o, 0, sizeof o);
    double W[3][3], t[3], cpos[3];
    cam64(cam, W, t, cpos);
    for (int i = 0; i < 3; i++) o.p[i] = W[i][0] * g[0] + W[i][1] * g[1] + W[i][2] * g[2] + t[i];
    o.depth = o.p[2];
    if (o.p[2] < near) return o;
    double R[3][3], qn[4], ql;
    rot64(g + 6, R, qn, &ql);
    const double s[3] = {exp(g[3]), exp(g[4]), exp(g[5])};
    double Sig[3][3], Cc[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0;
            for (int k = 0; k < 3; k++) acc += R[i][k] * s[k] * s[k] * R[j][k];
            Sig[i][j] = acc;
        }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0;
            for (int k = 0; k < 3; k++)
                for (int l = 0; l < 3; l++) acc += W[i][k] * Sig[k][l] * W[j][l];
            Cc[i][j] = acc;
        }
    const double z = o.p[2];
    const double J[2][3] = {{cam->fx / z, 0, -cam->fx * o.p[0] / (z * z)}, {0, cam->fy / z, -cam->fy * o.p[1] / (z * z)}};
    double cov[2][2];
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++) {
            double acc = 0;
            for (int k = 0; k < 3; k++)
                for (int l = 0; l < 3; l++) acc += J[a][k] * Cc[k][l] * J[b][l];
            cov[a][b] = acc;
        }
    o.a = cov[0][0] + dil;
    o.b = cov[0][1];
    o.c = cov[1][1] + dil;
    const double det = o.a * o.c - o.b * o.b;
    if (!(det > 0)) return o;
    o.ok = 1;
    o.u = cam->fx * o.p[0] / z + cam->cx;
    o.v = cam->fy * o.p[1] / z + cam->cy;
    o.A = o.c / det;
    o.B = -o.b / det;
    o.C = o.a / det;
    const double mid = 0.5 * (o.a + o.c);
    const double inner = mid * mid - det;
    o.radius = ceil(3.0 * sqrt(mid + sqrt(inner > 0.1 ? inner : 0.1)));
    o.opacity = 1.0 / (1.0 + exp(-g[10]));
    const int nk = nk_of(degree);
    double dv[3] = {g[0] - cpos[0], g[1] - cpos[1], g[2] - cpos[2]};
    o.dnorm = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
    for (int j = 0; j < 3; j++) o.dir[j] = dv[j] / o.dnorm;
    sh64(degree, o.dir, o.Y, NULL);
    for (int c = 0; c < 3; c++) {
        double acc = g[11 + c];
        for (int k = 0; k < nk; k++) acc += o.Y[k] * g[14 + c * nk + k];
        o.rgb[c] = acc;
    }
    return o;
}

typedef struct {
    double depth;
    int idx;
} D64Idx;

static int cmp_d64(const void* pa, const void* pb) {
    const D64Idx* a = (const D64Idx*)pa;
    const D64Idx* b = (const D64Idx*)pb;
    if (a->depth < b->depth) return -1;
    if (a->depth > b->depth) return 1;
    return (a->idx > b->idx) - (a->idx < b->idx);
}

static uint64_t fnv(uint64_t h, uint64_t v) {
    for (int k = 0; k < 8; k++) {
        h ^= (v >> (8 * k)) & 0xffu;
        h *= 1099511628211ull;
    }
    return h;
}

/* Candidate grid of the FP64 render: for each 16 x 16 block of pixels, the positions k
 * (into `order`, ascending) of the valid splats whose bounding square |dx|, |dy| <= radius
 * can reach a pixel of the block (with a one-pixel margin).  Every other splat fails
 * alpha64's box test at every pixel of the block, so walking a block's candidates in
 * order gives the same contributors as walking all valid splats. */
#define D64_BLOCK 16

typedef struct {
    int n, W, H;
    P64* P;
    int* order;   /* valid splats by (depth, index) */
    int nvalid;
    int nbx, nby;
    int64_t* cand_start;  /* [blocks + 1] */
    int* cand;            /* positions k into order */
    int64_t cand_max;     /* longest block list */
} Scene64;

static void scene64(Scene64* sc, const OrcCamera* cam, const double* params, int n, int degree, double near, double dil) {
    const int S = orc_stride(degree);
    sc->n = n;
    sc->W = cam->width;
    sc->H = cam->height;
    sc->P = (P64*)malloc(sizeof(P64) * (size_t)(n > 0 ? n : 1));
    D64Idx* tmp = (D64Idx*)malloc(sizeof(D64Idx) * (size_t)(n > 0 ? n : 1));
    int nv = 0;
    for (int i = 0; i < n; i++) {
        sc->P[i] = project64(cam, params + (size_t)i * S, degree, near, dil);
        if (sc->P[i].ok) {
            tmp[nv].depth = sc->P[i].depth;
            tmp[nv].idx = i;
            nv++;
        }
    }
    qsort(tmp, (size_t)nv, sizeof(D64Idx), cmp_d64);
    sc->order = (int*)malloc(sizeof(int) * (size_t)(nv > 0 ? nv : 1));
    for (int k = 0; k < nv; k++) sc->order[k] = tmp[k].idx;
    sc->nvalid = nv;
    free(tmp);
    const int nbx = (sc->W + D64_BLOCK - 1) / D64_BLOCK, nby = (sc->H + D64_BLOCK - 1) / D64_BLOCK;
    const int blocks = nbx * nby;
    sc->nbx = nbx;
    sc->nby = nby;
    int* rect = (int*)malloc(sizeof(int) * 4 * (size_t)(nv > 0 ? nv : 1));
    int64_t* cnt = (int64_t*)calloc((size_t)blocks + 1, sizeof(int64_t));
    for (int k = 0; k < nv; k++) {
        const P64* q = &sc->P[sc->order[k]];
        /* pixel x passes |x + 0.5 - u| <= r only for x in [u - r - 0.5, u + r - 0.5] */
        double bx0 = floor((q->u - q->radius - 1.5) / D64_BLOCK), bx1 = floor((q->u + q->radius + 0.5) / D64_BLOCK);
        double by0 = floor((q->v - q->radius - 1.5) / D64_BLOCK), by1 = floor((q->v + q->radius + 0.5) / D64_BLOCK);
        bx0 = fmax(bx0, 0.0); by0 = fmax(by0, 0.0);
        bx1 = fmin(bx1, (double)(nbx - 1)); by1 = fmin(by1, (double)(nby - 1));
        int* r = rect + (size_t)k * 4;
        if (!(bx0 <= bx1 && by0 <= by1)) {
            r[0] = r[1] = r[2] = r[3] = 0;
            continue;
        }
        r[0] = (int)bx0; r[1] = (int)bx1 + 1; r[2] = (int)by0; r[3] = (int)by1 + 1;
        for (int by = r[2]; by < r[3]; by++)
            for (int bx = r[0]; bx < r[1]; bx++) cnt[by * nbx + bx]++;
    }
    sc->cand_start = (int64_t*)malloc(sizeof(int64_t) * ((size_t)blocks + 1));
    int64_t run = 0;
    sc->cand_max = 0;
    for (int b = 0; b < blocks; b++) {
        sc->cand_start[b] = run;
        run += cnt[b];
        if (cnt[b] > sc->cand_max) sc->cand_max = cnt[b];
        cnt[b] = 0;
    }
    sc->cand_start[blocks] = run;
    sc->cand = (int*)malloc(sizeof(int) * (size_t)(run > 0 ? run : 1));
    for (int k = 0; k < nv; k++) {
        const int* r = rect + (size_t)k * 4;
        for (int by = r[2]; by < r[3]; by++)
            for (int bx = r[0]; bx < r[1]; bx++) {
                const int b = by * nbx + bx;
                sc->cand[sc->cand_start[b] + cnt[b]++] = k;
            }
    }
    free(cnt);
    free(rect);
}

static void scene64_free(Scene64* sc) {
    free(sc->P);
    free(sc->order);
    free(sc->cand_start);
    free(sc->cand);
}

static inline double alpha64(const P64* s, double px, double py, double amax, double amin, double* dx, double* dy,
                             int* clamped) {
    *dx = px - s->u;
    *dy = py - s->v;
    if (fabs(*dx) > s->radius || fabs(*dy) > s->radius) return 0.0;
    const double power = -0.5 * (s->A * *dx * *dx + s->C * *dy * *dy) - s->B * *dx * *dy;
    if (power > 0) return 0.0;
    double a = s->opacity * exp(power);
    *clamped = 0;
    if (a > amax) {
        a = amax;
        *clamped = 1;
    }
    if (a < amin) return 0.0;
    return a;
}

/* FP64 render.  Every pixel walks the valid splats in (depth, index) order, skipping only
 * those whose bounding square cannot reach it (the candidate grid above; the result is
 * that of walking all of them).  signature: a hash of every discrete decision (validity, radius,
 * contributors, clamps, stop points) so finite differences can skip kinks. */
EXPORT void d64_render(const OrcCamera* cam, const double* params, int n, int degree, double near, double dil,
                       double amax, double amin, double tmin, double* image, uint64_t* signature) {
    Scene64 sc;
    scene64(&sc, cam, params, n, degree, near, dil);
    const int W = cam->width, H = cam->height;
    uint64_t h = 1469598103934665603ull;
    for (int i = 0; i < n; i++) h = fnv(h, (uint64_t)sc.P[i].ok * 1000003ull + (uint64_t)(sc.P[i].ok ? sc.P[i].radius : 0));
    uint64_t* rowh = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)H);
#pragma omp parallel for schedule(dynamic, 2)
    for (int y = 0; y < H; y++) {
        uint64_t hr = 1469598103934665603ull;
        for (int x = 0; x < W; x++) {
            const double px = x + 0.5, py = y + 0.5;
            double T = 1.0, rgb[3] = {0, 0, 0};
            const int blk = (y / D64_BLOCK) * sc.nbx + x / D64_BLOCK;
            int klast = -1;
            for (int64_t j = sc.cand_start[blk]; j < sc.cand_start[blk + 1]; j++) {
                if (T <= tmin) break;
                const int k = sc.cand[j];
                const P64* s = &sc.P[sc.order[k]];
                double dx, dy;
                int cl = 0;
                const double a = alpha64(s, px, py, amax, amin, &dx, &dy, &cl);
                if (a == 0.0) continue;
                hr = fnv(hr, (uint64_t)sc.order[k] * 2 + (uint64_t)cl);
                for (int c = 0; c < 3; c++) rgb[c] += s->rgb[c] * a * T;
                T *= 1.0 - a;
                klast = k;
            }
            /* stop point: the walk over all valid splats stops at the one after the
             * last contributor once T <= tmin */
            if (T <= tmin && klast + 1 < sc.nvalid) hr = fnv(hr, 0xfeedull + (uint64_t)(klast + 1));
            for (int c = 0; c < 3; c++) image[((size_t)y * W + x) * 3 + c] = rgb[c];
        }
        rowh[y] = hr;
    }
    for (int y = 0; y < H; y++) h = fnv(h, rowh[y]);
    if (signature) *signature = h;
    free(rowh);
    scene64_free(&sc);
}

/* FP64 adjoint of d64_render for dLoss/dImage `dl`: parameter gradients in the host
 * record layout (grads), and optionally the screen-space gradients in the reference's
 * 16-float layout (screen16: 0-2 colour, 3 opacity logit, 4-8 u, v, A, B, C). */
EXPORT void d64_grad(const OrcCamera* cam, const double* params, int n, int degree, double near, double dil, double amax,
                     double amin, double tmin, const double* dl, double* grads, double* screen16) {
    Scene64 sc;
    scene64(&sc, cam, params, n, degree, near, dil);
    const int W = cam->width, H = cam->height, S = orc_stride(degree), nk = nk_of(degree);
    double* sg = (double*)calloc((size_t)(n > 0 ? n : 1) * 9, sizeof(double));
    const size_t cap = (size_t)(sc.cand_max > 0 ? sc.cand_max : 1);
#pragma omp parallel
    {
    int* contrib = (int*)malloc(sizeof(int) * cap);
    double* alph = (double*)malloc(sizeof(double) * cap);
    double* Ts = (double*)malloc(sizeof(double) * cap);
    double* dxs = (double*)malloc(sizeof(double) * cap * 2);
    int* cls = (int*)malloc(sizeof(int) * cap);
#pragma omp for schedule(dynamic, 2)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const double px = x + 0.5, py = y + 0.5;
            const double* g = dl + ((size_t)y * W + x) * 3;
            const int blk = (y / D64_BLOCK) * sc.nbx + x / D64_BLOCK;
            /* Forward with the transmittance before every contributor kept. */
            double T = 1.0;
            int m = 0;
            for (int64_t j = sc.cand_start[blk]; j < sc.cand_start[blk + 1]; j++) {
                if (T <= tmin) break;
                const int k = sc.cand[j];
                const P64* s = &sc.P[sc.order[k]];
                double dx, dy;
                int cl = 0;
                const double a = alpha64(s, px, py, amax, amin, &dx, &dy, &cl);
                if (a == 0.0) continue;
                contrib[m] = sc.order[k];
                alph[m] = a;
                Ts[m] = T;
                dxs[2 * m] = dx;
                dxs[2 * m + 1] = dy;
                cls[m] = cl;
                m++;
                T *= 1.0 - a;
            }
            /* C = sum_k c_k a_k T_k:  dC/dc_k = a_k T_k,
             * dC/da_k = c_k T_k - (sum_{j>k} c_j a_j T_j) / (1 - a_k). */
            double behind[3] = {0, 0, 0};
            for (int q = m - 1; q >= 0; q--) {
                const int i = contrib[q];
                const P64* s = &sc.P[i];
                const double a = alph[q], Tk = Ts[q];
                double v9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                for (int c = 0; c < 3; c++) v9[c] = g[c] * a * Tk;
                double dA = 0;
                for (int c = 0; c < 3; c++) dA += g[c] * (s->rgb[c] * Tk - behind[c] / (1.0 - a));
                for (int c = 0; c < 3; c++) behind[c] += s->rgb[c] * a * Tk;
                if (!cls[q]) {
                    /* a = op exp(power) */
                    const double dP = dA * a;
                    v9[3] = dA * a * (1.0 - s->opacity);
                    const double dx = dxs[2 * q], dy = dxs[2 * q + 1];
                    /* power = -0.5 (A dx^2 + C dy^2) - B dx dy, dx = px - u */
                    v9[4] = dP * (s->A * dx + s->B * dy);
                    v9[5] = dP * (s->C * dy + s->B * dx);
                    v9[6] = dP * (-0.5 * dx * dx);
                    v9[7] = dP * (-dx * dy);
                    v9[8] = dP * (-0.5 * dy * dy);
                }
                double* o = sg + (size_t)i * 9;
                for (int c = 0; c < 9; c++)
                    if (v9[c] != 0.0) {
#pragma omp atomic
                        o[c] += v9[c];
                    }
            }
        }
    free(contrib); free(alph); free(Ts); free(dxs); free(cls);
    }
    double Wm[3][3], tv[3], cpos[3];
    cam64(cam, Wm, tv, cpos);
    for (int i = 0; i < n; i++) {
        double* out = grads + (size_t)i * S;
        for (int k = 0; k < S; k++) out[k] = 0.0;
        const double* o = sg + (size_t)i * 9;
        if (screen16) {
            double* s16 = screen16 + (size_t)i * 16;
            for (int k = 0; k < 16; k++) s16[k] = k < 9 ? o[k] : 0.0;
        }
        const P64* s = &sc.P[i];
        if (!s->ok) continue;
        const double* gp = params + (size_t)i * S;
        /* colour: rgb = dc + sum_k Y_k c_k */
        out[10] = o[3];
        for (int c = 0; c < 3; c++) {
            out[11 + c] = o[c];
            for (int k = 0; k < nk; k++) out[14 + c * nk + k] = s->Y[k] * o[c];
        }
        double gmean[3] = {0, 0, 0};
        if (degree > 0) {
            double Yd[15], dY[45];
            sh64(degree, s->dir, Yd, dY);
            double gd[3] = {0, 0, 0};
            for (int c = 0; c < 3; c++)
                for (int k = 0; k < nk; k++)
                    for (int j = 0; j < 3; j++) gd[j] += o[c] * gp[14 + c * nk + k] * dY[k * 3 + j];
            const double dot = gd[0] * s->dir[0] + gd[1] * s->dir[1] + gd[2] * s->dir[2];
            for (int j = 0; j < 3; j++) gmean[j] += (gd[j] - s->dir[j] * dot) / s->dnorm;
        }
        /* conic (A, B, C) = (c, -b, a) / det -> (a, b, c) */
        const double a = s->a, b = s->b, c = s->c, det = a * c - b * b, d2 = det * det;
        const double gA = o[6], gB = o[7], gC = o[8];
        const double ga = gA * (-c * c / d2) + gB * (b * c / d2) + gC * (1.0 / det - a * c / d2);
        const double gb = gA * (2 * b * c / d2) + gB * (-1.0 / det - 2 * b * b / d2) + gC * (2 * a * b / d2);
        const double gc = gA * (1.0 / det - a * c / d2) + gB * (a * b / d2) + gC * (-a * a / d2);
        /* cov = J Cc J^T (+ dil):  dL/dCc = J^T G J with G = [[ga, gb/2], [gb/2, gc]];
         * dL/dJ = 2 G J Cc. */
        const double z = s->p[2], x = s->p[0], yy = s->p[1];
        const double fx = cam->fx, fy = cam->fy;
        const double J[2][3] = {{fx / z, 0, -fx * x / (z * z)}, {0, fy / z, -fy * yy / (z * z)}};
        const double G[2][2] = {{ga, gb / 2}, {gb / 2, gc}};
        double R[3][3], qn[4], ql;
        rot64(gp + 6, R, qn, &ql);
        const double sc3[3] = {exp(gp[3]), exp(gp[4]), exp(gp[5])};
        double Sig[3][3], Cc[3][3];
        for (int r = 0; r < 3; r++)
            for (int q = 0; q < 3; q++) {
                double acc = 0;
                for (int k = 0; k < 3; k++) acc += R[r][k] * sc3[k] * sc3[k] * R[q][k];
                Sig[r][q] = acc;
            }
        for (int r = 0; r < 3; r++)
            for (int q = 0; q < 3; q++) {
                double acc = 0;
                for (int k = 0; k < 3; k++)
                    for (int l = 0; l < 3; l++) acc += Wm[r][k] * Sig[k][l] * Wm[q][l];
                Cc[r][q] = acc;
            }
        double GCc[3][3], GJ[2][3];
        for (int r = 0; r < 3; r++)
            for (int q = 0; q < 3; q++) {
                double acc = 0;
                for (int aa = 0; aa < 2; aa++)
                    for (int bb = 0; bb < 2; bb++) acc += J[aa][r] * G[aa][bb] * J[bb][q];
                GCc[r][q] = acc;
            }
        for (int aa = 0; aa < 2; aa++)
            for (int q = 0; q < 3; q++) {
                double acc = 0;
                for (int bb = 0; bb < 2; bb++)
                    for (int k = 0; k < 3; k++) acc += 2 * G[aa][bb] * J[bb][k] * Cc[k][q];
                GJ[aa][q] = acc;
            }
        /* J(p) and u, v (p) -> dL/dp */
        double gpv[3] = {0, 0, 0};
        gpv[0] += o[4] * fx / z;
        gpv[2] += -o[4] * fx * x / (z * z);
        gpv[1] += o[5] * fy / z;
        gpv[2] += -o[5] * fy * yy / (z * z);
        gpv[2] += GJ[0][0] * (-fx / (z * z));
        gpv[0] += GJ[0][2] * (-fx / (z * z));
        gpv[2] += GJ[0][2] * (2 * fx * x / (z * z * z));
        gpv[2] += GJ[1][1] * (-fy / (z * z));
        gpv[1] += GJ[1][2] * (-fy / (z * z));
        gpv[2] += GJ[1][2] * (2 * fy * yy / (z * z * z));
        for (int j = 0; j < 3; j++) gmean[j] += Wm[0][j] * gpv[0] + Wm[1][j] * gpv[1] + Wm[2][j] * gpv[2];
        out[0] = gmean[0]; out[1] = gmean[1]; out[2] = gmean[2];
        /* Cc = W Sig W^T -> dL/dSig = W^T GCc W;  Sig = R diag(s^2) R^T. */
        double GS[3][3];
        for (int r = 0; r < 3; r++)
            for (int q = 0; q < 3; q++) {
                double acc = 0;
                for (int k = 0; k < 3; k++)
                    for (int l = 0; l < 3; l++) acc += Wm[k][r] * GCc[k][l] * Wm[l][q];
                GS[r][q] = acc;
            }
        /* dL/ds_k = sum_{r,q} GS[r][q] * d(Sig_rq)/ds_k = 2 s_k sum_{r,q} GS[r][q] R[r][k] R[q][k] */
        for (int k = 0; k < 3; k++) {
            double acc = 0;
            for (int r = 0; r < 3; r++)
                for (int q = 0; q < 3; q++) acc += GS[r][q] * R[r][k] * R[q][k];
            out[3 + k] = 2 * sc3[k] * acc * sc3[k];  /* times ds/dlogscale = s */
        }
        /* dL/dR[r][k] = sum_q (GS[r][q] + GS[q][r]) s_k^2 R[q][k] */
        double GR[3][3];
        for (int r = 0; r < 3; r++)
            for (int k = 0; k < 3; k++) {
                double acc = 0;
                for (int q = 0; q < 3; q++) acc += (GS[r][q] + GS[q][r]) * sc3[k] * sc3[k] * R[q][k];
                GR[r][k] = acc;
            }
        /* R(w, x, y, z) of the unit quaternion; then through the normalisation. */
        const double w = qn[0], qx = qn[1], qy = qn[2], qz = qn[3];
        double gq[4];
        gq[0] = 2 * (-qz * GR[0][1] + qy * GR[0][2] + qz * GR[1][0] - qx * GR[1][2] - qy * GR[2][0] + qx * GR[2][1]);
        gq[1] = 2 * (qy * GR[0][1] + qz * GR[0][2] + qy * GR[1][0] - 2 * qx * GR[1][1] - w * GR[1][2] + qz * GR[2][0] +
                     w * GR[2][1] - 2 * qx * GR[2][2]);
        gq[2] = 2 * (-2 * qy * GR[0][0] + qx * GR[0][1] + w * GR[0][2] + qx * GR[1][0] + qz * GR[1][2] - w * GR[2][0] +
                     qz * GR[2][1] - 2 * qy * GR[2][2]);
        gq[3] = 2 * (-2 * qz * GR[0][0] - w * GR[0][1] + qx * GR[0][2] + w * GR[1][0] - 2 * qz * GR[1][1] +
                     qy * GR[1][2] + qx * GR[2][0] + qy * GR[2][1]);
        const double dq = gq[0] * qn[0] + gq[1] * qn[1] + gq[2] * qn[2] + gq[3] * qn[3];
        for (int k = 0; k < 4; k++) out[6 + k] = (gq[k] - qn[k] * dq) / ql;
    }
    free(sg);
    scene64_free(&sc);
}

/* ---------------------------------------------------------------------------------
 * densify() (trainer/gpu.js:575-599), sequential as written there: in index order drop
 * transparent (sigmoid(logit) < min_opacity) and oversized (largest exp(logScale) >
 * max_size) Gaussians, keep those whose average gradient norm is below the threshold
 * or when no room is left, otherwise spend one unit of room on a clone (largest scale
 * <= size_threshold) or a split (two copies moved by (u - 0.5) exp(logScale), log-scales
 * minus ln 1.6).  JavaScript numbers are doubles; the records are float.  The
 * reference's Math.random() is replaced by the same counter-based SplitMix64 draw as the
 * library's (seed, index, copy, axis).  params/out: host records of `stride` floats;
 * sums/counts: the statistics.  Returns the new count (out must hold 2 n records).
 * --------------------------------------------------------------------------------- */
static uint64_t orc_splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double orc_uniform(uint64_t seed, uint64_t i, int k, int j) {
    const uint64_t z = orc_splitmix64(orc_splitmix64(seed) ^ ((i * 8ull + (uint64_t)(k * 4 + j)) * 0xD1B54A32D192ED03ull));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

static double js_max3(double a, double b, double c) {
    if (isnan(a) || isnan(b) || isnan(c)) return NAN;
    double m = a > b ? a : b;
    return m > c ? m : c;
}

int orc_densify(const float* params, int n, int stride, const float* sums, const float* counts, double grad_threshold,
                double size_threshold, double min_opacity, double max_size, int max_count, uint64_t seed, float* out) {
    const double log_split = log(1.6);
    long long room = (long long)max_count - n;
    int o = 0;
    for (int i = 0; i < n; i++) {
        const float* g = params + (size_t)i * stride;
        const double op = 1.0 / (1.0 + exp(-(double)g[10]));
        if (op < min_opacity) continue;
        const double size = js_max3(exp((double)g[3]), exp((double)g[4]), exp((double)g[5]));
        if (size > max_size) continue;
        const double avg = (counts[i] != 0.f && !isnan(counts[i])) ? (double)sums[i] / (double)counts[i] : 0.0;
        if (avg < grad_threshold || room <= 0) {
            memcpy(out + (size_t)o++ * stride, g, sizeof(float) * stride);
            continue;
        }
        room--;
        if (size <= size_threshold) {
            memcpy(out + (size_t)o++ * stride, g, sizeof(float) * stride);
            memcpy(out + (size_t)o++ * stride, g, sizeof(float) * stride);
        } else {
            for (int k = 0; k < 2; k++) {
                float* c = out + (size_t)o++ * stride;
                memcpy(c, g, sizeof(float) * stride);
                for (int j = 0; j < 3; j++) {
                    c[j] = (float)((double)g[j] + (orc_uniform(seed, (uint64_t)i, k, j) - 0.5) * exp((double)g[3 + j]));
                    c[3 + j] = (float)((double)g[3 + j] - log_split);
                }
            }
        }
    }
    return o;
}

/* ---------------------------------------------------------------------------------
 * neighbourSizes (trainer/neighbours.js:13-53): cubes of 0.1 m keyed as the reference
 * keys its Map; per point the three smallest squared distances (double) to other points
 * of the 27 surrounding cubes, their root mean, clamped; `fallback` with none.  Cubes are
 * found here by sorting (key, point) pairs and binary search (the result does not depend
 * on the order inside a cube).
 * --------------------------------------------------------------------------------- */
typedef struct {
    long long key;
    int idx;
} OrcCellPt;

static int cmp_cellpt(const void* a, const void* b) {
    const long long ka = ((const OrcCellPt*)a)->key, kb = ((const OrcCellPt*)b)->key;
    if (ka != kb) return ka < kb ? -1 : 1;
    return ((const OrcCellPt*)a)->idx - ((const OrcCellPt*)b)->idx;
}

static long long orc_cell(float v) { return (long long)floor((double)v / 0.1); }
static long long orc_key(long long i, long long j, long long k) {
    return ((i + 32768) * 65536 + (j + 32768)) * 65536 + (k + 32768);
}

void orc_neighbour_sizes(const float* xyz, int count, double mn, double mx, double fallback, float* sizes) {
    OrcCellPt* pts = (OrcCellPt*)malloc(sizeof(OrcCellPt) * (size_t)(count > 0 ? count : 1));
    for (int p = 0; p < count; p++) {
        pts[p].key = orc_key(orc_cell(xyz[p * 3]), orc_cell(xyz[p * 3 + 1]), orc_cell(xyz[p * 3 + 2]));
        pts[p].idx = p;
    }
    qsort(pts, (size_t)count, sizeof(OrcCellPt), cmp_cellpt);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int p = 0; p < count; p++) {
        double best[3] = {INFINITY, INFINITY, INFINITY};
        const long long ci = orc_cell(xyz[p * 3]), cj = orc_cell(xyz[p * 3 + 1]), ck = orc_cell(xyz[p * 3 + 2]);
        const double x = xyz[p * 3], y = xyz[p * 3 + 1], z = xyz[p * 3 + 2];
        for (int di = -1; di <= 1; di++)
            for (int dj = -1; dj <= 1; dj++)
                for (int dk = -1; dk <= 1; dk++) {
                    const long long key = orc_key(ci + di, cj + dj, ck + dk);
                    int lo = 0, hi = count;  /* first entry with key >= wanted */
                    while (lo < hi) {
                        const int mid = (lo + hi) / 2;
                        if (pts[mid].key < key) lo = mid + 1;
                        else hi = mid;
                    }
                    for (int t = lo; t < count && pts[t].key == key; t++) {
                        const int q = pts[t].idx;
                        if (q == p) continue;
                        const double dx = (double)xyz[q * 3] - x, dy = (double)xyz[q * 3 + 1] - y,
                                     dz = (double)xyz[q * 3 + 2] - z;
                        const double d2 = dx * dx + dy * dy + dz * dz;
                        if (d2 >= best[2]) continue;
                        if (d2 < best[0]) {
                            best[2] = best[1];
                            best[1] = best[0];
                            best[0] = d2;
                        } else if (d2 < best[1]) {
                            best[2] = best[1];
                            best[1] = d2;
                        } else {
                            best[2] = d2;
                        }
                    }
                }
        int found = 0;
        double sum = 0.0;
        for (int k = 0; k < 3; k++)
            if (isfinite(best[k])) {
                sum += best[k];
                found++;
            }
        const double size = found ? sqrt(sum / found) : fallback;
        sizes[p] = (float)fmin(mx, fmax(mn, size));
    }
    free(pts);
}
