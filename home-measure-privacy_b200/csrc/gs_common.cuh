// Shared device definitions of the Gaussian-splat training step (sm_100a).
//
// Layouts in HBM (n_pad = n rounded up to a multiple of 128):
//   parameters, gradients, Adam moments: plane-major float planes [P][n_pad], plane order
//     0-2 mean xyz, 3-5 log-scale, 6-9 rotation wxyz, 10 opacity logit, 11-13 colour
//     (SH DC, the reference's raw RGB), 14.. SH bands >= 1 channel-major (R, G, B; 1..K-1).
//   (view, Gaussian) pairs, pair = view_slot * n_pad + i:
//     geo0 float4 (u, v, conicA, conicB), geo1 float4 (conicC, opacity, radius, depth),
//     rgb float4 (r, g, b, 0), rect uint2 (x0 | x1 << 16, y0 | y1 << 16) tile rectangle
//     (half-open), depth key u32, screen gradients sg8 float[8] + sg1 float.
//   key instances (one per (pair, covered tile)): tile id u32 + pair u32.
//   per pixel (all views concatenated): image float[3] HWC, final T, last (u32), dL[3].
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include <math.h>

#define GS_TILE 16                    // default tile edge (the reference's); contexts may use 8 or 32
#define GS_MAX_VIEWS 64
#define GS_MAX_PLANES 59
#define GS_KEY_SENTINEL 0x7FFFFFFFu   // above +inf's bits: culled pairs sort last

namespace gs {

// Per-view descriptor on the device.
struct ViewDesc {
    float R[9];          // world-to-camera rotation, row-major
    float t[3];
    float fx, fy, cx, cy;
    float campos[3];     // camera centre in world space, -R^T t
    int width, height;
    int tiles_x, tiles_y;
    int tile_offset;     // first global tile id of this view
    int pixel_offset;    // first pixel of this view in the per-pixel buffers
    int loss_blocks_x, loss_blocks_y, loss_block_offset;
    int tile;            // tile edge in pixels (8, 16, 32 or 64; the same for every view)
};

// Step status kept on the device; mirrored to pinned host memory.  The first 24 bytes
// are per-forward counters, zeroed when a forward starts.
struct DevStatus {
    unsigned long long instances_needed;  // key instances the last forward wanted
    unsigned int overflow;                // 1 when they exceeded the capacity
    unsigned int visible_pairs;           // unused counter slot
    unsigned int work_counter;            // persistent raster queue head (forward)
    unsigned int work_counter_bwd;        // persistent raster queue head (backward)
    int step_t;                           // Adam updates applied
    int skipped;                          // the last step skipped its update
    float loss;                           // mean loss of the last step over its views
    int nonfinite;                        // last loss was not finite
    unsigned int sort_timeout;            // a radix look-back wait gave up (never expected)
    unsigned int debug_wait;              // test hook: polls of an extra wait in each sort pass (0 = off)
    unsigned int never_set;               // the word that extra wait polls: no code writes it
    unsigned int pad[3];
};
#define GS_STATUS_FORWARD_BYTES 24

// Offset and length of one sort segment (instances of a view, or of all views).
struct SegInfo {
    unsigned int base;
    unsigned int count;
};

__host__ __device__ __forceinline__ float __int_as_float_hd(int b) {
#ifdef __CUDA_ARCH__
    return __int_as_float(b);
#else
    float f;
    memcpy(&f, &b, sizeof f);
    return f;
#endif
}

// ---------------------------------------------------------------------------------
// Arithmetic with explicit rounding.  The projection's geometry (camera-space point,
// covariances, conic, radius, screen position) is computed with one IEEE-rounded
// operation per step and no fused multiply-add, in the order the reference's WGSL
// writes it (trainer/gpu.js:30-60).  A CPU restatement with the same order then
// reproduces the tile keys bit for bit.
// ---------------------------------------------------------------------------------
__host__ __device__ __forceinline__ float xmul(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
__host__ __device__ __forceinline__ float xadd(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
__host__ __device__ __forceinline__ float xsub(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
__host__ __device__ __forceinline__ float xdiv(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}
__host__ __device__ __forceinline__ float xsqrt(float a) {
#ifdef __CUDA_ARCH__
    return __fsqrt_rn(a);
#else
    return sqrtf(a);
#endif
}

// exp(x) in single precision, specified here so that host and device agree exactly:
// Cody-Waite reduction x = k ln2 + r (ln2 split into a 16-bit head and a tail), the
// degree-7 Taylor polynomial of e^r on |r| <= ln2/2 in Horner form (truncation error
// below 2e-9 relative), then scaling by 2^k through the exponent bits.  Each step is
// one rounded operation.  Results are within a few ulp of the true value.
__host__ __device__ __forceinline__ float spec_expf(float x) {
    if (!(x > -87.0f)) return (x != x) ? x : 0.0f;   // NaN stays NaN
    if (x > 88.0f) return __int_as_float_hd(0x7f800000);
    const float k = rintf(xmul(x, 1.44269502162933349609375f));
    const float r = xsub(xsub(x, xmul(k, 0.693145751953125f)), xmul(k, 1.428606765330187045e-06f));
    float p = 1.98412698412698412698e-04f;           // 1/5040
    p = xadd(xmul(p, r), 1.38888888888888888889e-03f);  // 1/720
    p = xadd(xmul(p, r), 8.33333333333333333333e-03f);  // 1/120
    p = xadd(xmul(p, r), 4.16666666666666666667e-02f);  // 1/24
    p = xadd(xmul(p, r), 1.66666666666666666667e-01f);  // 1/6
    p = xadd(xmul(p, r), 0.5f);
    p = xadd(xmul(p, r), 1.0f);
    p = xadd(xmul(p, r), 1.0f);
    const int ki = (int)k;
    return xmul(p, __int_as_float_hd((ki + 127) << 23));
}

// Camera-space point, EWA 2D covariance, conic, radius and screen position of one
// Gaussian in one view: projectShape (trainer/gpu.js:30-60), same operation order.
struct Projected {
    bool ok;
    float u, v, a, b, c, radius, depth;
};

// quatToMat (trainer/gpu.js:20-27): normalised w,x,y,z -> rotation, row-major.
__host__ __device__ __forceinline__ void quat_to_rot_exact(const float q[4], float Rq[9]) {
    const float len = xsqrt(xadd(xadd(xadd(xmul(q[0], q[0]), xmul(q[1], q[1])), xmul(q[2], q[2])),
                                 xmul(q[3], q[3])));
    const float d = fmaxf(len, 1e-12f);
    const float w = xdiv(q[0], d), x = xdiv(q[1], d), y = xdiv(q[2], d), z = xdiv(q[3], d);
    // Row i, column j.
    Rq[0] = xsub(1.0f, xmul(2.0f, xadd(xmul(y, y), xmul(z, z))));
    Rq[3] = xmul(2.0f, xadd(xmul(x, y), xmul(w, z)));
    Rq[6] = xmul(2.0f, xsub(xmul(x, z), xmul(w, y)));
    Rq[1] = xmul(2.0f, xsub(xmul(x, y), xmul(w, z)));
    Rq[4] = xsub(1.0f, xmul(2.0f, xadd(xmul(x, x), xmul(z, z))));
    Rq[7] = xmul(2.0f, xadd(xmul(y, z), xmul(w, x)));
    Rq[2] = xmul(2.0f, xadd(xmul(x, z), xmul(w, y)));
    Rq[5] = xmul(2.0f, xsub(xmul(y, z), xmul(w, x)));
    Rq[8] = xsub(1.0f, xmul(2.0f, xadd(xmul(x, x), xmul(y, y))));
}

// World covariance Sigma = (R S)(R S)^T, row-major 3x3 (symmetric by construction).
__host__ __device__ __forceinline__ void world_cov_exact(const float logscale[3], const float q[4],
                                                         float Sig[9]) {
    float Rq[9];
    quat_to_rot_exact(q, Rq);
    const float s0 = spec_expf(logscale[0]), s1 = spec_expf(logscale[1]), s2 = spec_expf(logscale[2]);
    float M[9];
    for (int i = 0; i < 3; i++) {
        M[i * 3 + 0] = xmul(Rq[i * 3 + 0], s0);
        M[i * 3 + 1] = xmul(Rq[i * 3 + 1], s1);
        M[i * 3 + 2] = xmul(Rq[i * 3 + 2], s2);
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            Sig[i * 3 + j] = xadd(xadd(xmul(M[i * 3 + 0], M[j * 3 + 0]), xmul(M[i * 3 + 1], M[j * 3 + 1])),
                                  xmul(M[i * 3 + 2], M[j * 3 + 2]));
}

__host__ __device__ __forceinline__ Projected project_exact(const ViewDesc& vw, const float mean[3],
                                                            const float Sig[9], float near_plane,
                                                            float dilation) {
    Projected o;
    o.ok = false;
    const float* W = vw.R;
    const float px = xadd(xadd(xadd(xmul(W[0], mean[0]), xmul(W[1], mean[1])), xmul(W[2], mean[2])), vw.t[0]);
    const float py = xadd(xadd(xadd(xmul(W[3], mean[0]), xmul(W[4], mean[1])), xmul(W[5], mean[2])), vw.t[1]);
    const float pz = xadd(xadd(xadd(xmul(W[6], mean[0]), xmul(W[7], mean[1])), xmul(W[8], mean[2])), vw.t[2]);
    o.depth = pz;
    if (pz < near_plane) return o;
    // A = W * Sigma, then C = A * W^T.
    float A[9], C[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            A[i * 3 + j] = xadd(xadd(xmul(W[i * 3 + 0], Sig[0 * 3 + j]), xmul(W[i * 3 + 1], Sig[1 * 3 + j])),
                                xmul(W[i * 3 + 2], Sig[2 * 3 + j]));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            C[i * 3 + j] = xadd(xadd(xmul(A[i * 3 + 0], W[j * 3 + 0]), xmul(A[i * 3 + 1], W[j * 3 + 1])),
                                xmul(A[i * 3 + 2], W[j * 3 + 2]));
    const float zz = xmul(pz, pz);
    const float j00 = xdiv(vw.fx, pz), j02 = xdiv(xmul(-vw.fx, px), zz);
    const float j11 = xdiv(vw.fy, pz), j12 = xdiv(xmul(-vw.fy, py), zz);
    // C * j0 and C * j1 (the zero entries of j0, j1 contribute exact zeros).
    const float cj0_0 = xadd(xmul(C[0], j00), xmul(C[2], j02));
    const float cj0_2 = xadd(xmul(C[6], j00), xmul(C[8], j02));
    const float cj1_0 = xadd(xmul(C[1], j11), xmul(C[2], j12));
    const float cj1_1 = xadd(xmul(C[4], j11), xmul(C[5], j12));
    const float cj1_2 = xadd(xmul(C[7], j11), xmul(C[8], j12));
    const float a = xadd(xadd(xmul(j00, cj0_0), xmul(j02, cj0_2)), dilation);
    const float b = xadd(xmul(j00, cj1_0), xmul(j02, cj1_2));
    const float c = xadd(xadd(xmul(j11, cj1_1), xmul(j12, cj1_2)), dilation);
    const float det = xsub(xmul(a, c), xmul(b, b));
    if (!(det > 0.0f)) return o;
    const float mid = xmul(xadd(a, c), 0.5f);
    o.ok = true;
    o.u = xadd(xmul(vw.fx, xdiv(px, pz)), vw.cx);
    o.v = xadd(xmul(vw.fy, xdiv(py, pz)), vw.cy);
    o.a = xdiv(c, det);
    o.b = xdiv(-b, det);
    o.c = xdiv(a, det);
    o.radius = ceilf(xmul(3.0f, xsqrt(xadd(mid, xsqrt(fmaxf(0.1f, xsub(xmul(mid, mid), det)))))));
    return o;
}

// Tile rectangle [x0, x1) x [y0, y1) of a splat for tiles of `tile` pixels.  mode 0:
// the reference's GPU BIN (trainer/gpu.js:632-635, f32, clamps so off-screen-right/bottom
// splats still land in the last tile column/row; its 1/16 is 1/tile here, exact for the
// powers of two allowed); mode 1: tileLists (trainer/gpu.js:456-461, f64 like JS,
// inclusive bounds made half-open).
__host__ __device__ __forceinline__ void tile_rect(float u, float v, float r, int tiles_x, int tiles_y,
                                                  int mode, int tile, int& x0, int& x1, int& y0, int& y1) {
    if (mode == 0) {
        const float tx = (float)(tiles_x - 1), ty = (float)(tiles_y - 1);
        const float it = 1.0f / (float)tile;
        const float fx0 = fminf(fmaxf(floorf(xmul(xsub(xsub(u, r), 0.5f), it)), 0.0f), tx);
        const float fx1 = fminf(fmaxf(floorf(xmul(xsub(xadd(u, r), 0.5f), it)), -1.0f), tx);
        const float fy0 = fminf(fmaxf(floorf(xmul(xsub(xsub(v, r), 0.5f), it)), 0.0f), ty);
        const float fy1 = fminf(fmaxf(floorf(xmul(xsub(xadd(v, r), 0.5f), it)), -1.0f), ty);
        x0 = (int)fx0; x1 = (int)xadd(fx1, 1.0f);
        y0 = (int)fy0; y1 = (int)xadd(fy1, 1.0f);
    } else {
        const double du = (double)u, dv = (double)v, dr = (double)r, dt = (double)tile;
        const double fx0 = floor((du - dr - 0.5) / dt), fx1 = floor((du + dr - 0.5) / dt);
        const double fy0 = floor((dv - dr - 0.5) / dt), fy1 = floor((dv + dr - 0.5) / dt);
        x0 = (int)fmax(0.0, fx0); x1 = (int)fmin((double)(tiles_x - 1), fx1) + 1;
        y0 = (int)fmax(0.0, fy0); y1 = (int)fmin((double)(tiles_y - 1), fy1) + 1;
    }
    if (x1 < x0) x1 = x0;
    if (y1 < y0) y1 = y0;
}

// Smallest value of the conic's quadratic form A dx^2 + 2 B dx dy + C dy^2 over the box
// [xl, xh] x [yl, yh] (offsets from the splat centre).  Convex, so: 0 when the centre is
// inside, else the least of the four edges' clamped 1-D minima.
__host__ __device__ __forceinline__ float conic_qmin_box(float A, float B, float C, float xl, float xh, float yl,
                                                         float yh) {
    if (xl <= 0.f && xh >= 0.f && yl <= 0.f && yh >= 0.f) return 0.f;
    const float iA = 1.0f / A, iC = 1.0f / C;
    float best, x, y, q;
    x = xl; y = fminf(fmaxf(-B * x * iC, yl), yh); best = A * x * x + 2.f * B * x * y + C * y * y;
    x = xh; y = fminf(fmaxf(-B * x * iC, yl), yh); q = A * x * x + 2.f * B * x * y + C * y * y; best = fminf(best, q);
    y = yl; x = fminf(fmaxf(-B * y * iA, xl), xh); q = A * x * x + 2.f * B * x * y + C * y * y; best = fminf(best, q);
    y = yh; x = fminf(fmaxf(-B * y * iA, xl), xh); q = A * x * x + 2.f * B * x * y + C * y * y; best = fminf(best, q);
    return best;
}

// Can a splat (centre u, v; conic A, B, C; radius r; culling bound thr = 2 ln(op /
// alpha_min) + slack) give any pixel centre in [px0, px1] x [py0, py1] alpha >=
// alpha_min?  Conservative: a pixel passes only inside the square |dx|, |dy| <= r and
// where the quadratic form is below thr.
__host__ __device__ __forceinline__ bool splat_reaches_box(float u, float v, float A, float B, float C, float r,
                                                           float thr, float px0, float px1, float py0, float py1) {
    const float xl = fmaxf(px0, u - r), xh = fminf(px1, u + r);
    const float yl = fmaxf(py0, v - r), yh = fminf(py1, v + r);
    if (xl > xh || yl > yh) return false;
    return conic_qmin_box(A, B, C, xl - u, xh - u, yl - v, yh - v) <= thr;
}

#define GS_SPAN_ROWS 12           // pairs up to this many tile rows get per-row tile spans
#define GS_PCOUNT_RECT 0x80000000u  // pcount flag: instances are the whole rectangle

// ---------------------------------------------------------------------------------
// Real spherical harmonics up to degree 3 (Condon-Shortley phase).  Coefficient k of a
// band l >= 1 uses index k = l^2 + l + m; constants are K_l^m = sqrt((2l+1)/(4 pi) *
// (l-|m|)!/(l+|m|)!), times sqrt(2) for m != 0, times the associated Legendre factor.
// The DC term is the colour itself (rgb = dc + sum_{k>=1} Y_k(d) c_k).
// ---------------------------------------------------------------------------------
#define SH_C1 0.48860251190291992f
#define SH_C2_0 1.0925484305920792f
#define SH_C2_1 -1.0925484305920792f
#define SH_C2_2 0.31539156525252005f
#define SH_C2_3 -1.0925484305920792f
#define SH_C2_4 0.54627421529603959f
#define SH_C3_0 -0.59004358992664352f
#define SH_C3_1 2.8906114426405538f
#define SH_C3_2 -0.45704579946446572f
#define SH_C3_3 0.37317633259011540f
#define SH_C3_4 -0.45704579946446572f
#define SH_C3_5 1.4453057213202769f
#define SH_C3_6 -0.59004358992664352f

// Y[0..K-2] = basis values of coefficients 1..K-1 at unit direction (x, y, z).
__host__ __device__ __forceinline__ void sh_basis(int degree, float x, float y, float z, float* Y) {
    if (degree < 1) return;
    Y[0] = -SH_C1 * y;
    Y[1] = SH_C1 * z;
    Y[2] = -SH_C1 * x;
    if (degree < 2) return;
    const float xx = x * x, yy = y * y, zz = z * z;
    Y[3] = SH_C2_0 * x * y;
    Y[4] = SH_C2_1 * y * z;
    Y[5] = SH_C2_2 * (2.0f * zz - xx - yy);
    Y[6] = SH_C2_3 * x * z;
    Y[7] = SH_C2_4 * (xx - yy);
    if (degree < 3) return;
    Y[8] = SH_C3_0 * y * (3.0f * xx - yy);
    Y[9] = SH_C3_1 * x * y * z;
    Y[10] = SH_C3_2 * y * (4.0f * zz - xx - yy);
    Y[11] = SH_C3_3 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
    Y[12] = SH_C3_4 * x * (4.0f * zz - xx - yy);
    Y[13] = SH_C3_5 * z * (xx - yy);
    Y[14] = SH_C3_6 * x * (xx - 3.0f * yy);
}

// dL/d(direction) given w_k = dL/dY_k for k = 1..K-1 (w[0..K-2]).
__host__ __device__ __forceinline__ void sh_basis_grad(int degree, float x, float y, float z,
                                                       const float* w, float& gx, float& gy,
                                                       float& gz) {
    gx = gy = gz = 0.0f;
    if (degree < 1) return;
    gy += -SH_C1 * w[0];
    gz += SH_C1 * w[1];
    gx += -SH_C1 * w[2];
    if (degree < 2) return;
    const float xx = x * x, yy = y * y, zz = z * z;
    gx += SH_C2_0 * y * w[3];               gy += SH_C2_0 * x * w[3];
    gy += SH_C2_1 * z * w[4];               gz += SH_C2_1 * y * w[4];
    gx += -2.0f * SH_C2_2 * x * w[5];       gy += -2.0f * SH_C2_2 * y * w[5];   gz += 4.0f * SH_C2_2 * z * w[5];
    gx += SH_C2_3 * z * w[6];               gz += SH_C2_3 * x * w[6];
    gx += 2.0f * SH_C2_4 * x * w[7];        gy += -2.0f * SH_C2_4 * y * w[7];
    if (degree < 3) return;
    gx += SH_C3_0 * 6.0f * x * y * w[8];    gy += SH_C3_0 * (3.0f * xx - 3.0f * yy) * w[8];
    gx += SH_C3_1 * y * z * w[9];           gy += SH_C3_1 * x * z * w[9];        gz += SH_C3_1 * x * y * w[9];
    gx += SH_C3_2 * -2.0f * x * y * w[10];  gy += SH_C3_2 * (4.0f * zz - xx - 3.0f * yy) * w[10];
    gz += SH_C3_2 * 8.0f * y * z * w[10];
    gx += SH_C3_3 * -6.0f * x * z * w[11];  gy += SH_C3_3 * -6.0f * y * z * w[11];
    gz += SH_C3_3 * (6.0f * zz - 3.0f * xx - 3.0f * yy) * w[11];
    gx += SH_C3_4 * (4.0f * zz - 3.0f * xx - yy) * w[12];
    gy += SH_C3_4 * -2.0f * x * y * w[12];  gz += SH_C3_4 * 8.0f * x * z * w[12];
    gx += SH_C3_5 * 2.0f * x * z * w[13];   gy += SH_C3_5 * -2.0f * y * z * w[13];
    gz += SH_C3_5 * (xx - yy) * w[13];
    gx += SH_C3_6 * (3.0f * xx - 3.0f * yy) * w[14];
    gy += SH_C3_6 * -6.0f * x * y * w[14];
}

__host__ __device__ __forceinline__ int sh_coeffs(int degree) { return (degree + 1) * (degree + 1); }
__host__ __device__ __forceinline__ int num_planes(int degree) { return 14 + 3 * (sh_coeffs(degree) - 1); }

}  // namespace gs
