// Fused Adam over all parameter planes, the step's book-keeping kernels and the
// layout conversions used by the C ABI's read-backs.
//
// ADAM (trainer/gpu.js:411-443): m = b1 m + (1 - b1) g, v = b2 v + (1 - b2) g^2,
// p -= lr (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps), per-group learning rates,
// then colour clamped to [0, 1] and the rotation quaternion renormalised.  Here it runs
// over the plane-major SoA: each thread owns 4 consecutive Gaussians and moves float4s
// through every plane (parameters, gradient, both moments), so each warp streams
// 512-byte rows.  A step whose key instances overflowed their buffer (its tile lists
// are truncated) skips the update.  The moments are updated with every operation
// rounded on its own, in the reference's order (explicit round-to-nearest intrinsics, no
// contraction into FMA): where a first moment has nearly cancelled, a contracted product
// would move the update by many ulps of its own size.  The bias corrections are applied as
// products with their reciprocals (within an ulp of the reference's quotients, and the
// update inherits no cancellation from them).
#include "../../include/gsb200.h"
#include "internal.h"

namespace gs {

// One thread per (plane, 4 Gaussians) float4 of every plane except the rotation's, and
// one per 4 Gaussians for the four rotation planes together (updated, then
// renormalised): 14M independent float4 updates at the benchmark size, so the loads of
// many planes are in flight at once.
__device__ __forceinline__ void adam4(float4& p, const float4& g, float4& m, float4& v, float lr, float b1, float b2,
                                      float omb1, float omb2, float ibc1, float ibc2, float eps) {
    float* pp = &p.x;
    const float* gg = &g.x;
    float* mm = &m.x;
    float* vv = &v.x;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        mm[e] = __fadd_rn(__fmul_rn(b1, mm[e]), __fmul_rn(omb1, gg[e]));
        vv[e] = __fadd_rn(__fmul_rn(b2, vv[e]), __fmul_rn(__fmul_rn(omb2, gg[e]), gg[e]));
        pp[e] -= lr * (mm[e] * ibc1) / (sqrtf(vv[e] * ibc2) + eps);
    }
}

#ifndef ADAM_GROUPS
#define ADAM_GROUPS 2  // groups of 4 Gaussians per thread: 2 keeps twice the loads in flight
#endif

__global__ void __launch_bounds__(256) adam_kernel(AdamArgs a) {
    // Skip the update when this step's instances overflowed -- on every replica at once
    // when the gradients were reduced across replicas (the tail's overflow count).
    if (a.skip ? (*a.skip > 0.f) : (a.status->overflow != 0u || a.status->sort_timeout != 0u)) return;
    const int groups = a.n_pad / 4;
    const int units_per_group = a.planes - 3;  // planes other than 6..9, plus one rotation unit
    // A thread takes ADAM_GROUPS groups of 4 Gaussians of one unit, gper apart (so a
    // warp's loads stay contiguous), loading all of them before it stores any.
    const int gper = (groups + ADAM_GROUPS - 1) / ADAM_GROUPS;
    const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= (long long)gper * units_per_group) return;
    const int unit = (int)(u / gper), grp0 = (int)(u % gper);
    const int t = a.status->step_t + 1;
    const float ibc1 = 1.0f / (1.0f - powf(a.beta1, (float)t));
    const float ibc2 = 1.0f / (1.0f - powf(a.beta2, (float)t));
    const float omb1 = 1.0f - a.beta1, omb2 = 1.0f - a.beta2;
    const size_t np = (size_t)a.n_pad;
    if (unit != 6) {
        const int j = unit < 6 ? unit : unit + 3;  // skip planes 7..9 (unit 6 = rotation)
        float4 p[ADAM_GROUPS], g[ADAM_GROUPS], m[ADAM_GROUPS], v[ADAM_GROUPS];
        size_t off[ADAM_GROUPS];
        bool ok[ADAM_GROUPS];
#pragma unroll
        for (int r = 0; r < ADAM_GROUPS; r++) {
            const int grp = grp0 + r * gper;
            ok[r] = grp < groups;
            off[r] = (size_t)j * np + (size_t)grp * 4;
            if (ok[r]) {
                p[r] = *reinterpret_cast<const float4*>(a.params + off[r]);
                g[r] = *reinterpret_cast<const float4*>(a.grads + off[r]);
                m[r] = *reinterpret_cast<const float4*>(a.m + off[r]);
                v[r] = *reinterpret_cast<const float4*>(a.v + off[r]);
            }
        }
#pragma unroll
        for (int r = 0; r < ADAM_GROUPS; r++) {
            if (!ok[r]) continue;
            adam4(p[r], g[r], m[r], v[r], a.lr[j], a.beta1, a.beta2, omb1, omb2, ibc1, ibc2, a.eps);
            if (j >= 11 && j <= 13) {  // colour (SH DC) clamped to [0, 1]
                p[r].x = fminf(fmaxf(p[r].x, 0.f), 1.f);
                p[r].y = fminf(fmaxf(p[r].y, 0.f), 1.f);
                p[r].z = fminf(fmaxf(p[r].z, 0.f), 1.f);
                p[r].w = fminf(fmaxf(p[r].w, 0.f), 1.f);
            }
            *reinterpret_cast<float4*>(a.params + off[r]) = p[r];
            *reinterpret_cast<float4*>(a.m + off[r]) = m[r];
            *reinterpret_cast<float4*>(a.v + off[r]) = v[r];
        }
        return;
    }
    for (int r = 0; r < ADAM_GROUPS; r++) {
    const int grp = grp0 + r * gper;
    if (grp >= groups) break;
    const size_t col = (size_t)grp * 4;
    // Rotation planes 6..9: update, then renormalise the quaternions.
    float4 q[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const size_t off = (size_t)(6 + k) * np + col;
        q[k] = *reinterpret_cast<const float4*>(a.params + off);
        const float4 g = *reinterpret_cast<const float4*>(a.grads + off);
        float4 m = *reinterpret_cast<const float4*>(a.m + off);
        float4 v = *reinterpret_cast<const float4*>(a.v + off);
        adam4(q[k], g, m, v, a.lr[6 + k], a.beta1, a.beta2, omb1, omb2, ibc1, ibc2, a.eps);
        *reinterpret_cast<float4*>(a.m + off) = m;
        *reinterpret_cast<float4*>(a.v + off) = v;
    }
    float* qw = &q[0].x;
    float* qx = &q[1].x;
    float* qy = &q[2].x;
    float* qz = &q[3].x;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const float ss = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(qw[e], qw[e]), __fmul_rn(qx[e], qx[e])),
                                             __fmul_rn(qy[e], qy[e])),
                                   __fmul_rn(qz[e], qz[e]));
        const float nrm = fmaxf(__fsqrt_rn(ss), 1e-12f);
        qw[e] = __fdiv_rn(qw[e], nrm);
        qx[e] = __fdiv_rn(qx[e], nrm);
        qy[e] = __fdiv_rn(qy[e], nrm);
        qz[e] = __fdiv_rn(qz[e], nrm);
    }
#pragma unroll
    for (int k = 0; k < 4; k++) *reinterpret_cast<float4*>(a.params + (size_t)(6 + k) * np + col) = q[k];
    }
}

void launch_adam(const AdamArgs& a, cudaStream_t s) {
    const long long units = (long long)((a.n_pad / 4 + ADAM_GROUPS - 1) / ADAM_GROUPS) * (a.planes - 3);
    const int threads = 256;
    const long long blocks = (units + threads - 1) / threads;
    if (blocks > 0) adam_kernel<<<(unsigned)blocks, threads, 0, s>>>(a);
}

// Loss of a step from the per-view sums: mean over views of
// (1 - lambda) * L1 + lambda * (1 - mean SSIM).
__device__ float step_loss(const double* acc, const ViewDesc* views, int view_first, int num_views, float lambda,
                           int window) {
    const int R = window == 0 ? 3 : 5;
    double total = 0.0;
    for (int s = 0; s < num_views; s++) {
        const ViewDesc& vw = views[view_first + s];
        const double n = (double)vw.width * vw.height * 3.0;
        const int wx = vw.width - 2 * R, wy = vw.height - 2 * R;
        const double windows = (wx > 0 && wy > 0) ? (double)wx * wy * 3.0 : 0.0;
        const double l1 = acc[2 * (view_first + s)] / n;
        const double ssim = windows > 0.0 ? acc[2 * (view_first + s) + 1] / windows : 1.0;
        total += (1.0 - lambda) * l1 + (lambda > 0.f ? lambda * (1.0 - ssim) : 0.0);
    }
    return (float)(total / (num_views > 0 ? num_views : 1));
}

__global__ void step_end_kernel(DevStatus* st, const double* acc, const ViewDesc* views, int view_first,
                                int num_views, float lambda, int window, int advance) {
    const float loss = step_loss(acc, views, view_first, num_views, lambda, window);
    st->loss = loss;
    st->nonfinite = isfinite(loss) ? 0 : 1;
    const bool skip = st->overflow || st->sort_timeout;  // truncated lists or unsure sort offsets
    st->skipped = skip ? 1 : 0;
    if (advance && !skip) st->step_t += 1;
}

void launch_step_end(DevStatus* status, const double* acc, const ViewDesc* views, int view_first, int num_views,
                     float lambda, int window, int advance, cudaStream_t s) {
    step_end_kernel<<<1, 1, 0, s>>>(status, acc, views, view_first, num_views, lambda, window, advance);
}

void launch_loss_from_acc(DevStatus* status, const double* acc, const ViewDesc* views, int view_first,
                          int num_views, float lambda, int window, cudaStream_t s) {
    step_end_kernel<<<1, 1, 0, s>>>(status, acc, views, view_first, num_views, lambda, window, 0);
}

// Tail of the gradient buffer after the gradients-only phase: [0] sum over this replica's
// views of their mean losses, [1] 1 if its instances overflowed, [2] its view count.
// Reduced (summed) across replicas together with the gradients.
__global__ void grad_tail_kernel(const DevStatus* st, const double* acc, const ViewDesc* views, int view_first,
                                 int num_views, float lambda, int window, float* tail) {
    const int t = threadIdx.x;
    if (t == 0) tail[0] = step_loss(acc, views, view_first, num_views, lambda, window) * (float)num_views;
    else if (t == 1) tail[1] = (st->overflow || st->sort_timeout) ? 1.f : 0.f;
    else if (t == 2) tail[2] = (float)num_views;
    else if (t < GS_GRAD_TAIL_FLOATS) tail[t] = 0.f;
}

void launch_grad_tail(const DevStatus* status, const double* acc, const ViewDesc* views, int view_first,
                      int num_views, float lambda, int window, float* tail, cudaStream_t s) {
    grad_tail_kernel<<<1, GS_GRAD_TAIL_FLOATS, 0, s>>>(status, acc, views, view_first, num_views, lambda, window,
                                                       tail);
}

// Book-keeping after the update from a reduced tail: loss = mean over all replicas'
// views, skipped when any replica overflowed.
__global__ void reduced_step_end_kernel(DevStatus* st, const float* tail) {
    const float views = fmaxf(tail[2], 1.f);
    const float loss = tail[0] / views;
    const bool skip = tail[1] > 0.f;
    st->loss = loss;
    st->nonfinite = isfinite(loss) ? 0 : 1;
    st->skipped = skip ? 1 : 0;
    if (!skip) st->step_t += 1;
}

void launch_reduced_step_end(DevStatus* status, const float* tail, cudaStream_t s) {
    reduced_step_end_kernel<<<1, 1, 0, s>>>(status, tail);
}

// Screen gradients of one view in the reference's 16-float per-Gaussian layout
// (trainer/gpu.js:9-10): 0-2 colour, 3 opacity logit, 4-8 u, v, conic A, B, C.
__global__ void screen_grads16_kernel(const float4* sg8, const float* sg1, int n, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = sg8[(size_t)i * 2], b = sg8[(size_t)i * 2 + 1];
    float* o = out + (size_t)i * 16;
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
    o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
    o[8] = sg1[i];
    for (int k = 9; k < 16; k++) o[k] = 0.f;
}

void launch_screen_grads16(const float4* sg8, const float* sg1, int n, float* out16, cudaStream_t s) {
    if (n > 0) screen_grads16_kernel<<<(n + 255) / 256, 256, 0, s>>>(sg8, sg1, n, out16);
}

// Splat records in the reference's 12-float layout (trainer/gpu.js:7).
__global__ void splats12_kernel(const float4* geo0, const float4* geo1, const float4* rgb, const uint32_t* keys,
                                int n, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 g0 = geo0[i], g1 = geo1[i], c = rgb[i];
    float* o = out + (size_t)i * 12;
    o[0] = g0.x; o[1] = g0.y; o[2] = g0.z; o[3] = g0.w;
    o[4] = g1.x; o[5] = g1.y; o[6] = g1.z; o[7] = g1.w;
    o[8] = c.x; o[9] = c.y; o[10] = c.z; o[11] = c.w;
    (void)keys;
}

void launch_splats12(const float4* geo0, const float4* geo1, const float4* rgb, const uint32_t* keys, int n,
                     float* out12, cudaStream_t s) {
    if (n > 0) splats12_kernel<<<(n + 255) / 256, 256, 0, s>>>(geo0, geo1, rgb, keys, n, out12);
}

}  // namespace gs
