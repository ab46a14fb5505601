// Fused photometric loss: (1 - lambda) * L1 + lambda * (1 - SSIM) and dLoss/dPixel in
// one pass over image and target, for every view of a step.
//
// The reference splits this into SSIM_COEF (trainer/gpu.js:336-372: per window centre
// and channel, SSIM and its partials a, b, d by the window mean, mean of squares and
// mean of products) and LOSS_GRAD (:374-409: each pixel sums a + 2 x b + y d over the
// windows that cover it, 49 taps each, reading the coefficients back from HBM).  Here
// one CTA owns a 32 x 32 block of output pixels and keeps everything in shared memory:
// it loads image and target with a 2R halo, forms the five window moments with a
// separable (horizontal then vertical) filter, turns them into the coefficients
// a, b, d at every window centre that can reach the block, and filters those
// coefficients back (again separably) to get each pixel's SSIM gradient.  Every pass
// gives each thread a short strip of outputs computed from a register window, so one
// shared-memory load feeds up to 2R + 1 filter taps.  Windows are
// the reference's: centres whose whole window lies inside the image (7x7 box, R = 3),
// or the 11-tap Gaussian (sigma 1.5, R = 5) with the same rule.  The kernel also sums
// |x - y| and the SSIM of the windows centred in its block for the loss value.
#include "internal.h"

namespace gs {

constexpr int LB_W = 32;
constexpr int LB_H = 32;
constexpr int LB_THREADS = 256;
// Strip lengths of the four separable passes (outputs per thread task).
constexpr int S1 = 7;   // horizontal moments
constexpr int S2 = 4;   // vertical moments -> SSIM coefficients
constexpr int S3 = 4;   // horizontal coefficients
constexpr int S4 = 4;   // vertical coefficients -> gradient

struct LossWeights {
    float w[11];
};

template <int R>
struct LossDims {
    static constexpr int RW = LB_W + 4 * R;   // region with halo 2R
    static constexpr int RH = LB_H + 4 * R;
    static constexpr int HW = LB_W + 2 * R;   // window centres reaching the block
    static constexpr int CH = LB_H + 2 * R;
    static constexpr int X_OFF = 0;
    static constexpr int Y_OFF = RH * RW;
    static constexpr int HM_OFF = 2 * RH * RW;               // 5 moments, RH x HW
    static constexpr int C_OFF = HM_OFF + 5 * RH * HW;       // 3 coefficients, CH x HW
    static constexpr int HC_OFF = HM_OFF;                    // 3 filtered coefs, CH x LB_W (aliases moments)
    static constexpr int FLOATS = C_OFF + 3 * CH * HW;
};

__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

template <typename TT>
__device__ __forceinline__ float load_target(const TT* t, size_t idx);
template <>
__device__ __forceinline__ float load_target<uint8_t>(const uint8_t* t, size_t idx) {
    return (float)t[idx] / 255.0f;
}
template <>
__device__ __forceinline__ float load_target<float>(const float* t, size_t idx) {
    return t[idx];
}

template <int R, typename TT>
__global__ void __launch_bounds__(LB_THREADS, 2) loss_kernel(LossArgs a, const TT* __restrict__ target,
                                                          LossWeights wts) {
    using D = LossDims<R>;
    constexpr int K = 2 * R + 1;
    extern __shared__ float sm[];
    __shared__ float s_red[2][LB_THREADS / 32];
    const int blk = a.block_first + blockIdx.x;
    int vi = a.view_first;
    const int vend = a.view_first + a.num_views;
    while (vi + 1 < vend && a.views[vi + 1].loss_block_offset <= blk) vi++;
    const ViewDesc& vw = a.views[vi];
    const int lb = blk - vw.loss_block_offset;
    const int W = vw.width, H = vw.height;
    const int bx0 = (lb % vw.loss_blocks_x) * LB_W, by0 = (lb / vw.loss_blocks_x) * LB_H;
    const size_t poff = (size_t)vw.pixel_offset;
    const float n = (float)((long long)W * H * 3);
    const int winx = W - 2 * R, winy = H - 2 * R;
    const float windows = (winx > 0 && winy > 0) ? (float)winx * (float)winy * 3.0f : 0.0f;
    const float l1_scale = (1.0f - a.lambda) / n;
    const float ssim_scale = windows > 0.0f ? a.lambda / windows : 0.0f;
    const bool use_ssim = a.lambda > 0.0f && windows > 0.0f;
    // Filter taps stay in the kernel-parameter constant bank (FFMA operands).
    const float* w = wts.w;
    float* X = sm + D::X_OFF;
    float* Y = sm + D::Y_OFF;
    float* HM = sm + D::HM_OFF;
    float* CF = sm + D::C_OFF;
    float* HC = sm + D::HC_OFF;
    float l1 = 0.f, ssim_sum = 0.f;
    const float C1 = 1e-4f, C2 = 9e-4f;
    constexpr int NS1 = (D::HW + S1 - 1) / S1;
    constexpr int NS2 = (D::CH + S2 - 1) / S2;
    constexpr int NS3 = LB_W / S3;
    constexpr int NS4 = LB_H / S4;
    for (int c = 0; c < 3; c++) {
        if (use_ssim) {
            for (int idx = threadIdx.x; idx < D::RH * D::RW; idx += LB_THREADS) {
                const int ry = idx / D::RW, rx = idx % D::RW;
                const int gx = bx0 - 2 * R + rx, gy = by0 - 2 * R + ry;
                float xv = 0.f, yv = 0.f;
                if (gx >= 0 && gy >= 0 && gx < W && gy < H) {
                    const size_t q = (poff + (size_t)gy * W + gx) * 3 + c;
                    xv = a.image[q];
                    yv = load_target<TT>(target, q);
                }
                X[idx] = xv;
                Y[idx] = yv;
            }
            __syncthreads();
            // P1: horizontal moments, S1 centre columns per task from a register window.
            for (int task = threadIdx.x; task < D::RH * NS1; task += LB_THREADS) {
                const int r = task / NS1, c0 = (task % NS1) * S1;
                // Products formed once per window element, not once per tap.
                float xs[S1 + 2 * R], ys[S1 + 2 * R], xx[S1 + 2 * R], yy[S1 + 2 * R], xy[S1 + 2 * R];
#pragma unroll
                for (int t = 0; t < S1 + 2 * R; t++) {
                    const int col = c0 + t;
                    xs[t] = col < D::RW ? X[r * D::RW + col] : 0.f;
                    ys[t] = col < D::RW ? Y[r * D::RW + col] : 0.f;
                    xx[t] = xs[t] * xs[t];
                    yy[t] = ys[t] * ys[t];
                    xy[t] = xs[t] * ys[t];
                }
#pragma unroll
                for (int k = 0; k < S1; k++) {
                    if (c0 + k >= D::HW) break;
                    float mx = 0.f, my = 0.f, sxx = 0.f, syy = 0.f, sxy = 0.f;
#pragma unroll
                    for (int t = 0; t < K; t++) {
                        const float wt = w[t];
                        mx = fmaf(wt, xs[k + t], mx);
                        my = fmaf(wt, ys[k + t], my);
                        sxx = fmaf(wt, xx[k + t], sxx);
                        syy = fmaf(wt, yy[k + t], syy);
                        sxy = fmaf(wt, xy[k + t], sxy);
                    }
                    const int o = r * D::HW + c0 + k;
                    HM[0 * D::RH * D::HW + o] = mx;
                    HM[1 * D::RH * D::HW + o] = my;
                    HM[2 * D::RH * D::HW + o] = sxx;
                    HM[3 * D::RH * D::HW + o] = syy;
                    HM[4 * D::RH * D::HW + o] = sxy;
                }
            }
            __syncthreads();
            // P2: vertical moments at S2 window centres per task -> SSIM coefficients.
            for (int task = threadIdx.x; task < D::HW * NS2; task += LB_THREADS) {
                const int hc = task % D::HW, h0 = (task / D::HW) * S2;
                float m[5][S2 + 2 * R];
#pragma unroll
                for (int q = 0; q < 5; q++)
#pragma unroll
                    for (int t = 0; t < S2 + 2 * R; t++) {
                        const int row = h0 + t;
                        m[q][t] = row < D::RH ? HM[q * D::RH * D::HW + row * D::HW + hc] : 0.f;
                    }
#pragma unroll
                for (int k = 0; k < S2; k++) {
                    const int hr = h0 + k;
                    if (hr >= D::CH) break;
                    const int gx = bx0 - R + hc, gy = by0 - R + hr;
                    float ca = 0.f, cb = 0.f, cd = 0.f;
                    if (gx >= R && gy >= R && gx < W - R && gy < H - R) {
                        float mm[5];
#pragma unroll
                        for (int q = 0; q < 5; q++) {
                            float acc = 0.f;
#pragma unroll
                            for (int t = 0; t < K; t++) acc += w[t] * m[q][k + t];
                            mm[q] = acc;
                        }
                        const float mx = mm[0], my = mm[1], sxx = mm[2], syy = mm[3], sxy = mm[4];
                        const float a1 = 2.0f * mx * my + C1;
                        const float a2 = 2.0f * (sxy - mx * my) + C2;
                        const float b1 = mx * mx + my * my + C1;
                        const float b2 = (sxx - mx * mx) + (syy - my * my) + C2;
                        // The approximate reciprocal instruction (about 1 ulp) without flushing
                        // subnormals; a1, b1 >= C1 and b2 >= C2 (variances are >= 0 up to
                        // rounding), a2 = 2 cov + C2 may take either sign.
                        const float ia1 = rcp_approx(a1), ia2 = rcp_approx(a2);
                        const float ib1 = rcp_approx(b1), ib2 = rcp_approx(b2);
                        const float ssim = a1 * a2 * ib1 * ib2;
                        ca = 2.0f * ssim * (my * ia1 - my * ia2 - mx * ib1 + mx * ib2);
                        cb = -ssim * ib2;
                        cd = 2.0f * ssim * ia2;
                        if (gx >= bx0 && gx < bx0 + LB_W && gy >= by0 && gy < by0 + LB_H) ssim_sum += ssim;
                    }
                    const int o = hr * D::HW + hc;
                    CF[0 * D::CH * D::HW + o] = ca;
                    CF[1 * D::CH * D::HW + o] = cb;
                    CF[2 * D::CH * D::HW + o] = cd;
                }
            }
            __syncthreads();
            // P3: filter the coefficients back, horizontal ...
            for (int task = threadIdx.x; task < D::CH * NS3; task += LB_THREADS) {
                const int hr = task / NS3, o0 = (task % NS3) * S3;
                float cf[3][S3 + 2 * R];
#pragma unroll
                for (int q = 0; q < 3; q++)
#pragma unroll
                    for (int t = 0; t < S3 + 2 * R; t++) cf[q][t] = CF[q * D::CH * D::HW + hr * D::HW + o0 + t];
#pragma unroll
                for (int k = 0; k < S3; k++)
#pragma unroll
                    for (int q = 0; q < 3; q++) {
                        float acc = 0.f;
#pragma unroll
                        for (int t = 0; t < K; t++) acc += w[t] * cf[q][k + t];
                        HC[q * D::CH * LB_W + hr * LB_W + o0 + k] = acc;
                    }
            }
            __syncthreads();
        }
        // P4: ... and vertical, then the per-pixel gradient (with the L1 term).
        for (int task = threadIdx.x; task < LB_W * NS4; task += LB_THREADS) {
            const int ox = task % LB_W, oy0 = (task / LB_W) * S4;
            const int gx = bx0 + ox;
            float hc[3][S4 + 2 * R];
            if (use_ssim) {
#pragma unroll
                for (int q = 0; q < 3; q++)
#pragma unroll
                    for (int t = 0; t < S4 + 2 * R; t++) hc[q][t] = HC[q * D::CH * LB_W + (oy0 + t) * LB_W + ox];
            }
#pragma unroll
            for (int k = 0; k < S4; k++) {
                const int oy = oy0 + k, gy = by0 + oy;
                if (gx >= W || gy >= H) continue;
                const size_t q = (poff + (size_t)gy * W + gx) * 3 + c;
                float xv, yv;
                if (use_ssim) {
                    xv = X[(oy + 2 * R) * D::RW + ox + 2 * R];
                    yv = Y[(oy + 2 * R) * D::RW + ox + 2 * R];
                } else {
                    xv = a.image[q];
                    yv = load_target<TT>(target, q);
                }
                const float diff = xv - yv;
                float g = l1_scale * (float)((diff > 0.f) - (diff < 0.f));
                l1 += fabsf(diff);
                if (use_ssim) {
                    float sa = 0.f, sb = 0.f, sd = 0.f;
#pragma unroll
                    for (int t = 0; t < K; t++) {
                        sa += w[t] * hc[0][k + t];
                        sb += w[t] * hc[1][k + t];
                        sd += w[t] * hc[2][k + t];
                    }
                    g -= ssim_scale * (sa + 2.0f * xv * sb + yv * sd);
                }
                a.dl[q] = g;
            }
        }
        __syncthreads();
    }
    // Block sums of |x - y| and SSIM -> per-view accumulators.
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        l1 += __shfl_xor_sync(0xffffffffu, l1, o);
        ssim_sum += __shfl_xor_sync(0xffffffffu, ssim_sum, o);
    }
    if (lane == 0) {
        s_red[0][warp] = l1;
        s_red[1][warp] = ssim_sum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int k = 0; k < LB_THREADS / 32; k++) {
            t0 += s_red[0][k];
            t1 += s_red[1][k];
        }
        atomicAdd(a.acc + 2 * vi + 0, t0);
        atomicAdd(a.acc + 2 * vi + 1, t1);
    }
}

static LossWeights make_weights(int window) {
    LossWeights w{};
    if (window == 0) {
        for (int k = 0; k < 7; k++) w.w[k] = (float)(1.0 / 7.0);
    } else {
        double g[11], s = 0.0;
        for (int k = 0; k < 11; k++) {
            const double d = k - 5;
            g[k] = exp(-d * d / (2.0 * 1.5 * 1.5));
            s += g[k];
        }
        for (int k = 0; k < 11; k++) w.w[k] = (float)(g[k] / s);
    }
    return w;
}

template <int R, typename TT>
static void loss_launch(const LossArgs& a, const TT* target, const LossWeights& w, cudaStream_t s) {
    const size_t smem = LossDims<R>::FLOATS * sizeof(float);
    loss_kernel<R, TT><<<a.num_blocks, LB_THREADS, smem, s>>>(a, target, w);
}

void launch_loss(const LossArgs& a, cudaStream_t s) {
    if (a.num_blocks <= 0) return;
    const LossWeights w = make_weights(a.window);
    if (a.window == 0) {
        if (a.target_u8) loss_launch<3, uint8_t>(a, a.target_u8, w, s);
        else loss_launch<3, float>(a, a.target_f32, w, s);
    } else {
        if (a.target_u8) loss_launch<5, uint8_t>(a, a.target_u8, w, s);
        else loss_launch<5, float>(a, a.target_f32, w, s);
    }
}

// Raises the dynamic shared-memory limit of the loss kernels on the current device.
cudaError_t loss_prepare() {
    cudaError_t e = cudaSuccess, r;
    r = cudaFuncSetAttribute(loss_kernel<3, uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(LossDims<3>::FLOATS * sizeof(float)));
    if (r != cudaSuccess) e = r;
    r = cudaFuncSetAttribute(loss_kernel<3, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(LossDims<3>::FLOATS * sizeof(float)));
    if (r != cudaSuccess) e = r;
    r = cudaFuncSetAttribute(loss_kernel<5, uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(LossDims<5>::FLOATS * sizeof(float)));
    if (r != cudaSuccess) e = r;
    r = cudaFuncSetAttribute(loss_kernel<5, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(LossDims<5>::FLOATS * sizeof(float)));
    if (r != cudaSuccess) e = r;
    return e;
}

int loss_block_w() { return LB_W; }
int loss_block_h() { return LB_H; }

}  // namespace gs
