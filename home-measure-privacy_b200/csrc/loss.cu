// Fused photometric loss: (1 - lambda) * L1 + lambda * (1 - SSIM) and dLoss/dPixel in
// one pass over image and target, for every view of a step.
//
// The reference splits this into SSIM_COEF (trainer/gpu.js:336-372: per window centre
// and channel, SSIM and its partials a, b, d by the window mean, mean of squares and
// mean of products) and LOSS_GRAD (:374-409: each pixel sums a + 2 x b + y d over the
// windows that cover it, 49 taps each, reading the coefficients back from HBM).  Here
// one CTA owns one colour channel of a 32 x 32 block of output pixels (the three
// channel CTAs of a block are neighbours in the grid, so they share the interleaved
// RGB lines in L2) and keeps everything in shared memory: it loads image and target
// with a 2R halo, forms the window moments with a separable (horizontal then
// vertical) filter, turns them into the coefficients a, b, d at every window centre
// that can reach the block, and filters those coefficients back (again separably) to
// get each pixel's SSIM gradient.  Only four moments are kept: the SSIM denominator
// needs the two means of squares only as their sum.  Each pass gives every thread a
// strip of outputs and streams the strip's inputs once, adding each input to every
// output whose window holds it, so the registers hold the strip's accumulators and not
// a window of inputs.  Windows are the reference's: centres whose whole window lies
// inside the image (7x7 box, R = 3), or the 11-tap Gaussian (sigma 1.5, R = 5) with the
// same rule.  The kernel also sums |x - y| and the SSIM of the windows centred in its
// block for the loss value.  The filters carry their values in pairs (x and y, the two
// moments of squares and products, coefficients a and b) through the packed FP32
// instructions of sm_100 (FFMA2), which round each half as the scalar FFMA does: the
// same sums with half the instructions.
#include "internal.h"

namespace gs {

// Output block of a CTA and its threads (build options; every pass gives each thread one
// strip of outputs, which the static assert below checks).
#ifndef LOSS_BW
#define LOSS_BW 32
#endif
#ifndef LOSS_BH
#define LOSS_BH 32
#endif
#ifndef LOSS_THREADS
#define LOSS_THREADS 256
#endif
#ifndef LOSS_NS1
#define LOSS_NS1 4  // strips per region row in the first pass
#endif
#ifndef LOSS_MIN_BLOCKS
#define LOSS_MIN_BLOCKS 3
#endif
constexpr int LB_W = LOSS_BW;
constexpr int LB_H = LOSS_BH;
constexpr int LB_THREADS = LOSS_THREADS;
static_assert(LB_THREADS >= 256 && LB_THREADS % 32 == 0, "the byte table takes one thread per value");

struct LossWeights {
    float w[11];
    float2 w2[11];  // each tap twice, a packed-FMA operand
};

__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

template <int R>
struct LossDims {
    static constexpr int K = 2 * R + 1;
    static constexpr int RW = LB_W + 4 * R;   // region with halo 2R
    static constexpr int RH = LB_H + 4 * R;
    static constexpr int HW = LB_W + 2 * R;   // window centres reaching the block
    static constexpr int CH = LB_H + 2 * R;
    static constexpr int HMP = HW + 2;        // row pitches chosen against bank conflicts
    static constexpr int CFP = HW + 1;
    // Strips: P1 horizontal moments, P2 vertical moments -> coefficients, P3 horizontal
    // coefficients, P4 vertical coefficients -> gradient.  One task per thread each.
    static constexpr int NS1 = LOSS_NS1;                    // strips per region row
    static constexpr int S1 = (HW + NS1 - 1) / NS1;
    static constexpr int S2 = 7;
    static constexpr int NS2 = (CH + S2 - 1) / S2;
    static constexpr int S3 = 6;
    static constexpr int NS3 = (LB_W + S3 - 1) / S3;
    static constexpr int S4 = 4;
    static constexpr int NS4 = LB_H / S4;
    // Region A: image and target with halo as (x, y) pairs, later the coefficients as
    // (a, b) pairs and d (the pixels are dead once the horizontal moments exist; the
    // gradient pass reads its own pixels from HBM).
    static constexpr int XY = 2 * RH * RW;
    static constexpr int CF = 3 * CH * CFP;
    static constexpr int A = ((XY > CF ? XY : CF) + 1) & ~1;  // even: region B holds float2
    // Region B: horizontal moments as (x, y) and (x^2 + y^2, xy) pairs, later the
    // horizontally filtered coefficients as (a, b) pairs and d.
    static constexpr int HM = 4 * RH * HMP;
    static constexpr int HC = 3 * CH * LB_W;
    static constexpr int B = HM > HC ? HM : HC;
    static constexpr int FLOATS = A + B;
    static_assert(RH * NS1 <= LB_THREADS && HW * NS2 <= LB_THREADS && CH * NS3 <= LB_THREADS &&
                      LB_W * NS4 <= LB_THREADS,
                  "one task per thread per pass");
};

__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Targets as floats: u8 photos through a per-CTA table of v / 255 (the correctly
// rounded quotient, equal to the reference's double quotient rounded to float for every
// byte), float targets as they are.
template <typename TT>
__device__ __forceinline__ float load_target(const TT* t, size_t idx, const float* lut);
template <>
__device__ __forceinline__ float load_target<uint8_t>(const uint8_t* t, size_t idx, const float* lut) {
    return lut[t[idx]];
}
template <>
__device__ __forceinline__ float load_target<float>(const float* t, size_t idx, const float*) {
    return t[idx];
}

template <int R, typename TT>
__global__ void __launch_bounds__(LB_THREADS, LOSS_MIN_BLOCKS) loss_kernel(LossArgs a, const TT* __restrict__ target,
                                                          LossWeights wts) {
    using D = LossDims<R>;
    constexpr int K = D::K;
    extern __shared__ __align__(16) float sm[];
    __shared__ float s_red[2][LB_THREADS / 32];
    __shared__ float s_lut[256];
    if (sizeof(TT) == 1 && threadIdx.x < 256) s_lut[threadIdx.x] = (float)threadIdx.x / 255.0f;
    const int blk = a.block_first + (int)(blockIdx.x / 3u);
    const int c = (int)(blockIdx.x % 3u);
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
    float2* XY = reinterpret_cast<float2*>(sm);                       // [RH][RW] (x, y)
    float2* CFAB = reinterpret_cast<float2*>(sm);                     // [CH][CFP] (a, b)
    float* CFD = sm + 2 * D::CH * D::CFP;                             // [CH][CFP] d
    float2* HMA = reinterpret_cast<float2*>(sm + D::A);               // [RH][HMP] (x, y)
    float2* HMB = HMA + D::RH * D::HMP;                               // [RH][HMP] (x^2 + y^2, xy)
    float2* HCAB = reinterpret_cast<float2*>(sm + D::A);              // [CH][LB_W] (a, b)
    float* HCD = sm + D::A + 2 * D::CH * LB_W;                        // [CH][LB_W] d
    float l1 = 0.f, ssim_sum = 0.f;
    const float C1 = 1e-4f, C2 = 9e-4f;
    const int tid = threadIdx.x;
    __syncthreads();  // byte table
    if (use_ssim) {
        // A thread owns one region column and every NRG-th row of it: one address step
        // per row, no index division.  All of its loads are issued before the first
        // shared-memory store.
        constexpr int NRG = LB_THREADS / D::RW;            // row groups
        constexpr int NL = (D::RH + NRG - 1) / NRG;        // rows per thread
        const int rx = tid % D::RW, rg = tid / D::RW;
        if (rg < NRG) {
            const int gx = bx0 - 2 * R + rx;
            const bool col_ok = gx >= 0 && gx < W;
            const int gy0 = by0 - 2 * R + rg;
            const long long q0 = ((long long)poff + (long long)gy0 * W + gx) * 3 + c;
            const long long step = (long long)NRG * W * 3;
            float xl[NL], yl[NL];
#pragma unroll
            for (int i = 0; i < NL; i++) {
                const int gy = gy0 + i * NRG;
                xl[i] = 0.f;
                yl[i] = 0.f;
                if (col_ok && rg + i * NRG < D::RH && gy >= 0 && gy < H) {
                    const size_t q = (size_t)(q0 + i * step);
                    xl[i] = a.image[q];
                    yl[i] = load_target<TT>(target, q, s_lut);
                }
            }
#pragma unroll
            for (int i = 0; i < NL; i++)
                if (rg + i * NRG < D::RH) XY[(rg + i * NRG) * D::RW + rx] = make_float2(xl[i], yl[i]);
        }
        __syncthreads();
        // P1: horizontal moments (x, y, x^2 + y^2, xy) at the centre columns of a strip.
        if (tid < D::RH * D::NS1) {
            const int r = tid / D::NS1, c0 = (tid % D::NS1) * D::S1;
            float2 acc[D::S1][2];  // (x, y), (x^2 + y^2, xy)
#pragma unroll
            for (int k = 0; k < D::S1; k++) acc[k][0] = acc[k][1] = make_float2(0.f, 0.f);
#pragma unroll
            for (int j = 0; j < D::S1 + 2 * R; j++) {
                const int col = c0 + j;
                const float2 v = col < D::RW ? XY[r * D::RW + col] : make_float2(0.f, 0.f);
                const float2 sq = make_float2(fmaf(v.x, v.x, v.y * v.y), v.x * v.y);
#pragma unroll
                for (int k = 0; k < D::S1; k++) {
                    if (j - k < 0 || j - k >= K) continue;
                    const float2 wt = wts.w2[j - k];
                    acc[k][0] = fma2(wt, v, acc[k][0]);
                    acc[k][1] = fma2(wt, sq, acc[k][1]);
                }
            }
#pragma unroll
            for (int k = 0; k < D::S1; k++) {
                if (c0 + k >= D::HW) break;
                HMA[r * D::HMP + c0 + k] = acc[k][0];
                HMB[r * D::HMP + c0 + k] = acc[k][1];
            }
        }
        __syncthreads();
        // P2: vertical moments at a strip of window centres -> SSIM coefficients.
        const bool p2 = tid < D::HW * D::NS2;
        const int hc = tid % D::HW, h0 = (tid / D::HW) * D::S2;
        float2 acc2[D::S2][2];
#pragma unroll
        for (int k = 0; k < D::S2; k++) acc2[k][0] = acc2[k][1] = make_float2(0.f, 0.f);
        if (p2) {
#pragma unroll
            for (int j = 0; j < D::S2 + 2 * R; j++) {
                const int row = h0 + j;
                const float2 va = row < D::RH ? HMA[row * D::HMP + hc] : make_float2(0.f, 0.f);
                const float2 vb = row < D::RH ? HMB[row * D::HMP + hc] : make_float2(0.f, 0.f);
#pragma unroll
                for (int k = 0; k < D::S2; k++) {
                    if (j - k < 0 || j - k >= K) continue;
                    const float2 wt = wts.w2[j - k];
                    acc2[k][0] = fma2(wt, va, acc2[k][0]);
                    acc2[k][1] = fma2(wt, vb, acc2[k][1]);
                }
            }
        }
        // The coefficients alias the pixels, which only P1 read.
        if (p2) {
            const int gx = bx0 - R + hc;
            const bool col_ok = gx >= R && gx < W - R;
            const bool col_in = gx >= bx0 && gx < bx0 + LB_W;
#pragma unroll
            for (int k = 0; k < D::S2; k++) {
                const int hr = h0 + k;
                if (hr >= D::CH) break;
                const int gy = by0 - R + hr;
                float ca = 0.f, cb = 0.f, cd = 0.f;
                if (col_ok && gy >= R && gy < H - R) {
                    const float mx = acc2[k][0].x, my = acc2[k][0].y, s2 = acc2[k][1].x, sxy = acc2[k][1].y;
                    const float a1 = 2.0f * mx * my + C1;
                    const float a2 = 2.0f * (sxy - mx * my) + C2;
                    const float b1 = mx * mx + my * my + C1;
                    const float b2 = (s2 - mx * mx - my * my) + C2;
                    // The approximate reciprocal instruction (about 1 ulp) without flushing
                    // subnormals; a1, b1 >= C1 and b2 >= C2 (variances are >= 0 up to
                    // rounding), a2 = 2 cov + C2 may take either sign.
                    const float ia1 = rcp_approx(a1), ia2 = rcp_approx(a2);
                    const float ib1 = rcp_approx(b1), ib2 = rcp_approx(b2);
                    const float ssim = a1 * a2 * ib1 * ib2;
                    ca = 2.0f * ssim * (my * ia1 - my * ia2 - mx * ib1 + mx * ib2);
                    cb = -ssim * ib2;
                    cd = 2.0f * ssim * ia2;
                    if (col_in && gy >= by0 && gy < by0 + LB_H) ssim_sum += ssim;
                }
                const int o = hr * D::CFP + hc;
                CFAB[o] = make_float2(ca, cb);
                CFD[o] = cd;
            }
        }
        __syncthreads();
        // P3: filter the coefficients back, horizontal ...
        if (tid < D::CH * D::NS3) {
            const int hr = tid / D::NS3, o0 = (tid % D::NS3) * D::S3;
            float2 acc[D::S3];
            float accd[D::S3];
#pragma unroll
            for (int k = 0; k < D::S3; k++) {
                acc[k] = make_float2(0.f, 0.f);
                accd[k] = 0.f;
            }
#pragma unroll
            for (int j = 0; j < D::S3 + 2 * R; j++) {
                const int col = o0 + j;
                const float2 vab = col < D::HW ? CFAB[hr * D::CFP + col] : make_float2(0.f, 0.f);
                const float vd = col < D::HW ? CFD[hr * D::CFP + col] : 0.f;
#pragma unroll
                for (int k = 0; k < D::S3; k++) {
                    if (j - k < 0 || j - k >= K) continue;
                    acc[k] = fma2(wts.w2[j - k], vab, acc[k]);
                    accd[k] = fmaf(w[j - k], vd, accd[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < D::S3; k++) {
                if (o0 + k >= LB_W) break;
                HCAB[hr * LB_W + o0 + k] = acc[k];
                HCD[hr * LB_W + o0 + k] = accd[k];
            }
        }
        __syncthreads();
    }
    // P4: ... and vertical, then the per-pixel gradient (with the L1 term).
    if (tid < LB_W * D::NS4) {
        const int ox = tid % LB_W, oy0 = (tid / LB_W) * D::S4;
        const int gx = bx0 + ox;
        float2 acc[D::S4];
        float accd[D::S4];
#pragma unroll
        for (int k = 0; k < D::S4; k++) {
            acc[k] = make_float2(0.f, 0.f);
            accd[k] = 0.f;
        }
        if (use_ssim) {
#pragma unroll
            for (int j = 0; j < D::S4 + 2 * R; j++) {
                const float2 vab = HCAB[(oy0 + j) * LB_W + ox];
                const float vd = HCD[(oy0 + j) * LB_W + ox];
#pragma unroll
                for (int k = 0; k < D::S4; k++) {
                    if (j - k < 0 || j - k >= K) continue;
                    acc[k] = fma2(wts.w2[j - k], vab, acc[k]);
                    accd[k] = fmaf(w[j - k], vd, accd[k]);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < D::S4; k++) {
            const int gy = by0 + oy0 + k;
            if (gx >= W || gy >= H) continue;
            const size_t q = (poff + (size_t)gy * W + gx) * 3 + c;
            const float xv = a.image[q];
            const float yv = load_target<TT>(target, q, s_lut);
            const float diff = xv - yv;
            float g = l1_scale * (float)((diff > 0.f) - (diff < 0.f));
            l1 += fabsf(diff);
            if (use_ssim) g -= ssim_scale * (acc[k].x + 2.0f * xv * acc[k].y + yv * accd[k]);
            a.dl[q] = g;
        }
    }
    // Block sums of |x - y| and SSIM -> per-view accumulators.
    const int lane = tid & 31, warp = tid >> 5;
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
    if (tid == 0) {
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
    for (int k = 0; k < 11; k++) w.w2[k] = make_float2(w.w[k], w.w[k]);
    return w;
}

template <int R, typename TT>
static void loss_launch(const LossArgs& a, const TT* target, const LossWeights& w, cudaStream_t s) {
    const size_t smem = LossDims<R>::FLOATS * sizeof(float);
    loss_kernel<R, TT><<<(unsigned)a.num_blocks * 3u, LB_THREADS, smem, s>>>(a, target, w);
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
