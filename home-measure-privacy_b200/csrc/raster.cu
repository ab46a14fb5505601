// Tiled alpha blending, forward and backward.
//
// One CTA of 256 threads owns one 16 x 16 pixel tile (one pixel per thread).  The
// tile's depth-ordered list is walked in batches: the CTA stages a batch of splat
// records (32-byte geometry + 16-byte colour, gathered by pair index) in shared memory
// with cp.async, double-buffered so the next batch's gather overlaps the current
// batch's blending, then every thread blends its pixel against the batch.
//
// Forward = FORWARD (trainer/gpu.js:105-137) with alphaAt (:91-103): square bounding-box
// test, Gaussian power, alpha = min(0.99, opacity * exp(power)), skip below 1/255, stop
// once T <= 1e-4, keep (final T, last contributor + 1).  A pixel that stopped retires;
// the CTA stops when all 256 have (one __syncthreads_count per batch).
//
// Backward = BACKWARD_SG (trainer/gpu.js:208-293): the tile walks its list back to front
// from the largest `last` of its pixels; each pixel rebuilds T before every splat from
// the stored final T (T_k = T / (1 - alpha)) and its running `behind` colour.  The nine
// gradients (colour, opacity logit, u, v, conic) of one splat are summed over the warp
// with a transposed butterfly (8 values in 9 shuffles, plus 5 for the ninth), after
// which 8 lanes issue one 32-byte vector of float reductions and lane 0 a ninth: one
// global atomic transaction per (warp, splat) instead of nine CAS loops per pixel
// (the reference's addF, :148-157).
//
// In the persistent mode a fixed grid pulls (view, tile) work items from a global
// counter, in an order that puts the longest tile lists first.
#include "internal.h"

namespace gs {

constexpr unsigned FULL_MASK = 0xffffffffu;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Thread -> pixels.  With PPT pixels per thread the CTA has 256 / PPT threads; warp w
// covers an 8 x (4 PPT) block of the 16 x 16 tile (a squarer footprint than full rows,
// so fewer splats reach each warp); lane l owns x = l & 7, y = l >> 3 (+ 4 p for its
// p-th pixel).
template <int PPT>
struct TileInfo {
    int g;                     // global tile id
    int x, y[PPT];             // this thread's pixels
    int width, height;
    int pixel_offset;
    bool inside[PPT];
    float wx0, wx1, wy0, wy1;  // pixel-centre rectangle of this thread's warp
};

template <int PPT>
__device__ __forceinline__ TileInfo<PPT> tile_info(const RasterArgs& a, int item) {
    TileInfo<PPT> ti;
    const int local = a.tile_order ? (int)a.tile_order[item] : item;
    ti.g = a.tile_first + local;
    int vi = a.view_first;
    const int vend = a.view_first + a.num_views;
    while (vi + 1 < vend && a.views[vi + 1].tile_offset <= ti.g) vi++;
    const ViewDesc& vw = a.views[vi];
    const int lt = ti.g - vw.tile_offset;
    const int tx = lt % vw.tiles_x, ty = lt / vw.tiles_x;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bx = tx * GS_TILE + (w & 1) * 8, by = ty * GS_TILE + (w >> 1) * 4 * PPT;
    ti.x = bx + (lane & 7);
#pragma unroll
    for (int p = 0; p < PPT; p++) {
        ti.y[p] = by + (lane >> 3) + 4 * p;
        ti.inside[p] = ti.x < vw.width && ti.y[p] < vw.height;
    }
    ti.width = vw.width;
    ti.height = vw.height;
    ti.pixel_offset = vw.pixel_offset;
    ti.wx0 = (float)bx + 0.5f;
    ti.wx1 = (float)bx + 7.5f;
    ti.wy0 = (float)by + 0.5f;
    ti.wy1 = (float)(by + 4 * PPT) - 0.5f;
    return ti;
}

// Next work item: the block index, or the queue head in persistent mode.
__device__ __forceinline__ int next_item(unsigned int* counter, int* s_item, int fallback) {
    if (!counter) return fallback;
    __syncthreads();
    if (threadIdx.x == 0) *s_item = (int)atomicAdd(counter, 1u);
    __syncthreads();
    return *s_item;
}

__device__ __forceinline__ void stage_batch(const RasterArgs& a, uint32_t first, int cnt, bool reverse,
                                            float4* s_g0, float4* s_g1, float4* s_c, uint32_t* s_pair) {
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
        const uint32_t k = reverse ? first - 1 - t : first + t;
        const uint32_t pair = __ldg(a.inst_pair + k);
        if (s_pair) s_pair[t] = pair;
        cp_async16(&s_g0[t], a.geo0 + pair);
        cp_async16(&s_g1[t], a.geo1 + pair);
        cp_async16(&s_c[t], a.rgb + pair);
    }
    cp_async_commit();
}

constexpr float LOG2E = 1.4426950408889634f;

// 2^e by the PTX ex2.approx instruction (relative error about 2^-22; e here lies in
// [log2(1/255), 0], far from the subnormal range the .ftz qualifier flushes).
__device__ __forceinline__ float ex2_approx(float e) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(e));
    return r;
}

// 1/x by the PTX rcp.approx instruction, for x = 1 - alpha in [0.01, 1].
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
constexpr float ALPHA_Q_BAND = 1e-4f;  // |q - log2(alpha_min)| below this: reference formula

// After the batch's copies landed, each staging thread derives for its splats:
// s_g1.w = the culling bound 2 ln(opacity / alpha_min) + slack (a pixel can reach
// alpha >= alpha_min only where the conic's quadratic form is below it), and
// s_q = (-A/2, -B, -C/2) log2(e) and log2(opacity), so that alpha = 2^q with
// q = log2(op) + qa dx^2 + qb dx dy + qc dy^2.
__device__ __forceinline__ void prepare_batch(int cnt, float4* s_g0, float4* s_g1, float4* s_q, float log_amin) {
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
        const float4 g0 = s_g0[t];
        const float4 g1 = s_g1[t];
        const float op = g1.y;
        s_g1[t].w = op > 0.f ? 2.0f * (__logf(op) - log_amin) + 1e-3f : -1.0f;
        s_q[t] = make_float4(-0.5f * LOG2E * g0.z, -LOG2E * g0.w, -0.5f * LOG2E * g1.x,
                             op > 0.f ? __log2f(op) : -1e30f);
    }
}

// alpha of splat (g0, g1, q) at offset (dx, dy), or 0 when the pixel skips it:
// alphaAt (trainer/gpu.js:91-103).  2^q by the fast exp2; within ALPHA_Q_BAND of the
// alpha_min threshold the reference expression min(0.99, op exp(power)) decides (a rare
// branch), so skip decisions match the reference's.  Otherwise branch-free.  Explicit
// rounding intrinsics keep forward and backward bit-identical.
__device__ __forceinline__ float alpha_band(const float4& g0, const float4& g1, float dx, float dy, float amax,
                                         float amin) {
    const float power = __fsub_rn(__fmul_rn(-0.5f, __fadd_rn(__fmul_rn(__fmul_rn(g0.z, dx), dx),
                                                             __fmul_rn(__fmul_rn(g1.x, dy), dy))),
                                  __fmul_rn(__fmul_rn(g0.w, dx), dy));
    if (power > 0.f) return 0.f;
    // The specified exp (gs_common.cuh), as the CPU restatement uses: the two agree
    // bit for bit even when alpha lies within an ulp of alpha_min.
    const float alpha = __fmul_rn(g1.y, spec_expf(power));
    return alpha < amin ? 0.f : fminf(amax, alpha);
}

__device__ __forceinline__ float alpha_at(const float4& g0, const float4& g1, const float4& q, float dx, float dy,
                                          float amax, float amin, float qlo, float qhi) {
    const float t = __fmaf_rn(q.y, dy, __fmul_rn(q.x, dx));
    float e = __fmaf_rn(dx, t, q.w);
    e = __fmaf_rn(__fmul_rn(q.z, dy), dy, e);
    const bool inb = fabsf(dx) <= g1.z && fabsf(dy) <= g1.z;
    float alpha = (inb && e >= qhi) ? fminf(amax, ex2_approx(e)) : 0.f;
    if (inb && e >= qlo && e < qhi) alpha = alpha_band(g0, g1, dx, dy, amax, amin);
    return alpha;
}

// Can splat (g0, g1) give any pixel centre of the warp's rectangle alpha >= alpha_min?
// Conservative: the pixels' own tests (bounding box, then alpha) decide; this only
// skips splats that cannot pass them anywhere in the rectangle.
template <int PPT>
__device__ __forceinline__ bool warp_reaches(const float4& g0, const float4& g1, const TileInfo<PPT>& ti) {
    return splat_reaches_box(g0.x, g0.y, g0.z, g0.w, g1.x, g1.z, g1.w, ti.wx0, ti.wx1, ti.wy0, ti.wy1);
}

// Resident CTAs per SM the register allocation is sized for (64 threads with 4 pixels
// each get more registers per thread than 16 CTAs would leave them).
constexpr int fwd_min_ctas(int ppt) { return ppt == 4 ? 12 : 4 * ppt; }
constexpr int bwd_min_ctas(int ppt) { return ppt == 4 ? 10 : (ppt == 2 ? 7 : 4); }

template <int BATCH, int PPT>
__global__ void __launch_bounds__(256 / PPT, fwd_min_ctas(PPT)) raster_fwd_kernel(RasterArgs a) {
    __shared__ __align__(16) float4 s_g0[2][BATCH];
    __shared__ __align__(16) float4 s_g1[2][BATCH];
    __shared__ __align__(16) float4 s_c[2][BATCH];
    __shared__ __align__(16) float4 s_q[2][BATCH];
    __shared__ int s_item;
    const int lane = threadIdx.x & 31;
    const float log_amin = __logf(a.alpha_min);
    const float qthr = __log2f(a.alpha_min);
    const float qlo = qthr - ALPHA_Q_BAND, qhi = qthr + ALPHA_Q_BAND;
    int item = next_item(a.work_counter, &s_item, blockIdx.x);
    while (item < a.num_tiles) {
        const TileInfo<PPT> ti = tile_info<PPT>(a, item);
        const uint2 rg = a.ranges[ti.g];
        const uint32_t start = rg.x, end = rg.y;
        const float pxf = (float)ti.x + 0.5f;
        float pyf[PPT], T[PPT], cr[PPT], cg[PPT], cb[PPT];
        uint32_t last[PPT];
        bool done[PPT];
#pragma unroll
        for (int p = 0; p < PPT; p++) {
            pyf[p] = (float)ti.y[p] + 0.5f;
            T[p] = 1.0f;
            cr[p] = cg[p] = cb[p] = 0.f;
            last[p] = start;
            done[p] = !ti.inside[p];
        }
        int buf = 0;
        if (start < end) stage_batch(a, start, min((uint32_t)BATCH, end - start), false, s_g0[0], s_g1[0], s_c[0], nullptr);
        for (uint32_t b0 = start; b0 < end; b0 += BATCH) {
            const int cnt = (int)min((uint32_t)BATCH, end - b0);
            const uint32_t nb = b0 + BATCH;
            if (nb < end) {
                stage_batch(a, nb, min((uint32_t)BATCH, end - nb), false, s_g0[buf ^ 1], s_g1[buf ^ 1], s_c[buf ^ 1],
                            nullptr);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            prepare_batch(cnt, s_g0[buf], s_g1[buf], s_q[buf], log_amin);
            __syncthreads();
            const float4* g0s = s_g0[buf];
            const float4* g1s = s_g1[buf];
            const float4* cs = s_c[buf];
            const float4* qs = s_q[buf];
            bool all_done = true;
#pragma unroll
            for (int p = 0; p < PPT; p++) all_done = all_done && done[p];
            bool warp_done = __all_sync(FULL_MASK, all_done);
            for (int gb = 0; gb < cnt && !warp_done; gb += 32) {
                const int jl = gb + lane;
                const bool rel = jl < cnt && warp_reaches<PPT>(g0s[jl], g1s[jl], ti);
                uint32_t mask = __ballot_sync(FULL_MASK, rel);
                while (mask) {
                    const int j = gb + __ffs(mask) - 1;
                    mask &= mask - 1;
                    const float4 g0 = g0s[j];
                    const float4 g1 = g1s[j];
                    const float4 q = qs[j];
                    const float dx = pxf - g0.x;
#pragma unroll
                    for (int p = 0; p < PPT; p++) {
                        // Branch-free per lane (alpha = 0 leaves colour, T and last as
                        // they are); the warp skips the pixel row when no lane blends.
                        float alpha = alpha_at(g0, g1, q, dx, pyf[p] - g0.y, a.alpha_max, a.alpha_min, qlo, qhi);
                        alpha = done[p] ? 0.f : alpha;
                        if (!__any_sync(FULL_MASK, alpha != 0.f)) continue;
                        const float4 c = cs[j];
                        const float w = alpha * T[p];
                        cr[p] += c.x * w;
                        cg[p] += c.y * w;
                        cb[p] += c.z * w;
                        T[p] *= 1.0f - alpha;
                        last[p] = alpha != 0.f ? b0 + (uint32_t)j + 1u : last[p];
                        done[p] = done[p] || T[p] <= a.t_min;
                    }
                }
                all_done = true;
#pragma unroll
                for (int p = 0; p < PPT; p++) all_done = all_done && done[p];
                warp_done = __all_sync(FULL_MASK, all_done);
            }
            buf ^= 1;
            // All pixels done: the rest of the list cannot change the tile.
            if (__syncthreads_count(all_done) == (int)blockDim.x) {
                cp_async_wait<0>();
                break;
            }
        }
#pragma unroll
        for (int p = 0; p < PPT; p++) {
            if (!ti.inside[p]) continue;
            const size_t pix = (size_t)ti.pixel_offset + (size_t)ti.y[p] * ti.width + ti.x;
            a.image[pix * 3 + 0] = cr[p];
            a.image[pix * 3 + 1] = cg[p];
            a.image[pix * 3 + 2] = cb[p];
            a.t_final[pix] = T[p];
            a.last[pix] = last[p];
        }
        if (!a.work_counter) break;
        item = next_item(a.work_counter, &s_item, 0);
    }
}

// Sum of v[0..7] over the warp, transposed: afterwards lane l with (l & 3) == 0 holds the
// total of value (l >> 2).  9 shuffles instead of 40.
__device__ __forceinline__ float warp_sum8_transposed(float v[8]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const bool hi = lane & 16;
        const float send = hi ? v[i] : v[i + 4];
        const float keep = hi ? v[i + 4] : v[i];
        v[i] = keep + __shfl_xor_sync(FULL_MASK, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const bool hi = lane & 8;
        const float send = hi ? v[i] : v[i + 2];
        const float keep = hi ? v[i + 2] : v[i];
        v[i] = keep + __shfl_xor_sync(FULL_MASK, send, 8);
    }
    {
        const bool hi = lane & 4;
        const float send = hi ? v[0] : v[1];
        const float keep = hi ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(FULL_MASK, send, 4);
    }
    v[0] += __shfl_xor_sync(FULL_MASK, v[0], 2);
    v[0] += __shfl_xor_sync(FULL_MASK, v[0], 1);
    return v[0];
}

template <int BATCH, int PPT>
__global__ void __launch_bounds__(256 / PPT, bwd_min_ctas(PPT)) raster_bwd_kernel(RasterArgs a) {
    __shared__ __align__(16) float4 s_g0[2][BATCH];
    __shared__ __align__(16) float4 s_g1[2][BATCH];
    __shared__ __align__(16) float4 s_c[2][BATCH];
    __shared__ __align__(16) float4 s_q[2][BATCH];
    __shared__ uint32_t s_pair[2][BATCH];
    __shared__ int s_item;
    __shared__ unsigned int s_end;
    const int lane = threadIdx.x & 31;
    const float log_amin = __logf(a.alpha_min);
    const float qthr = __log2f(a.alpha_min);
    const float qlo = qthr - ALPHA_Q_BAND, qhi = qthr + ALPHA_Q_BAND;
    float* sg8f = reinterpret_cast<float*>(a.sg8);
    // Selector constants of this lane's reduced value g = lane / 4 (see the reduction):
    // (k0, kop, kA, kC) and kB.
    float4 sel;
    float sel_b;
    {
        const int g = lane >> 2;
        sel = make_float4(g < 4 ? 1.f : (g == 6 ? -0.5f : (g == 7 ? -1.f : 0.f)), g == 3 ? -1.f : 0.f,
                          g == 4 ? 1.f : 0.f, g == 5 ? 1.f : 0.f);
        sel_b = (g == 4 || g == 5) ? 1.f : 0.f;
    }
    int item = next_item(a.work_counter, &s_item, blockIdx.x);
    while (item < a.num_tiles) {
        const TileInfo<PPT> ti = tile_info<PPT>(a, item);
        const uint2 rg = a.ranges[ti.g];
        const uint32_t start = rg.x;
        const float pxf = (float)ti.x + 0.5f;
        float pyf[PPT], T[PPT], dlr[PPT], dlg[PPT], dlb[PPT], bd[PPT];
        uint32_t mylast[PPT];
        unsigned int tmax = start;
#pragma unroll
        for (int p = 0; p < PPT; p++) {
            pyf[p] = (float)ti.y[p] + 0.5f;
            T[p] = 0.f;
            dlr[p] = dlg[p] = dlb[p] = 0.f;
            bd[p] = 0.f;  // dL . (colour of the splats behind), "behind"
            mylast[p] = start;
            if (ti.inside[p]) {
                const size_t pix = (size_t)ti.pixel_offset + (size_t)ti.y[p] * ti.width + ti.x;
                T[p] = a.t_final[pix];
                mylast[p] = a.last[pix];
                dlr[p] = a.dl[pix * 3 + 0];
                dlg[p] = a.dl[pix * 3 + 1];
                dlb[p] = a.dl[pix * 3 + 2];
            }
            tmax = max(tmax, mylast[p]);
        }
        if (threadIdx.x == 0) s_end = start;
        __syncthreads();
        // Tile end = largest last of its pixels (BACKWARD_SG, trainer/gpu.js:247-253);
        // each warp also stops at its own largest last.
        unsigned int wmax = tmax;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) wmax = max(wmax, __shfl_xor_sync(FULL_MASK, wmax, o));
        if (lane == 0) atomicMax(&s_end, wmax);
        __syncthreads();
        const uint32_t end = s_end;
        int buf = 0;
        if (end > start)
            stage_batch(a, end, min((uint32_t)BATCH, end - start), true, s_g0[0], s_g1[0], s_c[0], s_pair[0]);
        for (uint32_t bend = end; bend > start;) {
            const uint32_t bstart = (bend - start > (uint32_t)BATCH) ? bend - BATCH : start;
            const int cnt = (int)(bend - bstart);
            if (bstart > start) {
                stage_batch(a, bstart, min((uint32_t)BATCH, bstart - start), true, s_g0[buf ^ 1], s_g1[buf ^ 1],
                            s_c[buf ^ 1], s_pair[buf ^ 1]);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            prepare_batch(cnt, s_g0[buf], s_g1[buf], s_q[buf], log_amin);
            __syncthreads();
            const float4* g0s = s_g0[buf];
            const float4* g1s = s_g1[buf];
            const float4* cs = s_c[buf];
            const float4* qs = s_q[buf];
            const uint32_t* ps = s_pair[buf];
            // Entry j of the batch is list position bend - 1 - j: ascending j walks back to
            // front.  Warps whose pixels all stopped before this batch skip it.
            if (bstart < wmax) {
                for (int gb = 0; gb < cnt; gb += 32) {
                    const int jl = gb + lane;
                    const bool rel = jl < cnt && (bend - 1 - (uint32_t)jl) < wmax && warp_reaches<PPT>(g0s[jl], g1s[jl], ti);
                    uint32_t mask = __ballot_sync(FULL_MASK, rel);
                    while (mask) {
                        const int j = gb + __ffs(mask) - 1;
                        mask &= mask - 1;
                        const uint32_t k = bend - 1 - (uint32_t)j;
                        const float4 g0 = g0s[j];
                        const float4 g1 = g1s[j];
                        const float4 q = qs[j];
                        const float dx = pxf - g0.x;
                        // Per pixel: colour terms and the moments of dP = dL/dpower over the
                        // offsets (sum dP, dP dx, dP dy, dP dx^2, dP dx dy, dP dy^2); the
                        // splat's conic and opacity turn the warp sums into the gradients of
                        // (opacity logit, u, v, A, B, C) after the reduction.
                        float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                        float v8 = 0.f;
                        bool contrib = false;  // warp-uniform
#pragma unroll
                        for (int p = 0; p < PPT; p++) {
                            // Branch-free per lane: alpha = 0 adds zeros and leaves T
                            // (T / 1) and dL.behind as they are.
                            const float dy = pyf[p] - g0.y;
                            float alpha = alpha_at(g0, g1, q, dx, dy, a.alpha_max, a.alpha_min, qlo, qhi);
                            alpha = k < mylast[p] ? alpha : 0.f;
                            if (!__any_sync(FULL_MASK, alpha != 0.f)) continue;
                            contrib = true;
                            const float4 c = cs[j];
                            const float ioma = rcp_approx(1.0f - alpha);
                            const float Tk = T[p] * ioma;
                            const float at = alpha * Tk;
                            v[0] += dlr[p] * at;
                            v[1] += dlg[p] * at;
                            v[2] += dlb[p] * at;
                            // dL/dalpha = dL.(c T_k - behind / (1 - alpha)); only dL.behind is
                            // kept per pixel.
                            const float dlc = dlr[p] * c.x + dlg[p] * c.y + dlb[p] * c.z;
                            const float dA = Tk * dlc - ioma * bd[p];
                            bd[p] += dlc * at;
                            T[p] = Tk;
                            // alpha clamped at alpha_max has no gradient through the power.
                            const float dP = alpha < a.alpha_max ? dA * alpha : 0.f;
                            const float dPx = dP * dx, dPy = dP * dy;
                            v[3] += dP;
                            v[4] += dPx;
                            v[5] += dPy;
                            v[6] += dPx * dx;
                            v[7] += dPx * dy;
                            v8 += dPy * dy;
                        }
                        if (contrib) {
                            float s = warp_sum8_transposed(v);
                            float s8 = v8;
#pragma unroll
                            for (int o = 16; o > 0; o >>= 1) s8 += __shfl_xor_sync(FULL_MASK, s8, o);
                            // lane 4g holds sum g: 3 -> opacity logit (x (1 - op)), 4/5 -> u/v
                            // (A Sx + B Sy, C Sy + B Sx), 6/7 -> A/B (-Sxx/2, -Sxy), C = -Syy/2.
                            // Branch-free: s = s (k0 + kop op + kA A + kC C) + other kB B with the
                            // lane's selector constants.
                            const float other = __shfl_xor_sync(FULL_MASK, s, 4);
                            const float m0 = fmaf(sel.w, g1.x, fmaf(sel.z, g0.z, fmaf(sel.y, g1.y, sel.x)));
                            s = fmaf(s, m0, other * (sel_b * g0.w));
                            s8 *= -0.5f;
                            const uint32_t pair = ps[j];
                            if ((lane & 3) == 0 && s != 0.0f) atomicAdd(sg8f + (size_t)pair * 8 + (lane >> 2), s);
                            if (lane == 0 && s8 != 0.0f) atomicAdd(a.sg1 + pair, s8);
                        }
                    }
                }
            }
            buf ^= 1;
            bend = bstart;
            __syncthreads();
        }
        if (!a.work_counter) break;
        item = next_item(a.work_counter, &s_item, 0);
    }
}

// Variant = (shared-memory batch, pixels per thread); the autotuner picks one.
static const int kBatches[3] = {64, 128, 256};

template <int BATCH, int PPT>
static void fwd_launch(const RasterArgs& a, int ctas, cudaStream_t s) {
    raster_fwd_kernel<BATCH, PPT><<<ctas, 256 / PPT, 0, s>>>(a);
}
template <int BATCH, int PPT>
static void bwd_launch(const RasterArgs& a, int ctas, cudaStream_t s) {
    raster_bwd_kernel<BATCH, PPT><<<ctas, 256 / PPT, 0, s>>>(a);
}

#define RASTER_SWITCH(FN, batch, ppt, ...)                   \
    do {                                                     \
        if ((ppt) == 4) {                                    \
            switch (batch) {                                 \
                case 64: FN<64, 4>(__VA_ARGS__); break;      \
                case 128: FN<128, 4>(__VA_ARGS__); break;    \
                default: FN<256, 4>(__VA_ARGS__); break;     \
            }                                                \
        } else if ((ppt) == 2) {                             \
            switch (batch) {                                 \
                case 64: FN<64, 2>(__VA_ARGS__); break;      \
                case 128: FN<128, 2>(__VA_ARGS__); break;    \
                default: FN<256, 2>(__VA_ARGS__); break;     \
            }                                                \
        } else {                                             \
            switch (batch) {                                 \
                case 64: FN<64, 1>(__VA_ARGS__); break;      \
                case 128: FN<128, 1>(__VA_ARGS__); break;    \
                default: FN<256, 1>(__VA_ARGS__); break;     \
            }                                                \
        }                                                    \
    } while (0)

void launch_raster_fwd(const RasterArgs& a, int batch, int ppt, int persistent_ctas, cudaStream_t s) {
    const int ctas = a.work_counter ? persistent_ctas : a.num_tiles;
    if (ctas <= 0 || a.num_tiles <= 0) return;
    RASTER_SWITCH(fwd_launch, batch, ppt, a, ctas, s);
}

void launch_raster_bwd(const RasterArgs& a, int batch, int ppt, int persistent_ctas, cudaStream_t s) {
    const int ctas = a.work_counter ? persistent_ctas : a.num_tiles;
    if (ctas <= 0 || a.num_tiles <= 0) return;
    RASTER_SWITCH(bwd_launch, batch, ppt, a, ctas, s);
}

template <int BATCH, int PPT>
static void occ(int* n, bool backward) {
    if (backward) cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, raster_bwd_kernel<BATCH, PPT>, 256 / PPT, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, raster_fwd_kernel<BATCH, PPT>, 256 / PPT, 0);
}

int raster_max_ctas_per_sm(int batch, int ppt, bool backward) {
    int n = 0;
    RASTER_SWITCH(occ, batch, ppt, &n, backward);
    cudaGetLastError();
    return n < 1 ? 1 : n;
}

// ---------------------------------------------------------------------------------
// Tile order for the persistent queue: tiles bucketed by floor(log2(list length)),
// longest bucket first (one block; the order inside a bucket does not matter).
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) tile_order_kernel(const uint2* ranges, int tile_first, int num_tiles,
                                                          uint32_t* order) {
    __shared__ unsigned int s_count[33];
    __shared__ unsigned int s_next[33];
    if (threadIdx.x < 33) s_count[threadIdx.x] = 0;
    __syncthreads();
    for (int t = threadIdx.x; t < num_tiles; t += blockDim.x) {
        const uint2 r = ranges[tile_first + t];
        const unsigned len = r.y - r.x;
        const int b = len ? 32 - __clz(len) : 0;  // 0..32
        atomicAdd(&s_count[b], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned run = 0;
        for (int b = 32; b >= 0; b--) {
            s_next[b] = run;
            run += s_count[b];
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < num_tiles; t += blockDim.x) {
        const uint2 r = ranges[tile_first + t];
        const unsigned len = r.y - r.x;
        const int b = len ? 32 - __clz(len) : 0;
        order[atomicAdd(&s_next[b], 1u)] = (uint32_t)t;
    }
}

void launch_tile_order(const uint2* ranges, int tile_first, int num_tiles, uint32_t* order, uint32_t* scratch,
                       cudaStream_t s) {
    (void)scratch;
    if (num_tiles <= 0) return;
    tile_order_kernel<<<1, 1024, 0, s>>>(ranges, tile_first, num_tiles, order);
}

// Blends of the last forward: sum over pixels of (last contributor + 1 - tile start),
// the (pixel, splat) evaluations the per-pixel blend of trainer/gpu.js:114-136 makes
// before the pixel stops; the backward replays the same pairs.
__global__ void blend_count_kernel(const ViewDesc* views, int view_first, const uint2* ranges,
                                   const uint32_t* last, unsigned long long* out) {
    const ViewDesc& vw = views[view_first + blockIdx.y];
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long n = 0;
    if (px < vw.width * vw.height) {
        const int x = px % vw.width, y = px / vw.width;
        const int tile = vw.tile_offset + (y / GS_TILE) * vw.tiles_x + x / GS_TILE;
        const uint32_t start = ranges[tile].x, l = last[(size_t)vw.pixel_offset + px];
        n = l > start ? (unsigned long long)(l - start) : 0ull;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(out, n);
}

void launch_blend_count(const ViewDesc* views, int view_first, int num_views, int max_pixels, const uint2* ranges,
                        const uint32_t* last, unsigned long long* out, cudaStream_t s) {
    if (num_views <= 0 || max_pixels <= 0) return;
    dim3 grid((max_pixels + 255) / 256, num_views);
    blend_count_kernel<<<grid, 256, 0, s>>>(views, view_first, ranges, last, out);
}

}  // namespace gs
