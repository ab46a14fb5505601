// Tiled alpha blending, forward and backward.
//
// A tile of TILE x TILE pixels (8, 16, 32 or 64; 16 is the reference's) is cut into
// groups of 8 x 4 pixels; lane l of a warp holds pixel (l & 7, l >> 3) of each group the
// warp owns.  With PPT pixels per thread a CTA of WT^2 / PPT threads owns a WT x WT work
// tile (the whole tile, or a 16 x 16 part of a 32- or 64-pixel tile) and each warp a
// block of PPT groups (1 x PPT groups, or 2 x 4 with 8 pixels per thread; Lay below).
// The tile's depth-ordered list is walked in batches: the CTA stages a batch of splat
// records (32-byte geometry + 16-byte colour, gathered by pair index) in shared memory
// with cp.async, double-buffered so the next batch's gather overlaps the current
// batch's blending.  Each warp then takes the staged splats 32 at a time, a lane per
// splat, and finds for each the warp's groups that its alpha >= alpha_min ellipse
// (clipped to its bounding square) can reach and whose pixels are still live; the splats
// with any such group are blended in order, group by group, and only those groups are
// evaluated.  Skipped groups have alpha = 0 at every pixel, so results are those of
// evaluating every pixel against every splat, whatever the tile size.
//
// Forward = FORWARD (trainer/gpu.js:105-137) with alphaAt (:91-103): square bounding-box
// test, Gaussian power, alpha = min(0.99, opacity * exp(power)), skip below 1/255, stop
// once T <= 1e-4, keep (final T, last contributor + 1).  Pixels that stopped retire their
// group once all 32 have; the tile stops when every group has.
//
// Backward = BACKWARD_SG (trainer/gpu.js:208-293): the tile walks its list back to front
// from the largest `last` of its pixels (each group from the largest `last` of its own
// pixels); each pixel rebuilds T before every splat from the stored final T
// (T_k = T / (1 - alpha)) and its running `behind` colour.  The nine gradients (colour,
// opacity logit, u, v, conic) of one splat are summed over the warp with a transposed
// butterfly (8 values in 9 shuffles, plus 5 for the ninth), after which 8 lanes issue one
// 32-byte vector of float reductions and lane 0 a ninth: one global atomic transaction
// per (warp, splat) instead of nine CAS loops per pixel (the reference's addF, :148-157).
//
// A CTA covers the whole tile or, for 32 x 32 and 64 x 64 tiles, one 16 x 16 part of it
// (a work tile); every part walks the tile's whole list.
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

// 2^e by the PTX ex2.approx instruction (relative error about 2^-22; e here lies in
// [log2(1/255), 0], far from the subnormal range the .ftz qualifier flushes).
__device__ __forceinline__ float ex2_approx(float e) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(e));
    return r;
}

// 1/x by the PTX rcp.approx instruction (x = 1 - alpha in [0.01, 1], or a positive
// conic coefficient).
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Two pixels of a thread that share an x band travel together as one float2 through
// the packed FP32 instructions of sm_100 (FFMA2 / FADD2 / FMUL2): each half is rounded
// as the scalar instruction would round it, so the blend is bit-identical to the scalar
// arithmetic while issuing half the instructions.
__device__ __forceinline__ float2 f2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }

// Layout of a CTA over one TILE x TILE tile with PPT pixels per thread: the tile is
// GX x GY groups of 8 x 4 pixels; each warp owns a block of WX x WY groups (WX = 2 when
// a thread has 8 pixels, else 1) and its p-th group is column p / WY, row p % WY of that
// block.
template <int TILE, int PPT>
struct Lay {
    static constexpr int NT = TILE * TILE / PPT;  // threads per CTA
    static constexpr int GX = TILE / 8, GY = TILE / 4;
    static constexpr int WX = PPT == 8 ? 2 : 1;
    static constexpr int WY = PPT / WX;
    static constexpr int NWX = GX / WX;           // warps across the tile
    static_assert(WX <= GX && WY <= GY && NT >= 32 && NT <= 1024, "no such raster layout");
    __device__ static int xg(int w, int p) { return (w % NWX) * WX + p / WY; }
    __device__ static int yg(int w, int p) { return (w / NWX) * WY + p % WY; }
};

template <int PPT>
constexpr uint32_t all_groups() {
    return (1u << PPT) - 1u;
}

template <int PPT>
struct TileInfo {
    int g;                       // global tile id
    int x[PPT], y[PPT];          // this thread's pixels
    bool inside[PPT];
    int width, height;
    int pixel_offset;
    float cx0, cy0;              // centre of the tile's first pixel
};

// Work item -> the CTA's pixels: a tile (in the queue's order) and, when the CTA covers a
// WT x WT work tile smaller than the TILE x TILE list tile, which of the tile's
// (TILE / WT)^2 work tiles; all of them walk the tile's whole list.
template <int TILE, int WT>
constexpr int work_tiles() {
    return (TILE / WT) * (TILE / WT);
}

template <int TILE, int WT, int PPT>
__device__ __forceinline__ TileInfo<PPT> tile_info(const RasterArgs& a, int item) {
    using L = Lay<WT, PPT>;
    constexpr int Q = work_tiles<TILE, WT>();
    TileInfo<PPT> ti;
    const int tile_item = item / Q, q = item % Q;
    const int local = a.tile_order ? (int)a.tile_order[tile_item] : tile_item;
    ti.g = a.tile_first + local;
    int vi = a.view_first;
    const int vend = a.view_first + a.num_views;
    while (vi + 1 < vend && a.views[vi + 1].tile_offset <= ti.g) vi++;
    const ViewDesc& vw = a.views[vi];
    const int lt = ti.g - vw.tile_offset;
    const int tx = lt % vw.tiles_x, ty = lt / vw.tiles_x;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int x0 = tx * TILE + (q % (TILE / WT)) * WT, y0 = ty * TILE + (q / (TILE / WT)) * WT;
#pragma unroll
    for (int p = 0; p < PPT; p++) {
        ti.x[p] = x0 + 8 * L::xg(w, p) + (lane & 7);
        ti.y[p] = y0 + 4 * L::yg(w, p) + (lane >> 3);
        ti.inside[p] = ti.x[p] < vw.width && ti.y[p] < vw.height;
    }
    ti.width = vw.width;
    ti.height = vw.height;
    ti.pixel_offset = vw.pixel_offset;
    ti.cx0 = (float)x0 + 0.5f;  // first pixel centre of the work tile
    ti.cy0 = (float)y0 + 0.5f;
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
constexpr float ALPHA_Q_BAND = 1e-4f;  // |q - log2(alpha_min)| below this: reference formula
constexpr float KAPPA_CULL_MAX = 256.f; // elongation above which culling uses the bounding square only
constexpr float KAPPA_EXACT = 32.f;     // elongation above which every pixel uses the reference expression
#ifndef BWD_GROUPS
#define BWD_GROUPS 2  // backward: 8 x 4 pixel groups evaluated together (1, 2 or 4)
#endif
#ifndef FWD_GROUPS
#define FWD_GROUPS 2  // forward: the same, in pixel pairs (2 or 4)
#endif

// Elongation of a splat's conic, kappa = A C / (A C - B^2) >= 1: the quadratic form's
// terms reach kappa times its value, so rounding errors in the exponent (and in the
// ellipse arithmetic) grow with it.
__device__ __forceinline__ float conic_kappa(float A, float B, float C) {
    const float ac = A * C;
    return ac / fmaxf(ac - B * B, ac * 1e-12f + 1e-30f);
}

// After the batch's copies landed, each staging thread derives for its splats:
// s_g1.w = the culling bound 2 ln(opacity / alpha_min) + slack (a pixel can reach
// alpha >= alpha_min only where the conic's quadratic form is below it);
// s_q = (-A/2, -B, -C/2) log2(e) and log2(opacity), so that alpha = 2^q with
// q = log2(op) + qa dx^2 + qb dx dy + qc dy^2; and s_c.w = the half-width of the band
// around log2(alpha_min) in which the reference expression decides: 1e-4 plus a bound
// on the rounding of q and of the reference's own exponent, which grows with the
// conic's elongation (for near-degenerate splats seen from close by, the terms of q are
// thousands of times q itself).  Above KAPPA_EXACT the rounding of the reference's own
// exponent shows in alpha's value, so such splats (about 1 % of the benchmark's list
// entries) get an unbounded band: every pixel takes alpha from the reference expression.
// s_c.w holds the band's lower end qlo; the band is symmetric about log2(alpha_min).
__device__ __forceinline__ void prepare_batch(int cnt, float4* s_g0, float4* s_g1, float4* s_q, float4* s_c,
                                              float log_amin, float qthr) {
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
        const float4 g0 = s_g0[t];
        const float4 g1 = s_g1[t];
        const float op = g1.y;
        const float kappa = conic_kappa(g0.z, g0.w, g1.x);
        const float lop = op > 0.f ? __log2f(op) : -1e30f;
        s_g1[t].w = op > 0.f ? 2.0f * (__logf(op) - log_amin) * (1.0f + kappa * 1.52587890625e-05f) + 1e-3f : -1.0f;
        s_q[t] = make_float4(-0.5f * LOG2E * g0.z, -LOG2E * g0.w, -0.5f * LOG2E * g1.x, lop);
        s_c[t].w = kappa > KAPPA_EXACT
                       ? -1e30f
                       : qthr - (ALPHA_Q_BAND + 7.62939453125e-06f * kappa * fmaxf(lop - qthr, 1.0f));  // 2^-17
    }
}

// The warp's groups (bit p = its p-th group) where splat (g0, g1) can give a pixel
// centre alpha >= alpha_min.  Per x band of 8 pixel centres the warp covers: the y-range
// of the ellipse A dx^2 + 2B dx dy + C dy^2 <= thr (thr = g1.w) over the band, clipped to
// the splat's bounding square |dx|, |dy| <= radius, against each of its groups' 4 pixel
// rows.  Over a band the ellipse's upper edge is concave and its lower edge convex in
// dx, so the range's ends sit at the stationary points dx = -/+ B sqrt(thr / (A det))
// clamped to the band.  Conservative: the slack covers the approximate instructions; the
// pixels' own tests decide.
template <int TILE, int PPT>
__device__ __forceinline__ uint32_t group_mask(const float4& g0, const float4& g1, float cx0, float cy0, int w) {
    using L = Lay<TILE, PPT>;
    const float thr = g1.w;
    if (!(thr > 0.f)) return 0u;
    const float u = g0.x, v = g0.y, A = g0.z, B = g0.w, C = g1.x, r = g1.z;
    const float bx0 = cx0 + 8.0f * (float)L::xg(w, 0) - u;  // first pixel centre of the warp's first band, from u
    const float by0 = cy0 + 4.0f * (float)L::yg(w, 0) - v;  // first pixel-centre row of its first group row, from v
    if (conic_kappa(A, B, C) > KAPPA_CULL_MAX) {
        // Near-degenerate conic: its ellipse arithmetic is not trusted, cull by the
        // bounding square |dx|, |dy| <= radius alone.
        uint32_t m = 0u;
#pragma unroll
        for (int hh = 0; hh < L::WX; hh++) {
            const float bx = bx0 + 8.0f * (float)hh;
            if (bx > r || bx + 7.0f < -r) continue;
#pragma unroll
            for (int i = 0; i < L::WY; i++) {
                const float y0 = by0 + 4.0f * (float)i;
                if (y0 <= r && y0 + 3.0f >= -r) m |= 1u << (hh * L::WY + i);
            }
        }
        return m;
    }
    const float det = fmaxf(A * C - B * B, 1e-30f);
    const float idet = rcp_approx(det);
    const float iC = rcp_approx(C);
    const float xr = sqrt_approx(thr * C * idet);                  // the ellipse's x half-extent
    const float sx = B * sqrt_approx(thr * idet * rcp_approx(A));  // stationary point of the lower edge
    const float slack = 1e-3f * (1.0f + r);
    uint32_t m = 0u;
#pragma unroll
    for (int hh = 0; hh < L::WX; hh++) {
        const float bx = bx0 + 8.0f * (float)hh;  // first pixel centre of the band, from u
        const float xl = fmaxf(fmaxf(bx, -r), -xr - slack);
        const float xh = fminf(fminf(bx + 7.0f, r), xr + slack);
        if (xl > xh) continue;
        const float du = fminf(fmaxf(-sx, xl), xh);  // maximiser of the upper edge
        const float dl = fminf(fmaxf(sx, xl), xh);   // minimiser of the lower edge
        const float hi = fminf((-B * du + sqrt_approx(fmaxf(C * thr - det * du * du, 0.f))) * iC + slack, r);
        const float lo = fmaxf((-B * dl - sqrt_approx(fmaxf(C * thr - det * dl * dl, 0.f))) * iC - slack, -r);
#pragma unroll
        for (int i = 0; i < L::WY; i++) {
            const float y0 = by0 + 4.0f * (float)i;  // first pixel-centre row of the group, from v
            if (y0 <= hi && y0 + 3.0f >= lo) m |= 1u << (hh * L::WY + i);
        }
    }
    return m;
}

// alpha of splat (g0, g1) at offset (dx, dy), or 0 when the pixel skips it:
// alphaAt (trainer/gpu.js:91-103), in the reference's own arithmetic.  Used where the
// log2-domain exponent lies within ALPHA_Q_BAND of the alpha_min threshold (a rare
// branch), so skip decisions match the reference's.  Explicit rounding intrinsics keep
// forward and backward bit-identical.
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

// The pieces of the alpha exponent that depend on one splat and one pixel column:
// log2(alpha) = a0 + dy (b0 + qc dy) with a0 = log2(op) + qa dx^2, b0 = qb dx (both
// duplicated for a pixel pair); and whether |dx| <= radius.
struct XTerm {
    float dx;
    float2 a0, b0;
    bool inb;
};

__device__ __forceinline__ XTerm xterm(const float4& q, float dx, float radius) {
    XTerm t;
    t.dx = dx;
    t.a0 = f2(__fmaf_rn(dx, __fmul_rn(q.x, dx), q.w));
    t.b0 = f2(__fmul_rn(q.y, dx));
    t.inb = fabsf(dx) <= radius;
    return t;
}

// The exponents of a pixel pair of one column (row offsets dy).
__device__ __forceinline__ float2 exponent2(const XTerm& xt, float2 qc, float2 dy) {
    return fma2(dy, fma2(qc, dy, xt.b0), xt.a0);
}

// alpha at one pixel from its exponent e and row offset dy, or 0 when the pixel skips
// the splat (live: the pixel still takes part and its column lies within the bounding
// square): 2^e by the fast exp2; where |e - log2(alpha_min)| < hw (the splat's band,
// ec = e - log2(alpha_min)) the reference expression decides.  One compare tests the
// band: it is symmetric about the threshold.  hit = alpha != 0.  Branch-free but for the
// band.
__device__ __forceinline__ float alpha_pix(float e, float ec, float dx, float dy, bool live, const float4& g0,
                                           const float4& g1, float amax, float amin, float hw, bool& hit) {
    const bool inb = live && fabsf(dy) <= g1.z;
    hit = inb && ec >= hw;
    float alpha = hit ? fminf(amax, ex2_approx(e)) : 0.f;
    if (inb && fabsf(ec) < hw) {
        alpha = alpha_band(g0, g1, dx, dy, amax, amin);
        hit = alpha != 0.f;
    }
    return alpha;
}

// Resident CTAs per SM the register allocation is sized for (fewer threads with more
// pixels each get more registers per thread).
// For 16 x 16 tiles; other tiles scale the count by the threads per CTA.
constexpr int fwd_min_ctas16(int ppt) { return ppt == 8 ? 20 : (ppt == 4 ? 12 : 4 * ppt); }
constexpr int bwd_min_ctas16(int ppt) { return ppt == 8 ? 16 : (ppt == 4 ? 10 : (ppt == 2 ? 7 : 4)); }
constexpr int scale_ctas(int c16, int tile) {
    return c16 * 256 / (tile * tile) < 1 ? 1 : (c16 * 256 / (tile * tile) > 32 ? 32 : c16 * 256 / (tile * tile));
}
constexpr int fwd_min_ctas(int tile, int ppt) { return scale_ctas(fwd_min_ctas16(ppt), tile); }
constexpr int bwd_min_ctas(int tile, int ppt) { return scale_ctas(bwd_min_ctas16(ppt), tile); }

template <int TILE, int WT, int BATCH, int PPT>
__global__ void __launch_bounds__(Lay<WT, PPT>::NT, fwd_min_ctas(WT, PPT)) raster_fwd_kernel(RasterArgs a) {
    using L = Lay<WT, PPT>;
    const int items = a.num_tiles * work_tiles<TILE, WT>();
    __shared__ __align__(16) float4 s_g0[2][BATCH];
    __shared__ __align__(16) float4 s_g1[2][BATCH];
    __shared__ __align__(16) float4 s_c[2][BATCH];
    __shared__ __align__(16) float4 s_q[2][BATCH];
    __shared__ int s_item;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const float log_amin = __logf(a.alpha_min);
    const float qthr = __log2f(a.alpha_min);
    int item = next_item(a.work_counter, &s_item, blockIdx.x);
    while (item < items) {
        const TileInfo<PPT> ti = tile_info<TILE, WT, PPT>(a, item);
        const uint2 rg = a.ranges[ti.g];
        const uint32_t start = rg.x, end = rg.y;
        // Pixel pairs (2i, 2i + 1) share an x band.  A pixel blends while T > t_min (the
        // reference stops once T <= 1e-4); pixels outside the view start at T = 0.
        constexpr int NP = PPT / 2;
        float pxf[L::WX];
        float2 pyf[NP], T[NP], cr[NP], cg[NP], cb[NP];
        uint32_t last[PPT];
#pragma unroll
        for (int b = 0; b < L::WX; b++) pxf[b] = (float)ti.x[b * L::WY] + 0.5f;  // the warp's x bands
        uint32_t gdone = 0u;  // warp-uniform: groups whose pixels have all stopped
#pragma unroll
        for (int i = 0; i < NP; i++) {
            pyf[i] = make_float2((float)ti.y[2 * i] + 0.5f, (float)ti.y[2 * i + 1] + 0.5f);
            T[i] = make_float2(ti.inside[2 * i] ? 1.0f : 0.f, ti.inside[2 * i + 1] ? 1.0f : 0.f);
            cr[i] = cg[i] = cb[i] = f2(0.f);
            last[2 * i] = last[2 * i + 1] = start;
            if (__all_sync(FULL_MASK, !ti.inside[2 * i])) gdone |= 1u << (2 * i);
            if (__all_sync(FULL_MASK, !ti.inside[2 * i + 1])) gdone |= 2u << (2 * i);
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
            prepare_batch(cnt, s_g0[buf], s_g1[buf], s_q[buf], s_c[buf], log_amin, qthr);
            __syncthreads();
            const float4* g0s = s_g0[buf];
            const float4* g1s = s_g1[buf];
            const float4* cs = s_c[buf];
            const float4* qs = s_q[buf];
            for (int gb = 0; gb < cnt && gdone != all_groups<PPT>(); gb += 32) {
                const int jl = gb + lane;
                const uint32_t gm = jl < cnt ? group_mask<WT, PPT>(g0s[jl], g1s[jl], ti.cx0, ti.cy0, w) : 0u;
                uint32_t live = __ballot_sync(FULL_MASK, (gm & ~gdone) != 0u);
                while (live) {
                    const int jj = __ffs(live) - 1;
                    live &= live - 1;
                    const int j = gb + jj;
                    const uint32_t m = __shfl_sync(FULL_MASK, gm, jj) & ~gdone;  // warp-uniform
                    const float4 g0 = g0s[j];
                    const float4 g1 = g1s[j];
                    const float4 q = qs[j];
                    const float4 c = cs[j];
                    const float hw = qthr - c.w;  // half-width of the splat's band
                    const uint32_t pos = b0 + (uint32_t)j + 1u;
                    const float2 qc = f2(q.z), ngy = f2(-g0.y);
                    const float2 cx = f2(c.x), cy = f2(c.y), cz = f2(c.z);
                    XTerm xt[L::WX];
#pragma unroll
                    for (int b = 0; b < L::WX; b++) xt[b] = xterm(q, pxf[b] - g0.x, g1.z);
                    // Groups go in blocks of FWD_GROUPS (pixel pairs of a block share a
                    // basic block, so their dependency chains interleave).
                    constexpr int GB = FWD_GROUPS < PPT ? FWD_GROUPS : PPT;
#pragma unroll
                    for (int gi = 0; gi < PPT / GB; gi++) {
                        if (!((m >> (GB * gi)) & ((1u << GB) - 1u))) continue;
#pragma unroll
                        for (int hh = 0; hh < GB / 2; hh++) {
                        const int i = gi * (GB / 2) + hh;
                        // Branch-free per lane: alpha = 0 leaves colour, T and last as they are
                        // (also for a pair member whose group the mask left out).
                        const XTerm& x = xt[(2 * i) / L::WY];
                        const float2 dy = add2(pyf[i], ngy);
                        const float2 e = exponent2(x, qc, dy);
                        const float2 ec = add2(e, f2(-qthr));
                        bool h0, h1;
                        const float a0 = alpha_pix(e.x, ec.x, x.dx, dy.x, x.inb && T[i].x > a.t_min, g0, g1,
                                                   a.alpha_max, a.alpha_min, hw, h0);
                        const float a1 = alpha_pix(e.y, ec.y, x.dx, dy.y, x.inb && T[i].y > a.t_min, g0, g1,
                                                   a.alpha_max, a.alpha_min, hw, h1);
                        const float2 alpha = make_float2(a0, a1);
                        const float2 wgt = mul2(alpha, T[i]);
                        cr[i] = fma2(cx, wgt, cr[i]);
                        cg[i] = fma2(cy, wgt, cg[i]);
                        cb[i] = fma2(cz, wgt, cb[i]);
                        T[i] = mul2(T[i], fma2(alpha, f2(-1.0f), f2(1.0f)));  // T (1 - alpha)
                        last[2 * i] = h0 ? pos : last[2 * i];
                        last[2 * i + 1] = h1 ? pos : last[2 * i + 1];
                        }
                    }
                }
#pragma unroll
                for (int i = 0; i < NP; i++) {
                    if (__all_sync(FULL_MASK, !(T[i].x > a.t_min))) gdone |= 1u << (2 * i);
                    if (__all_sync(FULL_MASK, !(T[i].y > a.t_min))) gdone |= 2u << (2 * i);
                }
            }
            buf ^= 1;
            // All pixels done: the rest of the list cannot change the tile.
            if (__syncthreads_count(gdone == all_groups<PPT>()) == (int)blockDim.x) {
                cp_async_wait<0>();
                break;
            }
        }
#pragma unroll
        for (int p = 0; p < PPT; p++) {
            if (!ti.inside[p]) continue;
            const size_t pix = (size_t)ti.pixel_offset + (size_t)ti.y[p] * ti.width + ti.x[p];
            const int i = p / 2;
            a.image[pix * 3 + 0] = p & 1 ? cr[i].y : cr[i].x;
            a.image[pix * 3 + 1] = p & 1 ? cg[i].y : cg[i].x;
            a.image[pix * 3 + 2] = p & 1 ? cb[i].y : cb[i].x;
            a.t_final[pix] = p & 1 ? T[i].y : T[i].x;
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

template <int TILE, int WT, int BATCH, int PPT>
__global__ void __launch_bounds__(Lay<WT, PPT>::NT, bwd_min_ctas(WT, PPT)) raster_bwd_kernel(RasterArgs a) {
    using L = Lay<WT, PPT>;
    const int items = a.num_tiles * work_tiles<TILE, WT>();
    __shared__ __align__(16) float4 s_g0[2][BATCH];
    __shared__ __align__(16) float4 s_g1[2][BATCH];
    __shared__ __align__(16) float4 s_c[2][BATCH];
    __shared__ __align__(16) float4 s_q[2][BATCH];
    __shared__ uint32_t s_pair[2][BATCH];
    __shared__ int s_item;
    __shared__ unsigned int s_end;
    __shared__ uint32_t s_gmax[L::NT / 32][PPT];  // per warp and group: the largest last
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const float log_amin = __logf(a.alpha_min);
    const float qthr = __log2f(a.alpha_min);
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
    while (item < items) {
        const TileInfo<PPT> ti = tile_info<TILE, WT, PPT>(a, item);
        const uint2 rg = a.ranges[ti.g];
        const uint32_t start = rg.x;
        // Pixel rows: p's centre is pyf0 + 4 (p % WY), exact in float (recomputed where
        // used rather than held in registers).
        const float pyf0 = (float)ti.y[0] + 0.5f;
        float pxf[L::WX], T[PPT], dlr[PPT], dlg[PPT], dlb[PPT], bd[PPT];
        uint32_t mylast[PPT];
#pragma unroll
        for (int b = 0; b < L::WX; b++) pxf[b] = (float)ti.x[b * L::WY] + 0.5f;  // the warp's x bands
        unsigned int wmax = start;
#pragma unroll
        for (int p = 0; p < PPT; p++) {
            T[p] = 0.f;
            dlr[p] = dlg[p] = dlb[p] = 0.f;
            bd[p] = 0.f;  // dL . (colour of the splats behind), "behind"
            mylast[p] = start;
            if (ti.inside[p]) {
                const size_t pix = (size_t)ti.pixel_offset + (size_t)ti.y[p] * ti.width + ti.x[p];
                T[p] = a.t_final[pix];
                mylast[p] = a.last[pix];
                dlr[p] = a.dl[pix * 3 + 0];
                dlg[p] = a.dl[pix * 3 + 1];
                dlb[p] = a.dl[pix * 3 + 2];
            }
            // Each group walks from the largest last of its pixels.
            unsigned int gm = mylast[p];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) gm = max(gm, __shfl_xor_sync(FULL_MASK, gm, o));
            if (lane == 0) s_gmax[w][p] = gm;
            wmax = max(wmax, gm);
        }
        if (threadIdx.x == 0) s_end = start;
        __syncthreads();
        // Tile end = largest last of its pixels (BACKWARD_SG, trainer/gpu.js:247-253).
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
            prepare_batch(cnt, s_g0[buf], s_g1[buf], s_q[buf], s_c[buf], log_amin, qthr);
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
                    uint32_t gm = 0u;
                    if (jl < cnt) {
                        const uint32_t kl = bend - 1 - (uint32_t)jl;
                        uint32_t act = 0u;  // groups with a pixel whose last is past this entry
#pragma unroll
                        for (int p = 0; p < PPT; p++) act |= kl < s_gmax[w][p] ? (1u << p) : 0u;
                        if (act) gm = group_mask<WT, PPT>(g0s[jl], g1s[jl], ti.cx0, ti.cy0, w) & act;
                    }
                    uint32_t live = __ballot_sync(FULL_MASK, gm != 0u);
                    while (live) {
                        const int jj = __ffs(live) - 1;
                        live &= live - 1;
                        const int j = gb + jj;
                        const uint32_t m = __shfl_sync(FULL_MASK, gm, jj);  // warp-uniform
                        const uint32_t k = bend - 1 - (uint32_t)j;
                        const float4 g0 = g0s[j];
                        const float4 g1 = g1s[j];
                        const float4 q = qs[j];
                        const float4 c = cs[j];
                        const float hw = qthr - c.w;  // half-width of the splat's band
                        XTerm xt[L::WX];
#pragma unroll
                        for (int b = 0; b < L::WX; b++) xt[b] = xterm(q, pxf[b] - g0.x, g1.z);
                        // Per pixel: colour terms and dP = dL/dpower, summed per x band as
                        // sum dP, sum dP dy, sum dP dy^2 (the band's pixels share dx); after
                        // the group loop the bands give the moments (sum dP, dP dx, dP dy,
                        // dP dx^2, dP dx dy, dP dy^2) from which the splat's conic and
                        // opacity make the gradients of (opacity logit, u, v, A, B, C) after
                        // the reduction.  Scalar arithmetic: pairing the pixels for the
                        // packed instructions costs more register moves than it saves here.
                        float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                        float s0[L::WX], sy[L::WX], syy[L::WX];
#pragma unroll
                        for (int b = 0; b < L::WX; b++) s0[b] = sy[b] = syy[b] = 0.f;
                        // Groups go in blocks of BWD_GROUPS (a block is evaluated when any
                        // of its groups is live; the others' own tests give alpha = 0), so
                        // the compiler can interleave the dependency chains of a block's
                        // pixels.
                        constexpr int GB = BWD_GROUPS < PPT ? BWD_GROUPS : PPT;
#pragma unroll
                        for (int gi = 0; gi < PPT / GB; gi++) {
                            if (!((m >> (GB * gi)) & ((1u << GB) - 1u))) continue;
#pragma unroll
                            for (int h = 0; h < GB; h++) {
                            const int p = GB * gi + h;
                            // Branch-free per lane: alpha = 0 adds zeros and leaves T
                            // (T / 1) and dL.behind as they are.
                            const int b = p / L::WY;
                            const XTerm& x = xt[b];
                            const float dy = (pyf0 + (float)(4 * (p % L::WY))) - g0.y;
                            const float e = __fmaf_rn(dy, __fmaf_rn(q.z, dy, x.b0.x), x.a0.x);
                            bool hit;
                            const float alpha = alpha_pix(e, e - qthr, x.dx, dy, x.inb && k < mylast[p], g0, g1,
                                                          a.alpha_max, a.alpha_min, hw, hit);
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
                            const float dPy = dP * dy;
                            s0[b] += dP;
                            sy[b] += dPy;
                            syy[b] += dPy * dy;
                            }
                        }
                        float v8 = 0.f;
#pragma unroll
                        for (int b = 0; b < L::WX; b++) {
                            const float dx = xt[b].dx, tx = s0[b] * dx;
                            v[3] += s0[b];
                            v[4] += tx;
                            v[5] += sy[b];
                            v[6] += tx * dx;
                            v[7] += sy[b] * dx;
                            v8 += syy[b];
                        }
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
            buf ^= 1;
            bend = bstart;
            __syncthreads();
        }
        if (!a.work_counter) break;
        item = next_item(a.work_counter, &s_item, 0);
    }
}

// Variant = (list tile edge, work tile edge, shared-memory batch, pixels per thread);
// the autotuner picks one.
template <int TILE, int WT, int BATCH, int PPT>
static void fwd_launch(const RasterArgs& a, int ctas, cudaStream_t s) {
    if (!a.work_counter) ctas = a.num_tiles * work_tiles<TILE, WT>();
    raster_fwd_kernel<TILE, WT, BATCH, PPT><<<ctas, Lay<WT, PPT>::NT, 0, s>>>(a);
}
template <int TILE, int WT, int BATCH, int PPT>
static void bwd_launch(const RasterArgs& a, int ctas, cudaStream_t s) {
    if (!a.work_counter) ctas = a.num_tiles * work_tiles<TILE, WT>();
    raster_bwd_kernel<TILE, WT, BATCH, PPT><<<ctas, Lay<WT, PPT>::NT, 0, s>>>(a);
}

#define RASTER_BATCHES(FN, T, W, batch, P, ...)                 \
    do {                                                        \
        switch (batch) {                                        \
            case 32: FN<T, W, 32, P>(__VA_ARGS__); break;       \
            case 64: FN<T, W, 64, P>(__VA_ARGS__); break;       \
            case 128: FN<T, W, 128, P>(__VA_ARGS__); break;     \
            default: FN<T, W, 256, P>(__VA_ARGS__); break;      \
        }                                                       \
    } while (0)

#define RASTER_PPTS(FN, T, W, batch, ppt, ...)                                   \
    do {                                                                         \
        if ((ppt) == 8) RASTER_BATCHES(FN, T, W, batch, 8, __VA_ARGS__);         \
        else if ((ppt) == 4) RASTER_BATCHES(FN, T, W, batch, 4, __VA_ARGS__);    \
        else RASTER_BATCHES(FN, T, W, batch, 2, __VA_ARGS__);                    \
    } while (0)

// The (list tile, work tile, pixels per thread) variants that exist: 8 x 8 tiles with
// 2 pixels per thread; 16 x 16 tiles with 2, 4 or 8; 32 x 32 tiles with work tiles of
// 32 x 32 or 16 x 16 and 2, 4 or 8; 64 x 64 tiles with 16 x 16 work tiles and 2, 4 or 8
// (raster_variant_ok).
#define RASTER_SWITCH(FN, tile, wt, batch, ppt, ...)                                       \
    do {                                                                                   \
        if ((tile) == 8) {                                                                 \
            RASTER_BATCHES(FN, 8, 8, batch, 2, __VA_ARGS__);                               \
        } else if ((tile) == 32) {                                                         \
            if ((wt) == 16) RASTER_PPTS(FN, 32, 16, batch, ppt, __VA_ARGS__);              \
            else RASTER_PPTS(FN, 32, 32, batch, ppt, __VA_ARGS__);                         \
        } else if ((tile) == 64) {                                                         \
            RASTER_PPTS(FN, 64, 16, batch, ppt, __VA_ARGS__);                              \
        } else {                                                                           \
            RASTER_PPTS(FN, 16, 16, batch, ppt, __VA_ARGS__);                              \
        }                                                                                  \
    } while (0)

bool raster_variant_ok(int tile, int wt, int ppt) {
    if (tile == 8) return wt == 8 && ppt == 2;
    if (tile == 16) return wt == 16 && (ppt == 2 || ppt == 4 || ppt == 8);
    if (tile == 32) return (wt == 32 || wt == 16) && (ppt == 2 || ppt == 4 || ppt == 8);
    if (tile == 64) return wt == 16 && (ppt == 2 || ppt == 4 || ppt == 8);
    return false;
}

void launch_raster_fwd(const RasterArgs& a, int tile, int wt, int batch, int ppt, int persistent_ctas,
                       cudaStream_t s) {
    if (a.num_tiles <= 0 || (a.work_counter && persistent_ctas <= 0)) return;
    RASTER_SWITCH(fwd_launch, tile, wt, batch, ppt, a, persistent_ctas, s);
}

void launch_raster_bwd(const RasterArgs& a, int tile, int wt, int batch, int ppt, int persistent_ctas,
                       cudaStream_t s) {
    if (a.num_tiles <= 0 || (a.work_counter && persistent_ctas <= 0)) return;
    RASTER_SWITCH(bwd_launch, tile, wt, batch, ppt, a, persistent_ctas, s);
}

template <int TILE, int WT, int BATCH, int PPT>
static void occ(int* n, bool backward) {
    if (backward)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, raster_bwd_kernel<TILE, WT, BATCH, PPT>, Lay<WT, PPT>::NT, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, raster_fwd_kernel<TILE, WT, BATCH, PPT>, Lay<WT, PPT>::NT, 0);
}

int raster_max_ctas_per_sm(int tile, int wt, int batch, int ppt, bool backward) {
    int n = 0;
    RASTER_SWITCH(occ, tile, wt, batch, ppt, &n, backward);
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
        const int tile = vw.tile_offset + (y / vw.tile) * vw.tiles_x + x / vw.tile;
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
