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

struct TileInfo {
    int g;               // global tile id
    int x, y;            // this thread's pixel
    int width, height;
    int pixel_offset;
    bool inside;
};

__device__ __forceinline__ TileInfo tile_info(const RasterArgs& a, int item) {
    TileInfo ti;
    const int local = a.tile_order ? (int)a.tile_order[item] : item;
    ti.g = a.tile_first + local;
    int vi = a.view_first;
    const int vend = a.view_first + a.num_views;
    while (vi + 1 < vend && a.views[vi + 1].tile_offset <= ti.g) vi++;
    const ViewDesc& vw = a.views[vi];
    const int lt = ti.g - vw.tile_offset;
    const int tx = lt % vw.tiles_x, ty = lt / vw.tiles_x;
    ti.x = tx * GS_TILE + (threadIdx.x & (GS_TILE - 1));
    ti.y = ty * GS_TILE + (threadIdx.x / GS_TILE);
    ti.width = vw.width;
    ti.height = vw.height;
    ti.pixel_offset = vw.pixel_offset;
    ti.inside = ti.x < vw.width && ti.y < vw.height;
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

template <int BATCH>
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

template <int BATCH>
__global__ void __launch_bounds__(256) raster_fwd_kernel(RasterArgs a) {
    __shared__ __align__(16) float4 s_g0[2][BATCH];
    __shared__ __align__(16) float4 s_g1[2][BATCH];
    __shared__ __align__(16) float4 s_c[2][BATCH];
    __shared__ int s_item;
    int item = next_item(a.work_counter, &s_item, blockIdx.x);
    while (item < a.num_tiles) {
        const TileInfo ti = tile_info(a, item);
        const uint2 rg = a.ranges[ti.g];
        const uint32_t start = rg.x, end = rg.y;
        const float pxf = (float)ti.x + 0.5f, pyf = (float)ti.y + 0.5f;
        float T = 1.0f, cr = 0.f, cg = 0.f, cb = 0.f;
        uint32_t last = start;
        bool done = !ti.inside;
        int buf = 0;
        if (start < end) stage_batch<BATCH>(a, start, min((uint32_t)BATCH, end - start), false, s_g0[0], s_g1[0], s_c[0], nullptr);
        for (uint32_t b0 = start; b0 < end; b0 += BATCH) {
            const int cnt = (int)min((uint32_t)BATCH, end - b0);
            const uint32_t nb = b0 + BATCH;
            if (nb < end) {
                stage_batch<BATCH>(a, nb, min((uint32_t)BATCH, end - nb), false, s_g0[buf ^ 1], s_g1[buf ^ 1],
                                   s_c[buf ^ 1], nullptr);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            if (!done) {
                const float4* g0s = s_g0[buf];
                const float4* g1s = s_g1[buf];
                const float4* cs = s_c[buf];
                for (int j = 0; j < cnt; j++) {
                    const float4 g0 = g0s[j];
                    const float4 g1 = g1s[j];
                    const float dx = pxf - g0.x, dy = pyf - g0.y;
                    if (fabsf(dx) > g1.z || fabsf(dy) > g1.z) continue;
                    const float power = -0.5f * (g0.z * dx * dx + g1.x * dy * dy) - g0.w * dx * dy;
                    if (power > 0.0f) continue;
                    const float alpha = fminf(a.alpha_max, g1.y * expf(power));
                    if (alpha < a.alpha_min) continue;
                    const float4 c = cs[j];
                    cr += c.x * alpha * T;
                    cg += c.y * alpha * T;
                    cb += c.z * alpha * T;
                    T *= 1.0f - alpha;
                    last = b0 + (uint32_t)j + 1u;
                    if (T <= a.t_min) {
                        done = true;
                        break;
                    }
                }
            }
            buf ^= 1;
            // All pixels done: the rest of the list cannot change the tile.
            if (__syncthreads_count(done) == (int)blockDim.x) {
                cp_async_wait<0>();
                break;
            }
        }
        if (ti.inside) {
            const size_t pix = (size_t)ti.pixel_offset + (size_t)ti.y * ti.width + ti.x;
            a.image[pix * 3 + 0] = cr;
            a.image[pix * 3 + 1] = cg;
            a.image[pix * 3 + 2] = cb;
            a.t_final[pix] = T;
            a.last[pix] = last;
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

template <int BATCH>
__global__ void __launch_bounds__(256) raster_bwd_kernel(RasterArgs a) {
    __shared__ __align__(16) float4 s_g0[2][BATCH];
    __shared__ __align__(16) float4 s_g1[2][BATCH];
    __shared__ __align__(16) float4 s_c[2][BATCH];
    __shared__ uint32_t s_pair[2][BATCH];
    __shared__ int s_item;
    __shared__ unsigned int s_end;
    const int lane = threadIdx.x & 31;
    float* sg8f = reinterpret_cast<float*>(a.sg8);
    int item = next_item(a.work_counter, &s_item, blockIdx.x);
    while (item < a.num_tiles) {
        const TileInfo ti = tile_info(a, item);
        const uint2 rg = a.ranges[ti.g];
        const uint32_t start = rg.x;
        const float pxf = (float)ti.x + 0.5f, pyf = (float)ti.y + 0.5f;
        float T = 0.f, dlr = 0.f, dlg = 0.f, dlb = 0.f;
        uint32_t mylast = start;
        if (ti.inside) {
            const size_t pix = (size_t)ti.pixel_offset + (size_t)ti.y * ti.width + ti.x;
            T = a.t_final[pix];
            mylast = a.last[pix];
            dlr = a.dl[pix * 3 + 0];
            dlg = a.dl[pix * 3 + 1];
            dlb = a.dl[pix * 3 + 2];
        }
        if (threadIdx.x == 0) s_end = start;
        __syncthreads();
        // Tile end = largest last of its pixels (BACKWARD_SG, trainer/gpu.js:247-253).
        unsigned int wmax = mylast;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) wmax = max(wmax, __shfl_xor_sync(FULL_MASK, wmax, o));
        if (lane == 0) atomicMax(&s_end, wmax);
        __syncthreads();
        const uint32_t end = s_end;
        float br = 0.f, bg = 0.f, bb = 0.f;  // colour of the splats behind, "behind"
        int buf = 0;
        if (end > start)
            stage_batch<BATCH>(a, end, min((uint32_t)BATCH, end - start), true, s_g0[0], s_g1[0], s_c[0], s_pair[0]);
        for (uint32_t bend = end; bend > start;) {
            const uint32_t bstart = (bend - start > (uint32_t)BATCH) ? bend - BATCH : start;
            const int cnt = (int)(bend - bstart);
            if (bstart > start) {
                stage_batch<BATCH>(a, bstart, min((uint32_t)BATCH, bstart - start), true, s_g0[buf ^ 1],
                                   s_g1[buf ^ 1], s_c[buf ^ 1], s_pair[buf ^ 1]);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            const float4* g0s = s_g0[buf];
            const float4* g1s = s_g1[buf];
            const float4* cs = s_c[buf];
            const uint32_t* ps = s_pair[buf];
            // Warp-uniform skip: no pixel of this warp reaches this batch.
            const bool warp_active = __any_sync(FULL_MASK, ti.inside && bstart < mylast);
            if (warp_active) {
                for (int j = 0; j < cnt; j++) {
                    const uint32_t k = bend - 1 - (uint32_t)j;
                    float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                    float v8 = 0.f;
                    bool contrib = false;
                    if (ti.inside && k < mylast) {
                        const float4 g0 = g0s[j];
                        const float4 g1 = g1s[j];
                        const float dx = pxf - g0.x, dy = pyf - g0.y;
                        if (fabsf(dx) <= g1.z && fabsf(dy) <= g1.z) {
                            const float power = -0.5f * (g0.z * dx * dx + g1.x * dy * dy) - g0.w * dx * dy;
                            if (power <= 0.0f) {
                                const float alpha = fminf(a.alpha_max, g1.y * expf(power));
                                if (alpha >= a.alpha_min) {
                                    contrib = true;
                                    const float4 c = cs[j];
                                    const float oma = 1.0f - alpha;
                                    const float Tk = T / oma;
                                    v[0] = dlr * alpha * Tk;
                                    v[1] = dlg * alpha * Tk;
                                    v[2] = dlb * alpha * Tk;
                                    const float dA = dlr * (Tk * c.x - br / oma) + dlg * (Tk * c.y - bg / oma) +
                                                     dlb * (Tk * c.z - bb / oma);
                                    br += c.x * alpha * Tk;
                                    bg += c.y * alpha * Tk;
                                    bb += c.z * alpha * Tk;
                                    T = Tk;
                                    if (alpha < a.alpha_max) {
                                        const float op = g1.y;
                                        v[3] = dA * (alpha / op) * op * (1.0f - op);
                                        const float dP = dA * alpha;
                                        v[4] = dP * (g0.z * dx + g0.w * dy);
                                        v[5] = dP * (g1.x * dy + g0.w * dx);
                                        v[6] = dP * -0.5f * dx * dx;
                                        v[7] = dP * -dx * dy;
                                        v8 = dP * -0.5f * dy * dy;
                                    }
                                }
                            }
                        }
                    }
                    if (__any_sync(FULL_MASK, contrib)) {
                        const float s = warp_sum8_transposed(v);
                        float s8 = v8;
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) s8 += __shfl_xor_sync(FULL_MASK, s8, o);
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

template <int BATCH>
static void fwd_dispatch(const RasterArgs& a, int ctas, cudaStream_t s) {
    raster_fwd_kernel<BATCH><<<ctas, 256, 0, s>>>(a);
}
template <int BATCH>
static void bwd_dispatch(const RasterArgs& a, int ctas, cudaStream_t s) {
    raster_bwd_kernel<BATCH><<<ctas, 256, 0, s>>>(a);
}

void launch_raster_fwd(const RasterArgs& a, int batch, int persistent_ctas, cudaStream_t s) {
    const int ctas = a.work_counter ? persistent_ctas : a.num_tiles;
    if (ctas <= 0 || a.num_tiles <= 0) return;
    switch (batch) {
        case 64: fwd_dispatch<64>(a, ctas, s); break;
        case 128: fwd_dispatch<128>(a, ctas, s); break;
        default: fwd_dispatch<256>(a, ctas, s); break;
    }
}

void launch_raster_bwd(const RasterArgs& a, int batch, int persistent_ctas, cudaStream_t s) {
    const int ctas = a.work_counter ? persistent_ctas : a.num_tiles;
    if (ctas <= 0 || a.num_tiles <= 0) return;
    switch (batch) {
        case 64: bwd_dispatch<64>(a, ctas, s); break;
        case 128: bwd_dispatch<128>(a, ctas, s); break;
        default: bwd_dispatch<256>(a, ctas, s); break;
    }
}

int raster_max_ctas_per_sm(int batch, bool backward) {
    int n = 0;
    cudaError_t e;
    if (!backward) {
        switch (batch) {
            case 64: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, raster_fwd_kernel<64>, 256, 0); break;
            case 128: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, raster_fwd_kernel<128>, 256, 0); break;
            default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, raster_fwd_kernel<256>, 256, 0); break;
        }
    } else {
        switch (batch) {
            case 64: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, raster_bwd_kernel<64>, 256, 0); break;
            case 128: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, raster_bwd_kernel<128>, 256, 0); break;
            default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, raster_bwd_kernel<256>, 256, 0); break;
        }
    }
    if (e != cudaSuccess || n < 1) n = 1;
    return n;
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

}  // namespace gs
