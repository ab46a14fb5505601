// Initialisation from a point cloud: neighbourSizes (trainer/neighbours.js:13-53) and
// initFromPoints (trainer/gpu.js:507-521) on the device.
//
// neighbourSizes: points are bucketed in 0.1 m cubes; each point's size is the root mean
// square distance to its (up to) 3 nearest other points among the 27 cubes around its
// own, clamped to [min, max], or `fallback` when none is there.  The reference keys a
// JavaScript Map by ((i + 32768) 65536 + (j + 32768)) 65536 + (k + 32768); here the same
// 64-bit key goes into an open-addressing hash table built with atomicCAS, whose cells
// then receive their points through a count / scan / scatter, and one thread per point
// walks its 27 cubes.  The three smallest squared distances and their mean are order-
// independent, so the bucket order does not matter; distances use double arithmetic
// with explicit rounding (no fused multiply-add), as JavaScript evaluates them.
#include <algorithm>

#include "internal.h"

namespace gs {

constexpr double NB_CELL = 0.1;
constexpr unsigned long long NB_EMPTY = 0xffffffffffffffffull;

__device__ __forceinline__ long long nb_cell(float v) { return (long long)floor((double)v / NB_CELL); }

// The reference's cube key, in exact integer arithmetic (JavaScript doubles hold it
// exactly for cubes within reach).
__device__ __forceinline__ unsigned long long nb_key(long long i, long long j, long long k) {
    return (unsigned long long)(((i + 32768) * 65536 + (j + 32768)) * 65536 + (k + 32768));
}

__device__ __forceinline__ unsigned nb_hash(unsigned long long k, unsigned mask) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    return (unsigned)k & mask;
}

// Slot of key in the table (inserting it when absent); cell ids are given out densely.
__device__ unsigned nb_insert(unsigned long long* keys, unsigned* ids, unsigned mask, unsigned long long key,
                              unsigned* next_id) {
    unsigned h = nb_hash(key, mask);
    for (unsigned probe = 0; probe <= mask; probe++, h = (h + 1) & mask) {
        const unsigned long long prev = atomicCAS(keys + h, NB_EMPTY, key);
        if (prev == NB_EMPTY) {
            ids[h] = atomicAdd(next_id, 1u);
            return h;
        }
        if (prev == key) return h;
    }
    return 0xffffffffu;  // table full (sized at twice the points: does not happen)
}

__device__ unsigned nb_find(const unsigned long long* keys, unsigned mask, unsigned long long key) {
    unsigned h = nb_hash(key, mask);
    for (unsigned probe = 0; probe <= mask; probe++, h = (h + 1) & mask) {
        const unsigned long long k = keys[h];
        if (k == key) return h;
        if (k == NB_EMPTY) return 0xffffffffu;
    }
    return 0xffffffffu;
}

__global__ void nb_insert_kernel(NeighbourArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.count) return;
    const unsigned long long key =
        nb_key(nb_cell(a.xyz[p * 3]), nb_cell(a.xyz[p * 3 + 1]), nb_cell(a.xyz[p * 3 + 2]));
    a.point_slot[p] = nb_insert(a.keys, a.ids, a.mask, key, a.counters);
}

// Points per cell (ids are written by the inserting thread; read them after the launch).
__global__ void nb_count_kernel(NeighbourArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.count) return;
    const unsigned slot = a.point_slot[p];
    if (slot != 0xffffffffu) atomicAdd(a.cell_count + a.ids[slot], 1u);
}

// Exclusive scan of the cell counts (one block, cells <= count).
__global__ void __launch_bounds__(1024) nb_scan_kernel(NeighbourArgs a) {
    __shared__ unsigned s_tmp[32];
    const unsigned cells = a.counters[0];
    unsigned carry = 0;
    for (unsigned b = 0; b < cells; b += 1024) {
        const unsigned idx = b + threadIdx.x;
        const unsigned v = idx < cells ? a.cell_count[idx] : 0u;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        unsigned x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_tmp[warp] = x;
        __syncthreads();
        if (warp == 0) {
            unsigned t = s_tmp[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            s_tmp[lane] = t;
        }
        __syncthreads();
        const unsigned excl = carry + (warp > 0 ? s_tmp[warp - 1] : 0u) + x - v;
        const unsigned tot = s_tmp[31];
        __syncthreads();
        if (idx < cells) {
            a.cell_start[idx] = excl;
            a.cell_cursor[idx] = excl;
        }
        carry += tot;
    }
}

__global__ void nb_scatter_kernel(NeighbourArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.count) return;
    const unsigned slot = a.point_slot[p];
    if (slot == 0xffffffffu) return;
    const unsigned at = atomicAdd(a.cell_cursor + a.ids[slot], 1u);
    a.cell_points[at] = (unsigned)p;
}

__global__ void nb_size_kernel(NeighbourArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.count) return;
    const double x = a.xyz[p * 3], y = a.xyz[p * 3 + 1], z = a.xyz[p * 3 + 2];
    const long long ci = nb_cell(a.xyz[p * 3]), cj = nb_cell(a.xyz[p * 3 + 1]), ck = nb_cell(a.xyz[p * 3 + 2]);
    double b0 = INFINITY, b1 = INFINITY, b2 = INFINITY;
    for (int di = -1; di <= 1; di++)
        for (int dj = -1; dj <= 1; dj++)
            for (int dk = -1; dk <= 1; dk++) {
                const unsigned h = nb_find(a.keys, a.mask, nb_key(ci + di, cj + dj, ck + dk));
                if (h == 0xffffffffu) continue;
                const unsigned cell = a.ids[h];
                const unsigned s = a.cell_start[cell], e = s + a.cell_count[cell];
                for (unsigned t = s; t < e; t++) {
                    const unsigned q = a.cell_points[t];
                    if (q == (unsigned)p) continue;
                    const double dx = __dsub_rn((double)a.xyz[q * 3], x);
                    const double dy = __dsub_rn((double)a.xyz[q * 3 + 1], y);
                    const double dz = __dsub_rn((double)a.xyz[q * 3 + 2], z);
                    const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                    if (d2 >= b2) continue;  // as written in the reference (a NaN falls through)
                    if (d2 < b0) {
                        b2 = b1;
                        b1 = b0;
                        b0 = d2;
                    } else if (d2 < b1) {
                        b2 = b1;
                        b1 = d2;
                    } else {
                        b2 = d2;
                    }
                }
            }
    int found = 0;
    double sum = 0.0;
    if (isfinite(b0)) { sum = __dadd_rn(sum, b0); found++; }
    if (isfinite(b1)) { sum = __dadd_rn(sum, b1); found++; }
    if (isfinite(b2)) { sum = __dadd_rn(sum, b2); found++; }
    const double size = found ? __dsqrt_rn(__ddiv_rn(sum, (double)found)) : a.fallback;
    a.sizes[p] = (float)fmin(a.max_size, fmax(a.min_size, size));
}

// initFromPoints: one Gaussian per point, log-size on all axes, identity rotation,
// opacity 0.1, the point's colour (trainer/gpu.js:507-521).
__global__ void init_planes_kernel(const float* xyz, const float* rgb, const float* sizes, float fixed_size, int count,
                                   int n_pad, int planes, float* params) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pad) return;
    const size_t np = (size_t)n_pad;
    if (i >= count) {
        for (int k = 0; k < planes; k++) params[k * np + i] = k == 6 ? 1.f : 0.f;
        return;
    }
    const double s = log((double)(sizes ? sizes[i] : fixed_size));
    const float ls = (float)s;
    for (int k = 0; k < 3; k++) params[k * np + i] = xyz[i * 3 + k];
    for (int k = 0; k < 3; k++) params[(3 + k) * np + i] = ls;
    params[6 * np + i] = 1.f;
    params[7 * np + i] = 0.f;
    params[8 * np + i] = 0.f;
    params[9 * np + i] = 0.f;
    params[10 * np + i] = (float)log(0.1 / (1.0 - 0.1));
    for (int k = 0; k < 3; k++) params[(11 + k) * np + i] = rgb[i * 3 + k];
    for (int k = 14; k < planes; k++) params[k * np + i] = 0.f;
}

void launch_neighbour_sizes(const NeighbourArgs& a, cudaStream_t s) {
    const int blocks = (a.count + 255) / 256;
    if (blocks == 0) return;
    nb_insert_kernel<<<blocks, 256, 0, s>>>(a);
    nb_count_kernel<<<blocks, 256, 0, s>>>(a);
    nb_scan_kernel<<<1, 1024, 0, s>>>(a);
    nb_scatter_kernel<<<blocks, 256, 0, s>>>(a);
    nb_size_kernel<<<blocks, 256, 0, s>>>(a);
}

void launch_init_planes(const float* xyz, const float* rgb, const float* sizes, float fixed_size, int count, int n_pad,
                        int planes, float* params, cudaStream_t s) {
    const int blocks = (n_pad + 255) / 256;
    if (blocks > 0) init_planes_kernel<<<blocks, 256, 0, s>>>(xyz, rgb, sizes, fixed_size, count, n_pad, planes, params);
}

}  // namespace gs

// ---- photo selection (trainer/sharpness.js:15-31, trainer/dataset.js:45) ---------------------
namespace gs {

// Grey bytes of RGB bytes: (77 R + 150 G + 29 B) >> 8, as dataset.js:45 does.
__global__ void grey_kernel(const uint8_t* __restrict__ rgb, size_t pixels, uint8_t* __restrict__ grey) {
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pixels) return;
    grey[p] = (uint8_t)((rgb[p * 3] * 77 + rgb[p * 3 + 1] * 150 + rgb[p * 3 + 2] * 29) >> 8);
}

// Per image (blockIdx.y): sums of the 4-neighbour Laplacian and of its square over the
// interior pixels, in exact integers.
__global__ void laplacian_sums_kernel(const uint8_t* __restrict__ grey, int width, int height,
                                      long long* __restrict__ sums) {
    const uint8_t* g = grey + (size_t)blockIdx.y * width * height;
    long long s = 0, s2 = 0;
    const int inner_w = width - 2, inner = inner_w > 0 && height > 2 ? inner_w * (height - 2) : 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < inner; t += gridDim.x * blockDim.x) {
        const int x = 1 + t % inner_w, y = 1 + t / inner_w;
        const int i = y * width + x;
        const int lap = (int)g[i - 1] + g[i + 1] + g[i - width] + g[i + width] - 4 * (int)g[i];
        s += lap;
        s2 += (long long)lap * lap;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(sums + 2 * blockIdx.y), (unsigned long long)s);
        atomicAdd(reinterpret_cast<unsigned long long*>(sums + 2 * blockIdx.y + 1), (unsigned long long)s2);
    }
}

void launch_grey(const uint8_t* rgb, size_t pixels, uint8_t* grey, cudaStream_t s) {
    if (pixels) grey_kernel<<<(unsigned)((pixels + 255) / 256), 256, 0, s>>>(rgb, pixels, grey);
}

void launch_laplacian_sums(const uint8_t* grey, int count, int width, int height, long long* sums, cudaStream_t s) {
    if (count <= 0) return;
    const int inner = (width - 2) * (height - 2);
    const int blocks = inner > 0 ? std::min(64, (inner + 255) / 256) : 1;
    laplacian_sums_kernel<<<dim3(blocks, count), 256, 0, s>>>(grey, width, height, sums);
}

}  // namespace gs
