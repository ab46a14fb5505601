// Densification on the device: the gradient statistics of STATS (trainer/gpu.js:484-497),
// densify() (:575-599) and the opacity reset of trainScene (:902-903, :944).
//
// Statistics: every training step adds, per Gaussian, |(dL/du, dL/dv)| of each view it
// projects into and the number of such views (the projection counts the views, the
// projection backward adds the norms).  They land in step-local planes first and are
// committed by stats_commit only when the step's update was applied, so a step redone
// after an instance overflow is counted once.
//
// densify(): in index order, a Gaussian is dropped when sigmoid(opacity logit) <
// min_opacity or its largest scale exceeds max_size; kept as it is when its average
// gradient norm (sum / count, 0 without views) is below the threshold or no room is
// left; otherwise cloned (largest scale <= size_threshold: itself and a copy) or split
// (two copies, each mean moved by (u - 0.5) exp(logScale) per axis with u uniform in
// [0, 1), log-scales lowered by ln 1.6).  Each clone or split takes one unit of room =
// max_count - n.  The sequential room rule becomes a scan: with p = Gaussians kept or
// densified before i and c = densification candidates before i, the outputs of i start
// at p + min(c, room).  Decisions and the new values are computed in double precision
// from the float parameters, as the reference's JavaScript does, and rounded to float.
// The reference draws u with Math.random(); here u is SplitMix64 of (seed, index, copy,
// axis), so a run is reproducible and the CPU restatement gives the same bits.
#include "internal.h"

namespace gs {

constexpr int DN_THREADS = 256;

__global__ void stats_commit_kernel(float* __restrict__ stats, const float* __restrict__ step, int n_pad,
                                    const DevStatus* status, const float* skip) {
    if (skip ? (*skip > 0.f) : (status->overflow != 0u || status->sort_timeout != 0u)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * n_pad) return;
    const float v = step[i];
    if (v != 0.f) stats[i] += v;
}

void launch_stats_commit(float* stats, const float* step, int n_pad, const DevStatus* status, const float* skip,
                         cudaStream_t s) {
    const int blocks = (2 * n_pad + DN_THREADS - 1) / DN_THREADS;
    if (blocks > 0) stats_commit_kernel<<<blocks, DN_THREADS, 0, s>>>(stats, step, n_pad, status, skip);
}

// ---- densify ---------------------------------------------------------------------------
__host__ __device__ inline uint64_t dn_splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Uniform double in [0, 1) for (Gaussian i, copy k, axis j).
__host__ __device__ inline double dn_uniform(uint64_t seed, uint64_t i, int k, int j) {
    const uint64_t z = dn_splitmix64(dn_splitmix64(seed) ^ ((i * 8ull + (uint64_t)(k * 4 + j)) * 0xD1B54A32D192ED03ull));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// 0 = dropped, 1 = kept, 2 = candidate (clone or split when there is room).
__device__ __forceinline__ int dn_classify(const DensifyArgs& a, int i, double* size_out) {
    const size_t np = (size_t)a.n_pad;
    const double ol = (double)a.params[10 * np + i];
    const double op = 1.0 / (1.0 + exp(-ol));
    if (op < a.min_opacity) return 0;
    // Math.max semantics: NaN if any scale is NaN.
    const double e0 = exp((double)a.params[3 * np + i]), e1 = exp((double)a.params[4 * np + i]),
                 e2 = exp((double)a.params[5 * np + i]);
    const double size = (isnan(e0) || isnan(e1) || isnan(e2)) ? (double)NAN : fmax(fmax(e0, e1), e2);
    if (size_out) *size_out = size;
    if (size > a.max_size) return 0;
    // A zero or NaN count is falsy in the reference: average 0.
    const float cnt = a.stats[np + i];
    const double avg = (cnt != 0.f && !isnan(cnt)) ? (double)a.stats[i] / (double)cnt : 0.0;
    if (avg < a.grad_threshold) return 1;
    return 2;
}

template <int NT>
__device__ __forceinline__ uint2 dn_block_excl_scan(uint2 v, uint2* s_tmp, uint2& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = NT / 32;
    uint2 x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned yx = __shfl_up_sync(0xffffffffu, x.x, o), yy = __shfl_up_sync(0xffffffffu, x.y, o);
        if (lane >= o) {
            x.x += yx;
            x.y += yy;
        }
    }
    if (lane == 31) s_tmp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint2 t = lane < NW ? s_tmp[lane] : make_uint2(0u, 0u);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned yx = __shfl_up_sync(0xffffffffu, t.x, o), yy = __shfl_up_sync(0xffffffffu, t.y, o);
            if (lane >= o) {
                t.x += yx;
                t.y += yy;
            }
        }
        if (lane < NW) s_tmp[lane] = t;
    }
    __syncthreads();
    const uint2 prefix = warp > 0 ? s_tmp[warp - 1] : make_uint2(0u, 0u);
    total = s_tmp[NW - 1];
    __syncthreads();
    return make_uint2(prefix.x + x.x - v.x, prefix.y + x.y - v.y);
}

// Per block: (Gaussians not dropped, candidates).
__global__ void __launch_bounds__(DN_THREADS) dn_count_kernel(DensifyArgs a) {
    __shared__ uint2 s_tmp[32];
    const int i = blockIdx.x * DN_THREADS + threadIdx.x;
    uint2 v = make_uint2(0u, 0u);
    if (i < a.n) {
        const int c = dn_classify(a, i, nullptr);
        v = make_uint2(c > 0 ? 1u : 0u, c == 2 ? 1u : 0u);
    }
    uint2 tot;
    dn_block_excl_scan<DN_THREADS>(v, s_tmp, tot);
    if (threadIdx.x == 0) a.block_sums[blockIdx.x] = tot;
}

// One block: exclusive scan of the block sums; total count of the new set.
__global__ void __launch_bounds__(1024) dn_scan_kernel(DensifyArgs a, int blocks) {
    __shared__ uint2 s_tmp[32];
    uint2 carry = make_uint2(0u, 0u);
    for (int b = 0; b < blocks; b += 1024) {
        const int idx = b + threadIdx.x;
        const uint2 v = idx < blocks ? a.block_sums[idx] : make_uint2(0u, 0u);
        uint2 tot;
        const uint2 ex = dn_block_excl_scan<1024>(v, s_tmp, tot);
        if (idx < blocks) a.block_sums[idx] = make_uint2(carry.x + ex.x, carry.y + ex.y);
        carry.x += tot.x;
        carry.y += tot.y;
    }
    if (threadIdx.x == 0) {
        const long long room = a.room > 0 ? a.room : 0;
        a.result[0] = carry.x;  // kept or densified
        a.result[1] = carry.y;  // candidates
        a.result[2] = (unsigned)((long long)carry.x + (carry.y < (unsigned long long)room ? carry.y : room));
    }
}

// Writes the outputs of every Gaussian into the new planes [planes][new_n_pad].
__global__ void __launch_bounds__(DN_THREADS) dn_scatter_kernel(DensifyArgs a) {
    __shared__ uint2 s_tmp[32];
    const int i = blockIdx.x * DN_THREADS + threadIdx.x;
    int c = 0;
    double size = 0.0;
    if (i < a.n) c = dn_classify(a, i, &size);
    uint2 tot;
    const uint2 ex = dn_block_excl_scan<DN_THREADS>(make_uint2(c > 0 ? 1u : 0u, c == 2 ? 1u : 0u), s_tmp, tot);
    if (c == 0) return;
    const uint2 base = a.block_sums[blockIdx.x];
    const unsigned kept = base.x + ex.x, cands = base.y + ex.y;
    const long long room = a.room > 0 ? a.room : 0;
    const unsigned extra = (long long)cands < room ? cands : (unsigned)room;
    const size_t out = (size_t)kept + extra;
    const bool grow = c == 2 && (long long)cands < room;
    const size_t np = (size_t)a.n_pad, onp = (size_t)a.out_n_pad;
    if (!grow) {
        for (int k = 0; k < a.planes; k++) a.out[k * onp + out] = a.params[k * np + i];
        return;
    }
    if (size <= a.size_threshold) {
        // Clone: the Gaussian and an identical copy.
        for (int k = 0; k < a.planes; k++) {
            const float v = a.params[k * np + i];
            a.out[k * onp + out] = v;
            a.out[k * onp + out + 1] = v;
        }
        return;
    }
    // Split: two moved, shrunk copies.
    for (int cp = 0; cp < 2; cp++) {
        const size_t o = out + cp;
        for (int j = 0; j < 3; j++) {
            const double m = (double)a.params[j * np + i];
            const double l = (double)a.params[(3 + j) * np + i];
            const double u = dn_uniform(a.seed, (uint64_t)i, cp, j);
            a.out[j * onp + o] = __double2float_rn(m + (u - 0.5) * exp(l));
            a.out[(3 + j) * onp + o] = __double2float_rn(l - a.log_split);
        }
        for (int k = 6; k < a.planes; k++) a.out[k * onp + o] = a.params[k * np + i];
    }
}

// Padding of the new planes: zeros, unit quaternions.
__global__ void dn_pad_kernel(DensifyArgs a, int new_n) {
    const int i = new_n + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.out_n_pad) return;
    for (int k = 0; k < a.planes; k++) a.out[(size_t)k * a.out_n_pad + i] = k == 6 ? 1.f : 0.f;
}

int densify_blocks(int n) { return (n + DN_THREADS - 1) / DN_THREADS; }

void launch_densify_count(const DensifyArgs& a, cudaStream_t s) {
    const int blocks = densify_blocks(a.n);
    if (blocks > 0) dn_count_kernel<<<blocks, DN_THREADS, 0, s>>>(a);
    dn_scan_kernel<<<1, 1024, 0, s>>>(a, blocks);
}

void launch_densify_scatter(const DensifyArgs& a, int new_n, cudaStream_t s) {
    const int blocks = densify_blocks(a.n);
    if (blocks > 0) dn_scatter_kernel<<<blocks, DN_THREADS, 0, s>>>(a);
    const int pad = a.out_n_pad - new_n;
    if (pad > 0) dn_pad_kernel<<<(pad + 255) / 256, 256, 0, s>>>(a, new_n);
}

// ---- opacity reset -----------------------------------------------------------------
__global__ void opacity_cap_kernel(float* __restrict__ plane, int n, double max_logit) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float x = plane[i];
    // Math.min(logit, cap) in double (NaN stays NaN), stored as float (trainer/gpu.js:944,
    // then packGaussians).
    if ((double)x > max_logit) plane[i] = __double2float_rn(max_logit);
}

void launch_opacity_cap(float* plane, int n, double max_logit, cudaStream_t s) {
    if (n > 0) opacity_cap_kernel<<<(n + 255) / 256, 256, 0, s>>>(plane, n, max_logit);
}

}  // namespace gs
