// Tile binning on the device: depth sort of the (view, Gaussian) pairs, emission of one
// key instance per (pair, covered tile), stable sort of the instances by tile id and
// the tile-range kernel.
//
// The result is the order of the 64-bit key (tile id << 32 | float bits of depth) with
// ties broken by Gaussian index, which is what the reference's BIN + SORT produce per
// tile (trainer/gpu.js:616-685: per-tile bitonic sort on depth, stable on splat index,
// :673) and what tileLists does on the CPU (trainer/gpu.js:450-481: a stable global
// depth sort, then a scatter in that order).  It is built the second way: the pairs
// (about 5x fewer than the instances) are radix-sorted on the 31 significant bits of
// their depth, the instances are emitted in that order, and a stable radix sort on the
// tile id (16 bits for up to 65,536 tiles: two passes) groups them by tile without
// disturbing the depth order.  There is no per-tile cap (the reference drops entries
// beyond 1,024 per tile, :614, :640).
#include "internal.h"

namespace gs {

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;  // keys per partition
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr unsigned FULL = 0xffffffffu;

int radix_tile_items() { return RS_TILE; }

// 8-bit digits; an even number of passes so the result lands back in the input buffers
// (keys above end_bit are zero, so an extra pass over them keeps the order).
static void pass_plan(int begin_bit, int end_bit, int& passes, int& step) {
    const int bits = end_bit - begin_bit;
    passes = (bits + 7) / 8;
    if (passes < 1) passes = 1;
    if (passes & 1) passes += 1;
    step = 8;
}

int radix_sort_passes(int begin_bit, int end_bit) {
    int p, s;
    pass_plan(begin_bit, end_bit, p, s);
    return p;
}

// Exclusive scan over a block of NT threads (NT a multiple of 32, <= 1024).
template <int NT>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_tmp, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = NT / 32;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_tmp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t t = lane < NW ? s_tmp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, t, o);
            if (lane >= o) t += y;
        }
        if (lane < NW) s_tmp[lane] = t;
    }
    __syncthreads();
    const uint32_t prefix = warp > 0 ? s_tmp[warp - 1] : 0u;
    total = s_tmp[NW - 1];
    __syncthreads();
    return prefix + x - v;
}

// ---------------------------------------------------------------------------------
// Radix sort, one sweep per digit (the Onesweep scheme of Adinets and Merrill): one
// kernel counts the digits of every pass over the whole segment; each pass is then a
// single kernel in which a block takes the next partition of RS_TILE keys (in launch
// order, from a counter), ranks them in shared memory, publishes its digit counts,
// looks back over the earlier partitions' published counts for its global offsets
// (decoupled look-back) and scatters keys and values.  Keys and values are read once
// and written once per pass.
//
// Look-back words: top two bits = 0 (not yet published), 1 (this partition's count),
// 2 (inclusive prefix over partitions 0..p); the bits below = the count.  A block waits only
// on earlier partitions, which took their index earlier and wait only on theirs, so the
// waits end; each wait is still bounded (OS_SPIN_LIMIT polls), after which the block
// sets the timeout flag and goes on with a wrong offset instead of hanging.
// ---------------------------------------------------------------------------------
// Look-back word of W bits: flags in the top two bits, the count below.  32-bit words
// serve segments below 2^30 keys (half the memset and look-back traffic), 64-bit ones
// the rest.
template <typename W>
struct LookWord {
    static constexpr W AGG = (W)1 << (sizeof(W) * 8 - 2);
    static constexpr W INC = (W)2 << (sizeof(W) * 8 - 2);
    static constexpr W VALUE = AGG - 1;
};
constexpr int OS_SPIN_LIMIT = 1 << 22;
constexpr int OS_LOOK = 8;  // look-back words read per round trip
constexpr int OS_MAX_PASSES = 4;
constexpr int OS_HIST_BLOCKS = 1184;  // 148 SMs x 8

__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Digit counts of all passes over the segment: ghist[pass * 256 + digit].  Shared-memory
// atomics into per-warp rows (equal digits within a warp serialise in hardware, which
// costs little even when a byte is constant), four keys per thread per round.
__global__ void __launch_bounds__(RS_THREADS) radix_hist_all(const uint32_t* __restrict__ keys, const SegInfo* seg,
                                                             int begin_bit, int passes, uint32_t* __restrict__ ghist,
                                                             uint32_t* __restrict__ gex, uint32_t* blocks_done) {
    __shared__ uint32_t wh[OS_MAX_PASSES][RS_WARPS][256];
    const uint32_t base = seg->base, n = seg->count;
    const int warp = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < OS_MAX_PASSES * RS_WARPS * 256; d += RS_THREADS) (&wh[0][0][0])[d] = 0u;
    __syncthreads();
    const uint32_t stride = gridDim.x * RS_THREADS * 4;
    for (uint32_t i0 = blockIdx.x * RS_THREADS * 4 + threadIdx.x; i0 < n; i0 += stride) {
        uint32_t k[4];
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const uint32_t idx = i0 + t * RS_THREADS;
            k[t] = idx < n ? __ldg(keys + base + idx) : 0u;
        }
#pragma unroll
        for (int t = 0; t < 4; t++) {
            if (i0 + t * RS_THREADS >= n) continue;
            for (int p = 0; p < passes; p++) atomicAdd(&wh[p][warp][(k[t] >> (begin_bit + 8 * p)) & 0xffu], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += RS_THREADS) {
        const int p = i >> 8, d = i & 255;
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < RS_WARPS; w++) s += wh[p][w][d];
        if (s) atomicAdd(ghist + i, s);
    }
    // The last block to finish turns the counts into each pass's exclusive digit offsets.
    __shared__ uint32_t s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(blocks_done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    __shared__ uint32_t s_tmp[32];
    for (int p = 0; p < passes; p++) {
        uint32_t tot;
        const uint32_t c = threadIdx.x < 256 ? __ldcg(ghist + p * 256 + threadIdx.x) : 0u;
        const uint32_t ex = block_excl_scan<RS_THREADS>(c, s_tmp, tot);
        if (threadIdx.x < 256) gex[p * 256 + threadIdx.x] = ex;
    }
}

// One partition of OS_THREADS x OS_ITEMS = RS_TILE keys per block; 256 threads of 16
// keys leave room for four resident partitions per SM, which hides more of each
// partition's load, look-back and scatter latency than two blocks of 512 threads.
constexpr int OS_THREADS = 256;
constexpr int OS_ITEMS = RS_TILE / OS_THREADS;
constexpr int OS_WARPS = OS_THREADS / 32;

#ifndef OS_MIN_BLOCKS
#define OS_MIN_BLOCKS 4  // resident partitions per SM the registers are sized for
#endif

template <typename W>
__global__ void __launch_bounds__(OS_THREADS, OS_MIN_BLOCKS) radix_onesweep(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, uint32_t* __restrict__ keys_out,
    uint32_t* __restrict__ vals_out, const SegInfo* seg, int shift, const uint32_t* __restrict__ gex,
    W* look, uint32_t* counter, unsigned int* timeout, const unsigned int* debug_wait,
    const unsigned int* never_set, uint2* ranges) {
    using LW = LookWord<W>;
    __shared__ uint32_t s_keys[RS_TILE];
    __shared__ uint32_t s_vals[RS_TILE];
    // The warps' digit counts live in s_vals until the keys are placed.
    static_assert(OS_WARPS * 256 <= RS_TILE, "warp rows must fit in s_vals");
    uint32_t(*s_warp)[256] = reinterpret_cast<uint32_t(*)[256]>(s_vals);
    __shared__ uint32_t s_digit_start[256];
    __shared__ uint32_t s_global[256];
    __shared__ uint32_t s_tmp[32];
    __shared__ uint32_t s_part;
    const uint32_t base = seg->base, n = seg->count;
    const uint32_t P = (n + RS_TILE - 1) / RS_TILE;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    if (threadIdx.x == 0) s_part = atomicAdd(counter, 1u);
    for (int d = threadIdx.x; d < OS_WARPS * 256; d += OS_THREADS) {
        (&s_warp[0][0])[d] = 0u;
        s_keys[d] = 0u;
    }
    __syncthreads();
    const uint32_t p = s_part;
    if (p >= P) return;
    const uint32_t part_start = p * RS_TILE;
    const uint32_t warp_start = part_start + warp * (OS_ITEMS * 32);
    uint32_t k[OS_ITEMS], pos[OS_ITEMS];
#pragma unroll
    for (int j = 0; j < OS_ITEMS; j++) {
        const uint32_t idx = warp_start + j * 32 + lane;
        k[j] = idx < n ? __ldg(keys_in + base + idx) : 0xffffffffu;
    }
    // Item by item: the lanes holding the same digit (each lane ORs its bit into the
    // digit's word of the warp's match row, then reads the word back; a warp whose valid
    // lanes all hold one digit skips that), then the running counts in the warp's row.
    // The match rows live in s_keys until the keys are placed; they start zeroed and
    // each group's first lane clears its word again.
    uint32_t* s_match = s_keys + warp * 256;
#pragma unroll
    for (int j = 0; j < OS_ITEMS; j++) {
        const bool valid = warp_start + j * 32 + lane < n;
        const uint32_t d = (k[j] >> shift) & 0xffu;
        const uint32_t d0 = __shfl_sync(FULL, d, 0);
        const uint32_t vmask = __ballot_sync(FULL, valid);
        uint32_t pm;
        const bool uniform = __all_sync(FULL, !valid || d == d0);
        if (uniform) {
            pm = valid ? vmask : 0u;
        } else {
            if (valid) atomicOr(&s_match[d], 1u << lane);
            __syncwarp();
            pm = valid ? s_match[d] : 0u;
        }
        const uint32_t prev = valid ? s_warp[warp][d] : 0u;
        __syncwarp();
        const bool leader = valid && (pm & lt_mask) == 0u;
        if (leader) {
            if (!uniform) s_match[d] = 0u;
            s_warp[warp][d] = prev + __popc(pm);
        }
        pos[j] = prev + __popc(pm & lt_mask);
        __syncwarp();
    }
    __syncthreads();
    // Threads 0..255 own one digit each.
    const int d = threadIdx.x;
    const bool owner = d < 256;
    uint32_t cnt = 0;
    if (owner) {
#pragma unroll
        for (int w = 0; w < OS_WARPS; w++) {
            const uint32_t c = s_warp[w][d];
            s_warp[w][d] = cnt;
            cnt += c;
        }
    }
    // Publish this partition's count as early as possible.
    W* my = look + (size_t)p * 256 + (owner ? d : 0);
    if (owner) st_relaxed(my, (W)((p == 0 ? LW::INC : LW::AGG) | (W)cnt));
    if (owner) s_global[d] = __ldg(gex + d);
    {
        uint32_t tot;
        const uint32_t lex = block_excl_scan<OS_THREADS>(cnt, s_tmp, tot);
        if (owner) s_digit_start[d] = lex;
    }
    __syncthreads();
    // Keys to their block-sorted slots.
#pragma unroll
    for (int j = 0; j < OS_ITEMS; j++) {
        const uint32_t idx = warp_start + j * 32 + lane;
        if (idx < n) {
            const uint32_t dj = (k[j] >> shift) & 0xffu;
            pos[j] += s_digit_start[dj] + s_warp[warp][dj];
            s_keys[pos[j]] = k[j];
        }
    }
    // Values in flight while this thread looks back for digit d.
    uint32_t v[OS_ITEMS];
#pragma unroll
    for (int j = 0; j < OS_ITEMS; j++) {
        const uint32_t idx = warp_start + j * 32 + lane;
        v[j] = (idx < n) ? (vals_in ? __ldg(vals_in + base + idx) : base + idx) : 0u;
    }
    if (p == 1 && d == 0 && debug_wait) {
        // Failure-detection test hook: a wait on a word nothing writes, given up after the
        // armed number of polls exactly as a look-back wait gives up (the flag is set and
        // the block carries on; the look-back below still finds the true offsets).
        const uint32_t polls = ld_relaxed(debug_wait);
        for (uint32_t s = 0; polls && ld_relaxed(never_set) == 0u; s++) {
            if (s >= polls) {
                atomicOr(timeout, 1u);
                break;
            }
            __nanosleep(32);
        }
    }
    if (p > 0 && owner) {
        // Walk back OS_LOOK partitions per round trip: sum published counts until an
        // inclusive prefix; re-poll from the first partition that has published nothing.
        uint32_t excl = 0;
        int q = (int)p - 1;
        int spins = 0;
        bool done = false;
        while (!done) {
            W w[OS_LOOK];
#pragma unroll
            for (int t = 0; t < OS_LOOK; t++) w[t] = q - t >= 0 ? ld_relaxed(look + (size_t)(q - t) * 256 + d) : LW::INC;
            int used = 0;
            bool stop = false;
#pragma unroll
            for (int t = 0; t < OS_LOOK; t++) {
                if (stop) continue;
                const W flag = w[t] & ~LW::VALUE;
                if (flag == 0) {
                    stop = true;
                    continue;
                }
                excl += (uint32_t)(w[t] & LW::VALUE);
                used++;
                if (flag == LW::INC) {
                    stop = true;
                    done = true;
                }
            }
            q -= used;
            if (!done && used == 0) {
                if (++spins > OS_SPIN_LIMIT) {
                    atomicOr(timeout, 1u);
                    break;
                }
                __nanosleep(32);
            }
        }
        st_relaxed(my, (W)(LW::INC | (W)(excl + cnt)));
        s_global[d] += excl;
    }
    __syncthreads();  // every warp has read its row of s_warp
#pragma unroll
    for (int j = 0; j < OS_ITEMS; j++) {
        const uint32_t idx = warp_start + j * 32 + lane;
        if (idx < n) s_vals[pos[j]] = v[j];
    }
    __syncthreads();
    const uint32_t total = min((uint32_t)RS_TILE, n - part_start);
    if (ranges) {
        // Last pass of the tile sort: the sorted tile ids themselves are not needed, only
        // where each tile's run starts and ends.  Each run of one id in this partition
        // bounds its tile's range from both sides; the maxima over all partitions are the
        // range (the output is sorted, so a tile's instances are contiguous).
        for (uint32_t i = threadIdx.x; i < total; i += OS_THREADS) {
            const uint32_t key = s_keys[i];
            const uint32_t dk = (key >> shift) & 0xffu;
            const uint32_t out = base + s_global[dk] + (i - s_digit_start[dk]);
            if (i == 0 || s_keys[i - 1] != key) atomicMax(&ranges[key].x, ~out);
            if (i + 1 == total || s_keys[i + 1] != key) atomicMax(&ranges[key].y, out + 1);
            vals_out[out] = s_vals[i];
        }
        return;
    }
    for (uint32_t i = threadIdx.x; i < total; i += OS_THREADS) {
        const uint32_t key = s_keys[i];
        const uint32_t dk = (key >> shift) & 0xffu;
        const uint32_t out = base + s_global[dk] + (i - s_digit_start[dk]);
        if (keys_out) keys_out[out] = key;
        vals_out[out] = s_vals[i];
    }
}

void launch_radix_sort(const RadixSortArgs& a, cudaStream_t s, int num_sms) {
    (void)num_sms;
    int passes, step;
    pass_plan(a.begin_bit, a.end_bit, passes, step);
    const int grid = a.max_parts > 0 ? a.max_parts : 1;
    uint32_t* ghist = a.totals;                               // [passes][256] digit counts
    uint32_t* gex = a.totals + OS_MAX_PASSES * 256;           // [passes][256] exclusive offsets
    uint32_t* counters = a.totals + 2 * OS_MAX_PASSES * 256;  // one partition counter per pass
    uint32_t* blocks_done = counters + OS_MAX_PASSES;
    cudaMemsetAsync(a.totals, 0, (2 * OS_MAX_PASSES * 256 + OS_MAX_PASSES + 1) * sizeof(uint32_t), s);
    radix_hist_all<<<min(grid, OS_HIST_BLOCKS), RS_THREADS, 0, s>>>(a.keys, a.seg, a.begin_bit, passes, ghist, gex,
                                                                    blocks_done);
    uint32_t* kb[2] = {a.keys, a.keys_alt};
    uint32_t* vb[2] = {a.vals, a.vals_alt};
    // The largest key count this buffer can hold decides the look-back word width.
    const bool wide = (long long)grid * RS_TILE >= (1ll << 30);
    for (int p = 0; p < passes; p++) {
        const int in = p & 1, out = in ^ 1;
        const uint32_t* vin = (p == 0 && a.iota) ? nullptr : vb[in];
        uint2* rg = p == passes - 1 ? a.ranges : nullptr;
        uint32_t* kout = (p == passes - 1 && a.discard_keys) ? nullptr : kb[out];
        if (wide) {
            cudaMemsetAsync(a.hist, 0, (size_t)grid * 256 * sizeof(unsigned long long), s);
            radix_onesweep<unsigned long long><<<grid, OS_THREADS, 0, s>>>(
                kb[in], vin, kout, vb[out], a.seg, a.begin_bit + p * step, gex + p * 256,
                reinterpret_cast<unsigned long long*>(a.hist), counters + p, a.timeout, a.debug_wait, a.never_set,
                rg);
        } else {
            cudaMemsetAsync(a.hist, 0, (size_t)grid * 256 * sizeof(uint32_t), s);
            radix_onesweep<uint32_t><<<grid, OS_THREADS, 0, s>>>(kb[in], vin, kout, vb[out], a.seg,
                                                                  a.begin_bit + p * step, gex + p * 256,
                                                                  reinterpret_cast<uint32_t*>(a.hist), counters + p,
                                                                  a.timeout, a.debug_wait, a.never_set, rg);
        }
    }
}

// ---------------------------------------------------------------------------------
// Key-instance emission.  Depth-sorted pairs are taken in chunks of EM_CHUNK:
// (1) per-chunk sums of the pairs' tile counts; (2) one block scans the chunk sums and
// fixes the segment's size (clamped to the capacity, with the overflow flag set);
// (3) each chunk rescans its counts, writes every pair's first-instance offset, and
// marks, for every EM_OUT-th instance, the pair it belongs to; (4) the expansion walks
// the instances in equal blocks of EM_OUT: a block reads its first and last pair from
// the marks, stages their offsets, ids and rectangles in shared memory, and each thread
// binary-searches its instance's pair there.  Work per block is fixed however many
// tiles a splat covers (one splat can cover thousands), and consecutive threads write
// consecutive instances.
// ---------------------------------------------------------------------------------
constexpr int EM_THREADS = 256;
constexpr int EM_ITEMS = 8;
constexpr int EM_CHUNK = EM_THREADS * EM_ITEMS;
#ifndef GS_EM_OUT
#define GS_EM_OUT 512  // measured: 512 beats 1024 (-27 % emission) and 2048
#endif
constexpr int EM_OUT = GS_EM_OUT;  // instances per expansion block
static_assert(EM_OUT % EM_THREADS == 0, "whole instances per expansion thread");

int emit_chunk_items() { return EM_CHUNK; }
int emit_out_items() { return EM_OUT; }

__device__ __forceinline__ uint32_t pair_count(const EmitArgs& a, uint32_t pair) {
    return a.pcount[pair] & ~GS_PCOUNT_RECT;
}

__global__ void __launch_bounds__(EM_THREADS) emit_reduce(EmitArgs a) {
    __shared__ uint32_t s_tmp[32];
    const uint32_t M = *a.visible;
    const uint32_t base = a.pair_seg->base;
    const uint32_t chunks = (M + EM_CHUNK - 1) / EM_CHUNK;
    for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
        uint32_t sum = 0;
#pragma unroll
        for (int j = 0; j < EM_ITEMS; j++) {
            const uint32_t sidx = c * EM_CHUNK + j * EM_THREADS + threadIdx.x;
            if (sidx < M) {
                // The gathered count is kept in depth order (in pair_offsets, which
                // emit_offsets overwrites with the offsets), so the offsets pass reads it
                // sequentially instead of gathering it again.
                const uint32_t cnt = pair_count(a, __ldg(a.sorted_pairs + base + sidx));
                a.pair_offsets[sidx] = cnt;
                sum += cnt;
            }
        }
        uint32_t tot;
        block_excl_scan<EM_THREADS>(sum, s_tmp, tot);
        if (threadIdx.x == 0) a.block_sums[c] = tot;
    }
}

__global__ void __launch_bounds__(1024) emit_scan(EmitArgs a) {
    __shared__ uint32_t s_tmp[32];
    const uint32_t M = *a.visible;
    const uint32_t chunks = (M + EM_CHUNK - 1) / EM_CHUNK;
    unsigned long long carry = 0;
    for (uint32_t b = 0; b < chunks; b += 1024) {
        const uint32_t idx = b + threadIdx.x;
        const uint32_t v = idx < chunks ? a.block_sums[idx] : 0u;
        uint32_t tot;
        const uint32_t ex = block_excl_scan<1024>(v, s_tmp, tot);
        if (idx < chunks) a.block_sums[idx] = (uint32_t)(carry + ex);
        carry += tot;
    }
    if (threadIdx.x == 0) {
        const unsigned long long seg_base =
            a.prev_seg ? (unsigned long long)a.prev_seg->base + a.prev_seg->count : 0ull;
        const unsigned long long need = seg_base + carry;
        unsigned long long count = carry;
        if (need > a.capacity) {
            a.status->overflow = 1u;
            count = seg_base < a.capacity ? a.capacity - seg_base : 0ull;
        }
        if (need > a.status->instances_needed) a.status->instances_needed = need;
        a.inst_seg->base = (uint32_t)(seg_base < a.capacity ? seg_base : a.capacity);
        a.inst_seg->count = (uint32_t)count;
    }
}

__global__ void __launch_bounds__(EM_THREADS) emit_offsets(EmitArgs a) {
    __shared__ uint32_t s_cnt[EM_CHUNK];
    __shared__ uint32_t s_tmp[32];
    const uint32_t M = *a.visible;
    const uint32_t chunks = (M + EM_CHUNK - 1) / EM_CHUNK;
    const uint32_t total = a.inst_seg->count;
    for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
        const uint32_t first = c * EM_CHUNK;
        for (uint32_t j = threadIdx.x; j < EM_CHUNK; j += EM_THREADS) {
            const uint32_t s = first + j;
            s_cnt[j] = s < M ? a.pair_offsets[s] : 0u;  // the counts emit_reduce kept
        }
        __syncthreads();
        uint32_t cnt[EM_ITEMS];
        uint32_t local = 0;
#pragma unroll
        for (int j = 0; j < EM_ITEMS; j++) {
            cnt[j] = s_cnt[threadIdx.x * EM_ITEMS + j];
            local += cnt[j];
        }
        uint32_t tot;
        uint32_t run = block_excl_scan<EM_THREADS>(local, s_tmp, tot) + a.block_sums[c];
#pragma unroll
        for (int j = 0; j < EM_ITEMS; j++) {
            const uint32_t s = first + threadIdx.x * EM_ITEMS + j;
            if (s < M) {
                a.pair_offsets[s] = run;
                // Instances run, run + 1, ..., run + cnt - 1 belong to pair s: mark the
                // expansion blocks that start inside that range.
                uint32_t b = (run + EM_OUT - 1) / EM_OUT;
                const uint32_t end = min(run + cnt[j], total);
                for (; (unsigned long long)b * EM_OUT < end; b++) a.block_first_pair[b] = s;
            }
            run += cnt[j];
        }
        __syncthreads();
    }
}

// Inclusive max-scan over a block of NT threads.
template <int NT>
__device__ __forceinline__ uint32_t block_incl_max(uint32_t v, uint32_t* s_tmp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = NT / 32;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x = max(x, y);
    }
    if (lane == 31) s_tmp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t t = lane < NW ? s_tmp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, t, o);
            if (lane >= o) t = max(t, y);
        }
        if (lane < NW) s_tmp[lane] = t;
    }
    __syncthreads();
    const uint32_t prefix = warp > 0 ? s_tmp[warp - 1] : 0u;
    __syncthreads();
    return max(prefix, x);
}

// s_head is padded by one word per 32 (HP): each thread walks PER consecutive entries,
// and without the padding threads t and t + 32 / PER would hit the same bank.
__device__ __forceinline__ uint32_t HP(uint32_t i) { return i + (i >> 5); }
constexpr size_t EM_EXPAND_SMEM = (size_t)(EM_OUT + 1) * (4 + 4 + 16 + 16) + (size_t)(EM_OUT + EM_OUT / 32) * 4;

__global__ void __launch_bounds__(EM_THREADS) emit_expand(EmitArgs a) {
    constexpr int PER = EM_OUT / EM_THREADS;  // instances per thread
    extern __shared__ __align__(16) unsigned char em_smem[];
    uint4* s_span = reinterpret_cast<uint4*>(em_smem);                               // rows' tile spans
    uint4* s_geom = s_span + (EM_OUT + 1);  // first tile, tiles_x | width << 16 | rect flag, spans of rows 8..11
    uint32_t* s_off = reinterpret_cast<uint32_t*>(s_geom + (EM_OUT + 1));
    uint32_t* s_pair = s_off + (EM_OUT + 1);
    uint32_t* s_head = s_pair + (EM_OUT + 1);
    __shared__ uint32_t s_tmp[32];
    const uint32_t M = *a.visible;
    const uint32_t base = a.pair_seg->base;
    const uint32_t inst_base = a.inst_seg->base;
    const uint32_t total = a.inst_seg->count;
    const uint32_t blocks = (total + EM_OUT - 1) / EM_OUT;
    for (uint32_t b = blockIdx.x; b < blocks; b += gridDim.x) {
        const uint32_t o0 = b * EM_OUT;
        const uint32_t o1 = min(o0 + EM_OUT, total);
        const uint32_t p_lo = a.block_first_pair[b];
        const uint32_t p_hi = (b + 1 < blocks) ? a.block_first_pair[b + 1] : M - 1;
        // Every pair after p_lo starts after o0 and holds >= 1 instance, so the block
        // needs at most EM_OUT + 1 pairs (the bound matters for the last block when the
        // capacity clamped the instance count).
        const uint32_t np = min(p_hi - p_lo + 1, (uint32_t)EM_OUT + 1);
        for (uint32_t j = threadIdx.x; j < EM_OUT + EM_OUT / 32; j += EM_THREADS) s_head[j] = 0u;
        for (uint32_t j = threadIdx.x; j < np; j += EM_THREADS) {
            const uint32_t pair = __ldg(a.sorted_pairs + base + p_lo + j);
            const uint4* er = reinterpret_cast<const uint4*>(a.erec + pair);
            const uint4 h = __ldg(er);
            s_off[j] = a.pair_offsets[p_lo + j];
            s_pair[j] = pair;
            s_geom[j] = h;
            s_span[j] = __ldg(er + 1);
        }
        __syncthreads();
        // Head flags: the instance where each pair starts gets the pair's local index;
        // a running max then gives every instance its pair.
        for (uint32_t j = 1 + threadIdx.x; j < np; j += EM_THREADS) {
            const uint32_t pos = s_off[j] - o0;
            if (pos < (uint32_t)EM_OUT) s_head[HP(pos)] = j;
        }
        __syncthreads();
        uint32_t run = 0, loc[PER];
#pragma unroll
        for (int k = 0; k < PER; k++) {
            run = max(run, s_head[HP(threadIdx.x * PER + k)]);
            loc[k] = run;
        }
        const uint32_t prefix = block_incl_max<EM_THREADS>(run, s_tmp);
        const uint32_t carry = __shfl_up_sync(FULL, prefix, 1);
        // Exclusive prefix of this thread = inclusive max of the threads before it.
        uint32_t before = 0;
        {
            const int lane = threadIdx.x & 31;
            before = lane > 0 ? carry : 0u;
            if (lane == 0 && threadIdx.x > 0) before = s_tmp[(threadIdx.x >> 5) - 1];
        }
        __syncthreads();
        // Tile of each instance into shared memory (s_head holds tiles now), then
        // striped, coalesced stores.
        uint32_t jj[PER];
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const uint32_t ol = threadIdx.x * PER + k;
            const uint32_t j = max(before, loc[k]);
            jj[k] = j;
            const uint4 gm = s_geom[j];
            const uint32_t tx = gm.y & 0xffffu, w = (gm.y >> 16) & 0x7fffu;
            uint32_t t = o0 + ol - s_off[j];
            uint32_t tile;
            if (gm.y >> 31) {
                const uint32_t row = t / max(w, 1u);
                tile = gm.x + row * tx + (t - row * w);
            } else {
                // Walk the rows' spans (at most GS_SPAN_ROWS).
                const uint4 sp = s_span[j];
                const uint32_t words[6] = {sp.x, sp.y, sp.z, sp.w, gm.z, gm.w};
                tile = gm.x;
#pragma unroll
                for (int r = 0; r < GS_SPAN_ROWS; r++) {
                    const uint32_t h = (words[r >> 1] >> (16 * (r & 1))) & 0xffffu;
                    const uint32_t xs = h & 0xffu, len = (h >> 8) - xs;
                    if (t < len) {
                        tile = gm.x + (uint32_t)r * tx + xs + t;
                        break;
                    }
                    t -= len;
                }
            }
            s_head[HP(ol)] = tile;
        }
        __syncthreads();
        for (uint32_t ol = threadIdx.x; ol < o1 - o0; ol += EM_THREADS) a.inst_keys[inst_base + o0 + ol] = s_head[HP(ol)];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PER; k++) s_head[HP(threadIdx.x * PER + k)] = s_pair[jj[k]];
        __syncthreads();
        for (uint32_t ol = threadIdx.x; ol < o1 - o0; ol += EM_THREADS) a.inst_vals[inst_base + o0 + ol] = s_head[HP(ol)];
        __syncthreads();
    }
}

void launch_emit(const EmitArgs& a, cudaStream_t s, int num_sms) {
    // One block per chunk / output block of the capacity; idle blocks exit at once.
    const int grid = a.max_chunks > 0 ? a.max_chunks : 1;
    const int grid_out = (int)(a.capacity / EM_OUT + 1);
    (void)num_sms;
    emit_reduce<<<grid, EM_THREADS, 0, s>>>(a);
    emit_scan<<<1, 1024, 0, s>>>(a);
    emit_offsets<<<grid, EM_THREADS, 0, s>>>(a);
    emit_expand<<<grid_out, EM_THREADS, EM_EXPAND_SMEM, s>>>(a);
}


// ---------------------------------------------------------------------------------
// Tile ranges: each tile's [first, last + 1) in the tile-sorted instances (absolute
// indices), bounded by the tile sort's last pass.  Tiles without instances keep the
// zeroed (0, 0).
// ---------------------------------------------------------------------------------
// (~first, last + 1) -> (first, last + 1); an untouched (0, 0) stays.  No tile starts at
// index 0xffffffff (the instance capacity is below 2^32 - 1), so ~first is never 0.
__global__ void __launch_bounds__(256) ranges_finish_kernel(uint2* ranges, int count) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const uint32_t x = ranges[t].x;
        if (x) ranges[t].x = ~x;
    }
}

void launch_ranges_finish(uint2* ranges, int count, cudaStream_t s) {
    if (count <= 0) return;
    ranges_finish_kernel<<<(count + 255) / 256, 256, 0, s>>>(ranges, count);
}

cudaError_t radix_prepare() {
    return cudaFuncSetAttribute(emit_expand, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)EM_EXPAND_SMEM);
}

}  // namespace gs
