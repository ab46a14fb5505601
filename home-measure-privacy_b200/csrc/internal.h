// Host-side launch interface of the kernels (shared by the .cu files and the C ABI).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "gs_common.cuh"

namespace gs {

// What the instance emission gathers for one (view, Gaussian) pair, in one 32-byte
// sector: the global tile of the rectangle's corner (x0, y0), tiles_x | (x1 - x0) << 16
// | whole-rectangle flag << 31, and the per-row tile spans of up to 12 rows.
struct __align__(32) EmitRec {
    uint32_t first_tile;
    uint32_t geom;
    uint32_t spans_hi[2];    // rows 8..11, packed as below
    uint4 spans;             // row r < 8: tiles [xs, xe) as bytes (xs | xe << 8) << 16 * (r & 1), x0-relative
};

// Projection forward over view slots [0, num_views) of views[view_first + slot].
struct ProjectArgs {
    const float* params;     // [planes][n_pad]
    int n, n_pad, degree;
    const ViewDesc* views;   // device array of all views
    int view_first, num_views;
    int pair_slot_first;     // pair slot of view_first (0 in the batched path)
    float near_plane, dilation;
    int rect_mode;
    float4* geo0;            // [num_views * n_pad]
    float4* geo1;
    float4* rgb;
    uint32_t* keys;          // depth key, GS_KEY_SENTINEL when the pair covers no tile
    unsigned int* visible;   // optional counter of pairs with >= 1 tile
    int tile_cull;           // 1: only tiles the alpha >= alpha_min ellipse reaches
    float alpha_min;
    uint32_t* pcount;        // instances of the pair (0 when it covers no tile)
    EmitRec* erec;           // written for pairs that cover >= 1 tile
    float* stats_cnt;        // training steps: += views the Gaussian projects into (or nullptr)
};
void launch_project_fwd(const ProjectArgs& a, cudaStream_t s);

// Projection backward: screen gradients of the view slots -> parameter gradients.
struct ProjectBwdArgs {
    const float* params;
    int n, n_pad, degree;
    const ViewDesc* views;
    int view_first, num_views;
    int pair_slot_first;     // pair slot of view_first (0 in the batched path)
    float dilation;
    const float4* sg8;       // [pairs][2] float4
    const float* sg1;        // [pairs]
    float* grads;            // [planes][n_pad]
    int accumulate;          // add to grads instead of overwriting them
    float* stats_sum;        // training steps: += |(dL/du, dL/dv)| over the views (or nullptr)
};
void launch_project_bwd(const ProjectBwdArgs& a, cudaStream_t s);

// ---- densification -----------------------------------------------------------------
struct DensifyArgs {
    const float* params;     // [planes][n_pad]
    const float* stats;      // [2][n_pad]: sums of gradient norms, view counts
    int n, n_pad, planes;
    float* out;              // [planes][out_n_pad]
    int out_n_pad;
    double grad_threshold, size_threshold, min_opacity, max_size, log_split;
    long long room;          // max_count - n
    unsigned long long seed;
    uint2* block_sums;       // scratch, densify_blocks(n) entries
    unsigned* result;        // [0] kept or densified, [1] candidates, [2] new count
};
int densify_blocks(int n);
void launch_densify_count(const DensifyArgs& a, cudaStream_t s);
void launch_densify_scatter(const DensifyArgs& a, int new_n, cudaStream_t s);
void launch_opacity_cap(float* plane, int n, double max_logit, cudaStream_t s);
// stats += step unless the step's update was skipped (skip: reduced flag, or status).
void launch_stats_commit(float* stats, const float* step, int n_pad, const DevStatus* status, const float* skip,
                         cudaStream_t s);

// ---- sorting ----------------------------------------------------------------------
// LSD radix sort of u32 keys with u32 values over a segment [seg->base, +seg->count)
// (device-resident offsets).  Ping-pongs between (keys, vals) and (keys_alt, vals_alt);
// with an even number of passes the result is back in (keys, vals).
struct RadixSortArgs {
    uint32_t* keys;
    uint32_t* vals;
    uint32_t* keys_alt;
    uint32_t* vals_alt;
    int iota;                // 1: values start as the absolute element index
    const SegInfo* seg;
    int begin_bit, end_bit;  // bits to sort
    unsigned long long* hist;  // look-back words, 256 * max_parts
    uint32_t* totals;        // digit counts and offsets of every pass, partition counters (>= 2053 words)
    int max_parts;
    unsigned int* timeout;   // set when a look-back wait gave up
    const unsigned int* debug_wait;  // test hook (device word): partition 1 of every pass first
                                     // polls *never_set this many times, then gives up
    const unsigned int* never_set;
    // Non-null: the keys are tile ids and the last pass writes no keys; it bounds each
    // tile's run instead, ranges[t] = (~first, last + 1) by atomic maxima into zeroed
    // words (launch_ranges_finish turns ~first into first).
    uint2* ranges = nullptr;
    // True: only the sorted values are wanted; the last pass writes no keys.
    bool discard_keys = false;
};
int radix_sort_passes(int begin_bit, int end_bit);
void launch_radix_sort(const RadixSortArgs& a, cudaStream_t s, int num_sms);
int radix_tile_items();
cudaError_t radix_prepare();

// Emission of key instances from the depth-sorted pairs.
struct EmitArgs {
    const uint32_t* sorted_pairs;   // pairs in depth order (first `visible` are real)
    const SegInfo* pair_seg;        // pair segment: base into sorted_pairs, count
    const unsigned int* visible;    // number of visible pairs in the segment
    const uint32_t* pcount;
    const EmitRec* erec;
    const ViewDesc* views;
    int view_first, n_pad;
    int pair_slot_first;            // slot of the first pair of this segment
    uint32_t* block_sums;           // scratch, >= chunks
    uint32_t* pair_offsets;         // scratch: first instance of each sorted pair (>= pairs)
    uint32_t* block_first_pair;     // scratch: pair of every EM_OUT-th instance (>= cap/EM_OUT + 2)
    SegInfo* inst_seg;              // out: instance segment (base, count)
    const SegInfo* prev_seg;        // previous instance segment (plain path) or nullptr
    uint32_t* inst_keys;            // global tile id
    uint32_t* inst_vals;            // pair index
    unsigned long long capacity;
    DevStatus* status;
    int max_chunks;
};
void launch_emit(const EmitArgs& a, cudaStream_t s, int num_sms);
int emit_chunk_items();
int emit_out_items();

// Completes the ranges a tile sort's last pass bounded (RadixSortArgs::ranges) for tiles
// [0, count) of `ranges`: tiles without instances stay (0, 0).
void launch_ranges_finish(uint2* ranges, int count, cudaStream_t s);

// ---- rasterisation ---------------------------------------------------------------------
struct RasterArgs {
    const ViewDesc* views;
    int view_first, num_views;
    int tile_first, num_tiles;      // global tiles [tile_first, tile_first + num_tiles)
    int pixel_first;                // first pixel of view_first
    const uint2* ranges;
    const uint32_t* inst_pair;
    const float4* geo0;
    const float4* geo1;
    const float4* rgb;
    int pair_slot_first;            // pair index = pair - pair_slot_first * n_pad ... (unused)
    float alpha_max, alpha_min, t_min;
    // forward outputs / backward inputs (indexed by global pixel)
    float* image;
    float* t_final;
    uint32_t* last;
    const float* dl;                // backward: dL/dpixel
    float4* sg8;                    // backward outputs
    float* sg1;
    unsigned int* work_counter;     // persistent queue head (nullptr = one CTA per tile)
    const uint32_t* tile_order;     // optional permutation of the tiles (heavy first)
};
// Raster variants: tile edge (8, 16, 32 or 64 pixels), shared-memory batch (32, 64, 128 or 256
// splats), pixels per thread, and the work tile a CTA covers (the tile itself, or for
// 32- and 64-pixel tiles a 16 x 16 part of it; raster_variant_ok lists what exists).
bool raster_variant_ok(int tile, int wt, int ppt);
void launch_raster_fwd(const RasterArgs& a, int tile, int wt, int batch, int ppt, int persistent_ctas,
                       cudaStream_t s);
void launch_raster_bwd(const RasterArgs& a, int tile, int wt, int batch, int ppt, int persistent_ctas,
                       cudaStream_t s);
int raster_max_ctas_per_sm(int tile, int wt, int batch, int ppt, bool backward);

// ---- data-parallel exchange (NCCL, loaded at run time) --------------------------------
int dp_unique_id_bytes();
bool dp_unique_id(void* out, char* err, size_t n);
void* dp_comm_create(const void* id, int rank, int world, char* err, size_t n);
bool dp_allreduce_sum(void* comm, float* buf, size_t count, cudaStream_t s, char* err, size_t n);
void dp_comm_destroy(void* comm);

// Blends (pixel, splat evaluations) of the last forward, added to *out.
void launch_blend_count(const ViewDesc* views, int view_first, int num_views, int max_pixels, const uint2* ranges,
                        const uint32_t* last, unsigned long long* out, cudaStream_t s);

// Tiles ordered by descending list length (for the persistent queue).
void launch_tile_order(const uint2* ranges, int tile_first, int num_tiles, uint32_t* order,
                       uint32_t* scratch, cudaStream_t s);

// ---- loss ------------------------------------------------------------------------------
struct LossArgs {
    const ViewDesc* views;
    int view_first, num_views;
    int block_first, num_blocks;    // loss blocks of these views
    const float* image;
    const uint8_t* target_u8;       // one of the two
    const float* target_f32;
    float* dl;
    float lambda;
    int window;                     // 0 = 7x7 box, 1 = 11-tap Gaussian
    double* acc;                    // per view: [L1 sum, SSIM sum]
};
void launch_loss(const LossArgs& a, cudaStream_t s);
cudaError_t loss_prepare();
int loss_block_w();
int loss_block_h();

// ---- optimiser -------------------------------------------------------------------------
struct AdamArgs {
    float* params;
    const float* grads;
    float* m;
    float* v;
    int n, n_pad, planes;
    float lr[GS_MAX_PLANES];
    float beta1, beta2, eps;
    DevStatus* status;
    const float* skip;              // reduced overflow count (nullptr: this replica's status)
};
void launch_adam(const AdamArgs& a, cudaStream_t s);

// Data-parallel split: the gradient buffer's tail and the step's end from a reduced tail.
void launch_grad_tail(const DevStatus* status, const double* acc, const ViewDesc* views, int view_first,
                      int num_views, float lambda, int window, float* tail, cudaStream_t s);
void launch_reduced_step_end(DevStatus* status, const float* tail, cudaStream_t s);

// Finishes a step: loss from the accumulators, skip flag, Adam step counter.
void launch_step_end(DevStatus* status, const double* acc, const ViewDesc* views,
                     int view_first, int num_views, float lambda, int window, int advance,
                     cudaStream_t s);
void launch_loss_from_acc(DevStatus* status, const double* acc, const ViewDesc* views,
                          int view_first, int num_views, float lambda, int window,
                          cudaStream_t s);

// ---- layout conversion -----------------------------------------------------------------
void launch_screen_grads16(const float4* sg8, const float* sg1, int n, float* out16,
                           cudaStream_t s);
void launch_splats12(const float4* geo0, const float4* geo1, const float4* rgb,
                     const uint32_t* keys, int n, float* out12, cudaStream_t s);

// ---- initialisation from points -----------------------------------------------------------
struct NeighbourArgs {
    const float* xyz;
    int count;
    unsigned long long* keys;   // hash table of cube keys (mask + 1 entries, empty = all ones)
    unsigned* ids;              // dense cube id per table entry
    unsigned mask;
    unsigned* counters;         // [0] cubes
    unsigned* point_slot;       // table entry of each point's cube
    unsigned* cell_count;       // points per cube
    unsigned* cell_start;
    unsigned* cell_cursor;
    unsigned* cell_points;      // point indices grouped by cube
    float* sizes;
    double min_size, max_size, fallback;
};
void launch_neighbour_sizes(const NeighbourArgs& a, cudaStream_t s);
void launch_init_planes(const float* xyz, const float* rgb, const float* sizes, float fixed_size, int count, int n_pad,
                        int planes, float* params, cudaStream_t s);

void launch_grey(const uint8_t* rgb, size_t pixels, uint8_t* grey, cudaStream_t s);
void launch_laplacian_sums(const uint8_t* grey, int count, int width, int height, long long* sums, cudaStream_t s);

// ---- scene I/O -------------------------------------------------------------------------
struct PlyHeaderInfo {
    int64_t header_bytes, count;
    int nprops;
    int col[GS_MAX_PLANES];   // file column of each parameter plane (-1: absent)
    int dc[3];
    int file_sh_coeffs;       // f_rest coefficients per channel in the file
};
}  // namespace gs
#include <string>
#include <vector>
namespace gs {
int ply_parse(const void* data, int64_t bytes, int planes, PlyHeaderInfo* out, std::string* err);
void launch_ply_to_planes(const float* body, const PlyHeaderInfo& h, int n_pad, int planes, float* params,
                          cudaStream_t s);
std::string ply_header(int64_t n, int nk_out);
void launch_planes_to_ply(const float* params, int n, int n_pad, int planes, int nk_out, float* body, cudaStream_t s);
void launch_splat_records(const float* params, int n, int n_pad, unsigned char* rec, double* weight,
                          unsigned char* finite, cudaStream_t s);
std::vector<int> splat_order(const std::vector<double>& weight, const std::vector<unsigned char>& finite);

}  // namespace gs
