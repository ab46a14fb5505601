// The C ABI (include/gsb200.h): context, device buffers, the training-step pipeline
// in its batched and plain forms, CUDA-graph capture and per-stage timing.
//
// Host orchestration replaces createRenderer's closures (trainer/gpu.js:704-980): the
// reference builds a bind group, an encoder and a queue submit per dispatch (about 11
// per step, :728-736) and reads the image back every 25 steps (:934-940).  Here a step
// is a fixed sequence of kernel launches on one stream whose sizes all live in device
// memory, so the whole step is captured once as a CUDA graph and replayed.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/gsb200.h"
#include "internal.h"

// NVTX range over a C-ABI call, named after it: host-side structure for a timeline
// profiler (NVTX v3 is header-only; with no tool attached a range costs a pointer test).
struct NvtxScope {
    explicit NvtxScope(const char* name) { nvtxRangePushA(name); }
    ~NvtxScope() { nvtxRangePop(); }
    NvtxScope(const NvtxScope&) = delete;
    NvtxScope& operator=(const NvtxScope&) = delete;
};
#define GS_TRACE(name) NvtxScope gs_nvtx_scope_(name)

using namespace gs;

// ---------------------------------------------------------------------------------
// Errors.
// ---------------------------------------------------------------------------------
static thread_local std::string g_err = "no error";

static int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(x)                                                                                   \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) return fail(GS_ERR_CUDA, "%s failed: %s", #x, cudaGetErrorString(e_)); \
    } while (0)

#define CKI(x)                       \
    do {                             \
        int r_ = (x);                \
        if (r_ != GS_OK) return r_;  \
    } while (0)

// ---------------------------------------------------------------------------------
// Device buffers.
// ---------------------------------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    template <typename T>
    T* as() const { return reinterpret_cast<T*>(p); }
};

static int64_t g_generation_counter = 0;

enum Stage {
    ST_PROJECT = 0,
    ST_SORT_PAIRS,
    ST_EMIT,
    ST_SORT_INST,
    ST_RASTER_FWD,
    ST_LOSS,
    ST_RASTER_BWD,
    ST_PROJECT_BWD,
    ST_ADAM,
    ST_OTHER,
    ST_END = -1
};
static const char* kStageNames[GS_NUM_STAGES] = {"project",    "sort_pairs",  "emit",        "sort_instances",
                                                 "raster_fwd", "loss",        "raster_bwd",  "project_bwd",
                                                 "adam",       "other"};

struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    int64_t generation = -1;
    std::vector<int> tags;                 // stage tag of each timing mark
    std::vector<cudaGraphNode_t> nodes;    // event-record node of each mark
    int64_t launches[GS_NUM_STAGES] = {};
};

struct TimingSlot {
    std::vector<cudaEvent_t> ev;
    std::vector<int> tags;
    int64_t launches[GS_NUM_STAGES] = {};
    bool pending = false;
};

struct GraphKey {
    int first, count, batched, window, kind, loss_lambda_bits;
    int phase;  // 0 = whole step, 1 = gradients only (data-parallel split)
    GsAdamConfig adam;
    bool operator<(const GraphKey& o) const { return memcmp(this, &o, sizeof(GraphKey)) < 0; }
};

struct GsContext {
    GsConfig cfg;
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    std::string device_name;
    // scene
    int n = 0, n_pad = 0, degree = 0, planes = 14;
    // grads: planes x n_pad gradients, 2 x n_pad step-local densification statistics,
    // then GS_GRAD_TAIL_FLOATS (loss sum, overflow, views)
    DevBuf params, grads, mom1, mom2;
    bool grads_pending = false;         // gs_step_gradients queued, gs_step_apply not yet
    void* dp_comm = nullptr;            // NCCL communicator of gs_dp_init (data parallel)
    int dp_rank = 0, dp_world = 1;
    DevBuf stats;                       // densification statistics [2][n_pad]: norm sums, view counts
    bool stats_on = false;              // training steps accumulate them
    bool stats_active = false;          // set while a training step's kernels are enqueued
    DevBuf dn_scratch;                  // densify block sums and result; scene-file bodies
    DevBuf nb_scratch;                  // neighbour search: table, cubes, points
    // views: training views [0, V) plus one scratch view at index V for render /
    // gradients / loss-gradient calls on arbitrary cameras or images
    std::vector<GsCamera> cams;
    int V = 0;
    std::vector<ViewDesc> vdesc;
    int64_t total_pixels = 0, total_tiles = 0, total_loss_blocks = 0;
    int tile_bits = 1;
    std::vector<int> target_kind;  // 0 none, 1 u8, 2 f32
    DevBuf views_d, target_u8, target_f32, image, t_final, last, dl, ranges, tile_order;
    // pairs
    int64_t pair_cap = 0;
    DevBuf geo0, geo1, rgb, erec, pkeys, pvals, pkeys_alt, pvals_alt, sg8, sg1, pcount;
    // instances
    int64_t inst_cap = 0;
    bool inst_cap_valid = false;
    DevBuf ikeys, ivals, ikeys_alt, ivals_alt;
    DevBuf hist, totals, block_sums;  // radix histograms, digit totals, emission chunk sums
    DevBuf pair_offsets, block_first_pair;  // emission: per-pair offsets, expansion marks
    // segments: [0, 65) all-pairs segment of c views; [65, 129) pair segment of slot s;
    // [129] batched instance segment; [130, 194) instance segment of slot s
    DevBuf segs, visible, acc, scratch16;
    DevBuf status;
    DevStatus* status_host = nullptr;
    cudaEvent_t status_event = nullptr;
    // gs_train_step_host_async: a copy stream, two staging buffers for the step's photos,
    // and per slot the events "photos copied", "staging buffer free", "step done".
    cudaStream_t copy_stream = nullptr;
    DevBuf stage[2];
    cudaEvent_t ev_copied[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr}, ev_done[2] = {nullptr, nullptr};
    bool pipe_pending[2] = {false, false};
    int pipe_slot = 0;
    bool status_pending = false;
    int64_t skipped_steps = 0;
    unsigned int debug_wait_host = 0;   // source of gs_debug_lookback_wait's copy
    bool tuned = false;                 // cfg.autotune has run
    // last forward
    int last_first = -1, last_count = 0, last_batched = 1;
    bool have_loss = false;
    // raster tuning: shared-memory batch and pixels per thread of each kernel
    int tile = GS_TILE;                 // tile edge of binning and raster (8, 16, 32 or 64)
    int batch_fwd = 256, batch_bwd = 256, ppt_fwd = 4, ppt_bwd = 4;
    int wt_fwd = GS_TILE, wt_bwd = GS_TILE;  // raster work-tile edges (<= the tile edge)
    int ctas_fwd = 0, ctas_bwd = 0;
    // graphs
    int64_t generation = 0;
    std::map<GraphKey, StepGraph> graphs;
    // timing
    bool stage_timing = true;
    std::vector<cudaEvent_t> capture_events;
    std::vector<int> rec_tags;
    std::vector<cudaEvent_t> rec_events;
    bool capturing = false;
    TimingSlot slots[4];
    int slot_next = 0;
    int rec_slot = -1;
    int64_t rec_launches[GS_NUM_STAGES] = {};
    double stage_ms[GS_NUM_STAGES] = {};
    int64_t stage_launches[GS_NUM_STAGES] = {};
    int32_t timed_steps = 0;
    int64_t last_step_launches = 0;
    cudaEvent_t user_events[64] = {};
};

static const int SEG_ALL = 0, SEG_PAIR = 65, SEG_INST_ALL = 129, SEG_INST = 130, SEG_COUNT = 194;

// Gradient buffer layout: parameter gradients, step-local statistics, tail.
static float* step_stats(GsContext* c) { return c->grads.as<float>() + (size_t)c->planes * c->n_pad; }
static float* grad_tail(GsContext* c) { return c->grads.as<float>() + (size_t)(c->planes + 2) * c->n_pad; }
static size_t grad_buffer_floats(GsContext* c) { return (size_t)(c->planes + 2) * c->n_pad + GS_GRAD_TAIL_FLOATS; }

static int ensure(DevBuf& b, size_t bytes, GsContext* c) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return GS_OK;
    if (b.p) CK(cudaFree(b.p));
    b.p = nullptr;
    b.bytes = 0;
    const size_t grown = (bytes + bytes / 4 + 255) & ~(size_t)255;
    cudaError_t e = cudaMalloc(&b.p, grown);
    if (e != cudaSuccess) {
        cudaGetLastError();
        e = cudaMalloc(&b.p, bytes);
        if (e != cudaSuccess) return fail(GS_ERR_CUDA, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
        b.bytes = bytes;
    } else {
        b.bytes = grown;
    }
    c->generation = ++g_generation_counter;  // cached graphs hold the old pointers
    return GS_OK;
}

static void release(DevBuf& b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
}

// ---------------------------------------------------------------------------------
// Timing marks.
// ---------------------------------------------------------------------------------
static int mark(GsContext* c, int tag) {
    if (!c->stage_timing || (!c->capturing && c->rec_slot < 0)) return GS_OK;
    const size_t m = c->rec_tags.size();
    c->rec_tags.push_back(tag);
    if (c->capturing) {
        while (c->capture_events.size() <= m) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            c->capture_events.push_back(e);
        }
        CK(cudaEventRecordWithFlags(c->capture_events[m], c->stream, cudaEventRecordExternal));
    } else {
        TimingSlot& sl = c->slots[c->rec_slot];
        while (sl.ev.size() <= m) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            sl.ev.push_back(e);
        }
        CK(cudaEventRecord(sl.ev[m], c->stream));
    }
    return GS_OK;
}

static void count_launches(GsContext* c, int stage, int k) { c->rec_launches[stage] += k; }

static int harvest(GsContext* c, TimingSlot& sl) {
    if (!sl.pending) return GS_OK;
    sl.pending = false;
    if (sl.tags.size() < 2) return GS_OK;
    CK(cudaEventSynchronize(sl.ev[sl.tags.size() - 1]));
    for (size_t m = 0; m + 1 < sl.tags.size(); m++) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, sl.ev[m], sl.ev[m + 1]));
        if (sl.tags[m] >= 0 && sl.tags[m] < GS_NUM_STAGES) c->stage_ms[sl.tags[m]] += ms;
    }
    for (int s = 0; s < GS_NUM_STAGES; s++) c->stage_launches[s] += sl.launches[s];
    c->timed_steps += 1;
    return GS_OK;
}

// Starts recording a step's marks into the next ring slot (direct enqueue) or into the
// capture event list (graph capture).
static int begin_record(GsContext* c) {
    c->rec_tags.clear();
    for (int s = 0; s < GS_NUM_STAGES; s++) c->rec_launches[s] = 0;
    if (!c->capturing) {
        c->rec_slot = c->slot_next;
        c->slot_next = (c->slot_next + 1) % 4;
        CKI(harvest(c, c->slots[c->rec_slot]));
    }
    return GS_OK;
}

static int end_record(GsContext* c) {
    CKI(mark(c, ST_END));
    int64_t total = 0;
    for (int s = 0; s < GS_NUM_STAGES; s++) total += c->rec_launches[s];
    c->last_step_launches = total;
    if (!c->capturing && c->stage_timing && c->rec_slot >= 0) {
        TimingSlot& sl = c->slots[c->rec_slot];
        sl.tags = c->rec_tags;
        for (int s = 0; s < GS_NUM_STAGES; s++) sl.launches[s] = c->rec_launches[s];
        sl.pending = true;
    }
    c->rec_slot = -1;
    return GS_OK;
}

// ---------------------------------------------------------------------------------
// Views and layout.
// ---------------------------------------------------------------------------------
static ViewDesc make_desc(const GsCamera& cam, int tile) {
    ViewDesc d;
    memset(&d, 0, sizeof d);
    const float* m = cam.view;
    d.R[0] = m[0]; d.R[1] = m[1]; d.R[2] = m[2];
    d.R[3] = m[4]; d.R[4] = m[5]; d.R[5] = m[6];
    d.R[6] = m[8]; d.R[7] = m[9]; d.R[8] = m[10];
    d.t[0] = m[3]; d.t[1] = m[7]; d.t[2] = m[11];
    d.fx = cam.fx; d.fy = cam.fy; d.cx = cam.cx; d.cy = cam.cy;
    // C = -R^T t (trainer/colmap.js:67-71).
    for (int j = 0; j < 3; j++) d.campos[j] = -(d.R[0 * 3 + j] * d.t[0] + d.R[1 * 3 + j] * d.t[1] + d.R[2 * 3 + j] * d.t[2]);
    d.width = cam.width;
    d.height = cam.height;
    d.tile = tile;
    d.tiles_x = (cam.width + tile - 1) / tile;
    d.tiles_y = (cam.height + tile - 1) / tile;
    d.loss_blocks_x = (cam.width + loss_block_w() - 1) / loss_block_w();
    d.loss_blocks_y = (cam.height + loss_block_h() - 1) / loss_block_h();
    return d;
}

static int valid_camera(const GsCamera& cam) {
    if (cam.width <= 0 || cam.height <= 0 || cam.width > 16384 || cam.height > 16384) return 0;
    for (int k = 0; k < 12; k++)
        if (!std::isfinite(cam.view[k])) return 0;
    return std::isfinite(cam.fx) && std::isfinite(cam.fy) && std::isfinite(cam.cx) && std::isfinite(cam.cy);
}

// Lays out views [0, V] (V = scratch) and sizes the per-pixel and per-tile buffers.
static int layout(GsContext* c) {
    c->vdesc.resize(c->cams.size());
    int64_t pix = 0, tiles = 0, lb = 0;
    for (size_t v = 0; v < c->cams.size(); v++) {
        ViewDesc d = make_desc(c->cams[v], c->tile);
        d.tile_offset = (int)tiles;
        d.pixel_offset = (int)pix;
        d.loss_block_offset = (int)lb;
        tiles += (int64_t)d.tiles_x * d.tiles_y;
        pix += (int64_t)d.width * d.height;
        lb += (int64_t)d.loss_blocks_x * d.loss_blocks_y;
        c->vdesc[v] = d;
    }
    if (pix > 0x7fffffffLL || tiles > 0x7fffffffLL) return fail(GS_ERR_INVALID_ARG, "views too large");
    c->total_pixels = pix;
    c->total_tiles = tiles;
    c->total_loss_blocks = lb;
    int bits = 1;
    while ((1LL << bits) < tiles) bits++;
    c->tile_bits = bits;
    CKI(ensure(c->views_d, sizeof(ViewDesc) * (GS_MAX_VIEWS + 1), c));
    CK(cudaMemcpyAsync(c->views_d.p, c->vdesc.data(), sizeof(ViewDesc) * c->vdesc.size(), cudaMemcpyHostToDevice,
                       c->stream));
    CKI(ensure(c->image, (size_t)pix * 12, c));
    CKI(ensure(c->dl, (size_t)pix * 12, c));
    CKI(ensure(c->t_final, (size_t)pix * 4, c));
    CKI(ensure(c->last, (size_t)pix * 4, c));
    CKI(ensure(c->ranges, (size_t)tiles * 8, c));
    CKI(ensure(c->tile_order, (size_t)tiles * 4, c));
    return GS_OK;
}

static int set_scratch_camera(GsContext* c, const GsCamera& cam) {
    if (!valid_camera(cam)) return fail(GS_ERR_INVALID_ARG, "invalid camera");
    if ((int)c->cams.size() == c->V + 1) {
        const GsCamera& old = c->cams[c->V];
        if (memcmp(&old, &cam, sizeof cam) == 0) return GS_OK;
        c->cams[c->V] = cam;
    } else {
        c->cams.resize(c->V);
        c->cams.push_back(cam);
    }
    c->target_kind.resize(c->V + 1, 0);
    c->target_kind[c->V] = 0;
    c->inst_cap_valid = false;
    return layout(c);
}

// Pair buffers for `views` view slots and the segment table.
static int size_pairs(GsContext* c, int views) {
    const int64_t pairs = (int64_t)std::max(views, 1) * c->n_pad;
    if (pairs > 0x7fffffffLL) return fail(GS_ERR_INVALID_ARG, "too many (view, Gaussian) pairs");
    if (pairs > c->pair_cap) {
        CKI(ensure(c->geo0, (size_t)pairs * 16, c));
        CKI(ensure(c->geo1, (size_t)pairs * 16, c));
        CKI(ensure(c->rgb, (size_t)pairs * 16, c));
        CKI(ensure(c->erec, (size_t)pairs * sizeof(EmitRec), c));
        CKI(ensure(c->pcount, (size_t)pairs * 4, c));
        CKI(ensure(c->pkeys, (size_t)pairs * 4, c));
        CKI(ensure(c->pvals, (size_t)pairs * 4, c));
        CKI(ensure(c->pkeys_alt, (size_t)pairs * 4, c));
        CKI(ensure(c->pvals_alt, (size_t)pairs * 4, c));
        CKI(ensure(c->sg8, (size_t)pairs * 32, c));
        CKI(ensure(c->sg1, (size_t)pairs * 4, c));
        CKI(ensure(c->block_sums, (size_t)(pairs / emit_chunk_items() + 2) * 4, c));
        CKI(ensure(c->pair_offsets, (size_t)pairs * 4, c));
        c->pair_cap = pairs;
        const int64_t parts = (std::max(pairs, c->inst_cap) + radix_tile_items() - 1) / radix_tile_items() + 1;
        CKI(ensure(c->hist, (size_t)parts * 256 * 8, c));
        // Zeroed once; every backward re-zeroes the slots it uses.
        CK(cudaMemsetAsync(c->sg8.p, 0, c->sg8.bytes, c->stream));
        CK(cudaMemsetAsync(c->sg1.p, 0, c->sg1.bytes, c->stream));
    }
    return GS_OK;
}

static int write_segments(GsContext* c) {
    std::vector<SegInfo> h(SEG_COUNT);
    memset(h.data(), 0, sizeof(SegInfo) * SEG_COUNT);
    for (int k = 0; k <= GS_MAX_VIEWS; k++) h[SEG_ALL + k] = SegInfo{0u, (unsigned)(k * c->n_pad)};
    for (int s = 0; s < GS_MAX_VIEWS; s++) h[SEG_PAIR + s] = SegInfo{(unsigned)(s * c->n_pad), (unsigned)c->n_pad};
    CKI(ensure(c->segs, sizeof(SegInfo) * SEG_COUNT, c));
    CK(cudaMemcpyAsync(c->segs.p, h.data(), sizeof(SegInfo) * SEG_COUNT, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return GS_OK;
}

static int size_instances(GsContext* c, int64_t cap) {
    if (cap > 0xfffff000LL) cap = 0xfffff000LL;  // instance positions are 32-bit
    if (cap <= c->inst_cap) return GS_OK;
    CKI(ensure(c->ikeys, (size_t)cap * 4, c));
    CKI(ensure(c->ivals, (size_t)cap * 4, c));
    CKI(ensure(c->ikeys_alt, (size_t)cap * 4, c));
    CKI(ensure(c->ivals_alt, (size_t)cap * 4, c));
    CKI(ensure(c->block_first_pair, (size_t)(cap / emit_out_items() + 2) * 4, c));
    c->inst_cap = cap;
    const int64_t parts = (std::max(c->pair_cap, c->inst_cap) + radix_tile_items() - 1) / radix_tile_items() + 1;
    CKI(ensure(c->hist, (size_t)parts * 256 * 8, c));
    return GS_OK;
}

// ---------------------------------------------------------------------------------
// Pipeline stages (enqueue only).
// ---------------------------------------------------------------------------------
static SegInfo* seg_ptr(GsContext* c, int idx) { return c->segs.as<SegInfo>() + idx; }

static int persistent_ctas(GsContext* c, bool backward) {
    const int per_sm = backward ? raster_max_ctas_per_sm(c->tile, c->wt_bwd, c->batch_bwd, c->ppt_bwd, true)
                                : raster_max_ctas_per_sm(c->tile, c->wt_fwd, c->batch_fwd, c->ppt_fwd, false);
    return c->num_sms * per_sm;
}

static RasterArgs raster_args(GsContext* c, int first, int count) {
    RasterArgs r;
    memset(&r, 0, sizeof r);
    r.views = c->views_d.as<ViewDesc>();
    r.view_first = first;
    r.num_views = count;
    r.tile_first = c->vdesc[first].tile_offset;
    const ViewDesc& lastv = c->vdesc[first + count - 1];
    r.num_tiles = lastv.tile_offset + lastv.tiles_x * lastv.tiles_y - r.tile_first;
    r.pixel_first = c->vdesc[first].pixel_offset;
    r.ranges = c->ranges.as<uint2>();
    r.inst_pair = c->ivals.as<uint32_t>();
    r.geo0 = c->geo0.as<float4>();
    r.geo1 = c->geo1.as<float4>();
    r.rgb = c->rgb.as<float4>();
    r.alpha_max = c->cfg.alpha_max;
    r.alpha_min = c->cfg.alpha_min;
    r.t_min = c->cfg.t_min;
    r.image = c->image.as<float>();
    r.t_final = c->t_final.as<float>();
    r.last = c->last.as<uint32_t>();
    r.dl = c->dl.as<float>();
    r.sg8 = c->sg8.as<float4>();
    r.sg1 = c->sg1.as<float>();
    return r;
}

// Start of a forward over views [first, first + count): clear the per-forward counters
// and the tile ranges.
static int forward_begin(GsContext* c, int first, int count) {
    CKI(mark(c, ST_OTHER));
    CK(cudaMemsetAsync(c->status.p, 0, GS_STATUS_FORWARD_BYTES, c->stream));
    CK(cudaMemsetAsync(c->visible.p, 0, sizeof(unsigned) * (GS_MAX_VIEWS + 1), c->stream));
    const ViewDesc& a = c->vdesc[first];
    const ViewDesc& b = c->vdesc[first + count - 1];
    const int64_t t0 = a.tile_offset, t1 = b.tile_offset + (int64_t)b.tiles_x * b.tiles_y;
    CK(cudaMemsetAsync(c->ranges.as<uint2>() + t0, 0, (size_t)(t1 - t0) * 8, c->stream));
    return GS_OK;
}

// Projection, binning and blending of views [vfirst, vfirst + vcount) of a step that
// starts at view step_first: all of them in one batch (one launch per stage, persistent
// raster), or one view (slot vfirst - step_first, its own sort segments).
static int forward_group(GsContext* c, int step_first, int vfirst, int vcount, bool batched) {
    DevStatus* st = c->status.as<DevStatus>();
    const int slot = vfirst - step_first;
    unsigned* visible = c->visible.as<unsigned>() + (batched ? 0 : 1 + slot);
    SegInfo* pair_seg = batched ? seg_ptr(c, SEG_ALL + vcount) : seg_ptr(c, SEG_PAIR + slot);
    SegInfo* inst_seg = batched ? seg_ptr(c, SEG_INST_ALL) : seg_ptr(c, SEG_INST + slot);
    const SegInfo* prev_seg = (!batched && slot > 0) ? seg_ptr(c, SEG_INST + slot - 1) : nullptr;
    // Projection.
    CKI(mark(c, ST_PROJECT));
    ProjectArgs pa;
    memset(&pa, 0, sizeof pa);
    pa.params = c->params.as<float>();
    pa.n = c->n;
    pa.n_pad = c->n_pad;
    pa.degree = c->degree;
    pa.views = c->views_d.as<ViewDesc>();
    pa.view_first = vfirst;
    pa.num_views = vcount;
    pa.pair_slot_first = slot;
    pa.near_plane = c->cfg.near_plane;
    pa.dilation = c->cfg.cov_dilation;
    pa.rect_mode = c->cfg.rect_mode;
    pa.geo0 = c->geo0.as<float4>();
    pa.geo1 = c->geo1.as<float4>();
    pa.rgb = c->rgb.as<float4>();
    pa.keys = c->pkeys.as<uint32_t>();
    pa.visible = visible;
    pa.tile_cull = c->cfg.tile_cull;
    pa.alpha_min = c->cfg.alpha_min;
    pa.pcount = c->pcount.as<uint32_t>();
    pa.erec = c->erec.as<EmitRec>();
    pa.stats_cnt = c->stats_active ? step_stats(c) + c->n_pad : nullptr;
    launch_project_fwd(pa, c->stream);
    count_launches(c, ST_PROJECT, 1);
    // Depth sort of the pairs (31 bits: depths are positive, the sentinel is 0x7fffffff).
    CKI(mark(c, ST_SORT_PAIRS));
    RadixSortArgs ra;
    ra.keys = c->pkeys.as<uint32_t>();
    ra.vals = c->pvals.as<uint32_t>();
    ra.keys_alt = c->pkeys_alt.as<uint32_t>();
    ra.vals_alt = c->pvals_alt.as<uint32_t>();
    ra.iota = 1;
    ra.seg = pair_seg;
    ra.begin_bit = 0;
    ra.end_bit = 31;
    ra.discard_keys = true;  // the emission reads the sorted pairs only
    ra.hist = c->hist.as<unsigned long long>();
    ra.totals = c->totals.as<uint32_t>();
    ra.timeout = &c->status.as<DevStatus>()->sort_timeout;
    ra.debug_wait = &c->status.as<DevStatus>()->debug_wait;
    ra.never_set = &c->status.as<DevStatus>()->never_set;
    ra.max_parts = (int)(((int64_t)vcount * c->n_pad + radix_tile_items() - 1) / radix_tile_items());
    launch_radix_sort(ra, c->stream, c->num_sms);
    count_launches(c, ST_SORT_PAIRS, 1 + radix_sort_passes(0, 31));
    // Key instances in depth order.
    CKI(mark(c, ST_EMIT));
    EmitArgs ea;
    memset(&ea, 0, sizeof ea);
    ea.sorted_pairs = c->pvals.as<uint32_t>();
    ea.pair_seg = pair_seg;
    ea.visible = visible;
    ea.pcount = c->pcount.as<uint32_t>();
    ea.erec = c->erec.as<EmitRec>();
    ea.views = c->views_d.as<ViewDesc>();
    ea.view_first = step_first;  // pair / n_pad is the slot relative to the step's first view
    ea.n_pad = c->n_pad;
    ea.block_sums = c->block_sums.as<uint32_t>();
    ea.pair_offsets = c->pair_offsets.as<uint32_t>();
    ea.block_first_pair = c->block_first_pair.as<uint32_t>();
    ea.inst_seg = inst_seg;
    ea.prev_seg = prev_seg;
    ea.inst_keys = c->ikeys.as<uint32_t>();
    ea.inst_vals = c->ivals.as<uint32_t>();
    ea.capacity = (unsigned long long)c->inst_cap;
    ea.status = st;
    ea.max_chunks = (int)((int64_t)vcount * c->n_pad / emit_chunk_items() + 1);
    launch_emit(ea, c->stream, c->num_sms);
    count_launches(c, ST_EMIT, 4);
    // Stable sort by tile id; its last pass bounds the tile ranges.
    CKI(mark(c, ST_SORT_INST));
    RadixSortArgs rb = ra;
    rb.keys = c->ikeys.as<uint32_t>();
    rb.vals = c->ivals.as<uint32_t>();
    rb.keys_alt = c->ikeys_alt.as<uint32_t>();
    rb.vals_alt = c->ivals_alt.as<uint32_t>();
    rb.iota = 0;
    rb.seg = inst_seg;
    rb.begin_bit = 0;
    rb.end_bit = c->tile_bits;
    rb.max_parts = (int)((c->inst_cap + radix_tile_items() - 1) / radix_tile_items());
    rb.ranges = c->ranges.as<uint2>();
    launch_radix_sort(rb, c->stream, c->num_sms);
    RasterArgs r = raster_args(c, vfirst, vcount);
    launch_ranges_finish(c->ranges.as<uint2>() + r.tile_first, r.num_tiles, c->stream);
    count_launches(c, ST_SORT_INST, 1 + radix_sort_passes(0, c->tile_bits) + 1);
    // Blend.
    if (batched) {
        if (c->cfg.lpt_order) {
            launch_tile_order(c->ranges.as<uint2>(), r.tile_first, r.num_tiles, c->tile_order.as<uint32_t>(), nullptr,
                              c->stream);
            count_launches(c, ST_SORT_INST, 1);
            r.tile_order = c->tile_order.as<uint32_t>();
        }
        r.work_counter = &st->work_counter;
    }
    CKI(mark(c, ST_RASTER_FWD));
    launch_raster_fwd(r, c->tile, c->wt_fwd, c->batch_fwd, c->ppt_fwd, batched ? c->ctas_fwd : 0, c->stream);
    count_launches(c, ST_RASTER_FWD, 1);
    CK(cudaGetLastError());
    return GS_OK;
}

static int enqueue_forward(GsContext* c, int first, int count, bool batched) {
    CKI(forward_begin(c, first, count));
    if (batched) return forward_group(c, first, first, count, true);
    for (int v = first; v < first + count; v++) CKI(forward_group(c, first, v, 1, false));
    return GS_OK;
}

static int enqueue_loss_view(GsContext* c, int first, int count, const GsLossConfig& lc, int kind) {
    CKI(mark(c, ST_LOSS));
    LossArgs la;
    memset(&la, 0, sizeof la);
    la.views = c->views_d.as<ViewDesc>();
    la.view_first = first;
    la.num_views = count;
    la.block_first = c->vdesc[first].loss_block_offset;
    const ViewDesc& lv = c->vdesc[first + count - 1];
    la.num_blocks = lv.loss_block_offset + lv.loss_blocks_x * lv.loss_blocks_y - la.block_first;
    la.image = c->image.as<float>();
    la.target_u8 = kind == 1 ? c->target_u8.as<uint8_t>() : nullptr;
    la.target_f32 = kind == 2 ? c->target_f32.as<float>() : nullptr;
    la.dl = c->dl.as<float>();
    la.lambda = lc.ssim_lambda;
    la.window = lc.window;
    la.acc = c->acc.as<double>();
    launch_loss(la, c->stream);
    count_launches(c, ST_LOSS, 1);
    return GS_OK;
}

static int enqueue_backward_view(GsContext* c, int first, int step_first, int count, bool batched, bool accumulate) {
    DevStatus* st = c->status.as<DevStatus>();
    const int slot = first - step_first;
    CKI(mark(c, ST_RASTER_BWD));
    CK(cudaMemsetAsync(c->sg8.as<float4>() + (size_t)slot * c->n_pad * 2, 0, (size_t)count * c->n_pad * 32, c->stream));
    CK(cudaMemsetAsync(c->sg1.as<float>() + (size_t)slot * c->n_pad, 0, (size_t)count * c->n_pad * 4, c->stream));
    RasterArgs r = raster_args(c, first, count);
    if (batched) {
        CK(cudaMemsetAsync(&st->work_counter_bwd, 0, 4, c->stream));
        r.work_counter = &st->work_counter_bwd;
        if (c->cfg.lpt_order) r.tile_order = c->tile_order.as<uint32_t>();
    }
    launch_raster_bwd(r, c->tile, c->wt_bwd, c->batch_bwd, c->ppt_bwd, batched ? c->ctas_bwd : 0, c->stream);
    count_launches(c, ST_RASTER_BWD, 1);
    CKI(mark(c, ST_PROJECT_BWD));
    ProjectBwdArgs pb;
    memset(&pb, 0, sizeof pb);
    pb.params = c->params.as<float>();
    pb.n = c->n;
    pb.n_pad = c->n_pad;
    pb.degree = c->degree;
    pb.views = c->views_d.as<ViewDesc>();
    pb.view_first = first;
    pb.num_views = count;
    pb.pair_slot_first = slot;
    pb.dilation = c->cfg.cov_dilation;
    pb.sg8 = c->sg8.as<float4>();
    pb.sg1 = c->sg1.as<float>();
    pb.grads = c->grads.as<float>();
    pb.accumulate = accumulate ? 1 : 0;
    pb.stats_sum = c->stats_active ? step_stats(c) : nullptr;
    launch_project_bwd(pb, c->stream);
    count_launches(c, ST_PROJECT_BWD, 1);
    CK(cudaGetLastError());
    return GS_OK;
}

static void fill_lrs(GsContext* c, const GsAdamConfig& ad, float* lr) {
    for (int j = 0; j < GS_MAX_PLANES; j++) lr[j] = 0.f;
    for (int j = 0; j < 3; j++) lr[j] = ad.lr_mean;
    for (int j = 3; j < 6; j++) lr[j] = ad.lr_scale;
    for (int j = 6; j < 10; j++) lr[j] = ad.lr_rotation;
    lr[10] = ad.lr_opacity;
    for (int j = 11; j < 14; j++) lr[j] = ad.lr_color;
    for (int j = 14; j < c->planes; j++) lr[j] = ad.lr_sh;
}

// The whole training step (no host synchronisation inside).

static void fill_adam_args(GsContext* c, const GsAdamConfig& ad, AdamArgs& aa) {
    memset(&aa, 0, sizeof aa);
    aa.params = c->params.as<float>();
    aa.grads = c->grads.as<float>();
    aa.m = c->mom1.as<float>();
    aa.v = c->mom2.as<float>();
    aa.n = c->n;
    aa.n_pad = c->n_pad;
    aa.planes = c->planes;
    fill_lrs(c, ad, aa.lr);
    aa.beta1 = ad.beta1;
    aa.beta2 = ad.beta2;
    aa.eps = ad.eps;
    aa.status = c->status.as<DevStatus>();
}

// phase 0: the whole step; phase 1: forward, loss and backward only, then the gradient
// buffer's tail (loss sum, overflow, views) for a cross-replica reduction.
static int enqueue_step(GsContext* c, const GsAdamConfig& ad, const GsLossConfig& lc, int first, int count,
                        bool batched, int kind, int phase = 0) {
    CK(cudaMemsetAsync(c->acc.p, 0, sizeof(double) * 2 * (GS_MAX_VIEWS + 1), c->stream));
    if (c->stats_on) CK(cudaMemsetAsync(step_stats(c), 0, (size_t)2 * c->n_pad * 4, c->stream));
    struct StatsScope {
        GsContext* c;
        ~StatsScope() { c->stats_active = false; }
    } stats_scope{c};
    c->stats_active = c->stats_on;
    if (batched) {
        CKI(enqueue_forward(c, first, count, true));
        CKI(enqueue_loss_view(c, first, count, lc, kind));
        CKI(enqueue_backward_view(c, first, first, count, true, false));
    } else {
        // One view at a time: forward, loss and backward of a view before the next.
        CKI(forward_begin(c, first, count));
        for (int v = first; v < first + count; v++) {
            CKI(forward_group(c, first, v, 1, false));
            CKI(enqueue_loss_view(c, v, 1, lc, kind));
            CKI(enqueue_backward_view(c, v, first, 1, false, v > first));
        }
    }
    c->stats_active = false;
    if (phase == 1) {
        launch_grad_tail(c->status.as<DevStatus>(), c->acc.as<double>(), c->views_d.as<ViewDesc>(), first, count,
                         lc.ssim_lambda, lc.window, grad_tail(c), c->stream);
        count_launches(c, ST_PROJECT_BWD, 1);
        CK(cudaGetLastError());
        return GS_OK;
    }
    CKI(mark(c, ST_ADAM));
    AdamArgs aa;
    fill_adam_args(c, ad, aa);
    launch_adam(aa, c->stream);
    if (c->stats_on) {
        launch_stats_commit(c->stats.as<float>(), step_stats(c), c->n_pad, c->status.as<DevStatus>(), nullptr,
                            c->stream);
        count_launches(c, ST_ADAM, 1);
    }
    launch_step_end(c->status.as<DevStatus>(), c->acc.as<double>(), c->views_d.as<ViewDesc>(), first, count,
                    lc.ssim_lambda, lc.window, 1, c->stream);
    count_launches(c, ST_ADAM, 2);
    CK(cudaGetLastError());
    return GS_OK;
}

// ---------------------------------------------------------------------------------
// Graphs.
// ---------------------------------------------------------------------------------
static void drop_graph(StepGraph& g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g.exec = nullptr;
    g.graph = nullptr;
}

static void drop_graphs(GsContext* c) {
    for (auto& kv : c->graphs) drop_graph(kv.second);
    c->graphs.clear();
}

static int capture_step(GsContext* c, StepGraph& g, const GsAdamConfig& ad, const GsLossConfig& lc, int first,
                        int count, bool batched, int kind, int phase = 0) {
    drop_graph(g);
    // Events used by the capture are created before it starts.
    while (c->capture_events.size() < 1024) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        c->capture_events.push_back(e);
    }
    c->capturing = true;
    CKI(begin_record(c));
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) {
        c->capturing = false;
        return fail(GS_ERR_CUDA, "cudaStreamBeginCapture failed: %s", cudaGetErrorString(e));
    }
    int rc = enqueue_step(c, ad, lc, first, count, batched, kind, phase);
    if (rc == GS_OK) rc = end_record(c);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(c->stream, &graph);
    c->capturing = false;
    if (rc != GS_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return fail(GS_ERR_CUDA, "cudaStreamEndCapture failed: %s", cudaGetErrorString(e));
    g.graph = graph;
    g.tags = c->rec_tags;
    for (int s = 0; s < GS_NUM_STAGES; s++) g.launches[s] = c->rec_launches[s];
    // Map each timing mark to its event-record node.
    g.nodes.assign(g.tags.size(), nullptr);
    if (c->stage_timing && !g.tags.empty()) {
        size_t num = 0;
        CK(cudaGraphGetNodes(graph, nullptr, &num));
        std::vector<cudaGraphNode_t> nodes(num);
        CK(cudaGraphGetNodes(graph, nodes.data(), &num));
        for (size_t k = 0; k < num; k++) {
            cudaGraphNodeType t;
            CK(cudaGraphNodeGetType(nodes[k], &t));
            if (t != cudaGraphNodeTypeEventRecord) continue;
            cudaEvent_t ev;
            CK(cudaGraphEventRecordNodeGetEvent(nodes[k], &ev));
            for (size_t m = 0; m < g.tags.size(); m++)
                if (c->capture_events[m] == ev) g.nodes[m] = nodes[k];
        }
        for (size_t m = 0; m < g.tags.size(); m++)
            if (!g.nodes[m]) return fail(GS_ERR_CUDA, "timing mark %zu has no graph node", m);
    }
    CK(cudaGraphInstantiate(&g.exec, graph, 0));
    g.generation = c->generation;
    return GS_OK;
}

static int launch_graph(GsContext* c, StepGraph& g) {
    if (c->stage_timing && !g.tags.empty()) {
        const int slot = c->slot_next;
        c->slot_next = (c->slot_next + 1) % 4;
        TimingSlot& sl = c->slots[slot];
        CKI(harvest(c, sl));
        while (sl.ev.size() < g.tags.size()) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            sl.ev.push_back(e);
        }
        for (size_t m = 0; m < g.tags.size(); m++) CK(cudaGraphExecEventRecordNodeSetEvent(g.exec, g.nodes[m], sl.ev[m]));
        sl.tags = g.tags;
        for (int s = 0; s < GS_NUM_STAGES; s++) sl.launches[s] = g.launches[s];
        CK(cudaGraphLaunch(g.exec, c->stream));
        sl.pending = true;
    } else {
        CK(cudaGraphLaunch(g.exec, c->stream));
    }
    int64_t total = 0;
    for (int s = 0; s < GS_NUM_STAGES; s++) total += g.launches[s];
    c->last_step_launches = total;
    return GS_OK;
}

// ---------------------------------------------------------------------------------
// Capacity: the first forward of a scene/view set measures the key instances it needs.
// ---------------------------------------------------------------------------------
// A radix look-back wait that gave up: the step that saw it skipped its update (its
// tile lists may be wrong).  The flag is cleared once reported, so the context goes on
// with the next call.
static int sort_timed_out(GsContext* c) {
    c->status_host->sort_timeout = 0;
    CK(cudaMemsetAsync(&c->status.as<DevStatus>()->sort_timeout, 0, sizeof(unsigned int), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return fail(GS_ERR_CUDA, "radix sort look-back wait timed out; the step's update was skipped");
}

static int read_status(GsContext* c) {
    CK(cudaMemcpyAsync(c->status_host, c->status.p, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (c->status_host->sort_timeout) return sort_timed_out(c);
    return GS_OK;
}

static int grow_instances(GsContext* c, unsigned long long needed) {
    int64_t cap = (int64_t)(needed + needed / 4) + (1 << 20);
    CKI(size_instances(c, cap));
    drop_graphs(c);
    return GS_OK;
}

static int ensure_capacity(GsContext* c, int first, int count) {
    if (c->inst_cap_valid) return GS_OK;
    if (c->cfg.instance_capacity > 0) {
        CKI(size_instances(c, c->cfg.instance_capacity));
        c->inst_cap_valid = true;
        return GS_OK;
    }
    if (c->inst_cap < (1 << 20)) CKI(size_instances(c, 1 << 20));
    for (int tries = 0; tries < 4; tries++) {
        CKI(enqueue_forward(c, first, count, true));
        CKI(read_status(c));
        if (!c->status_host->overflow) {
            const unsigned long long need = c->status_host->instances_needed;
            if ((int64_t)(need + need / 8) > c->inst_cap) CKI(grow_instances(c, need));
            c->inst_cap_valid = true;
            return GS_OK;
        }
        CKI(grow_instances(c, c->status_host->instances_needed));
    }
    return fail(GS_ERR_CAPACITY, "key instance buffer could not be sized");
}

// ---------------------------------------------------------------------------------
// C ABI.
// ---------------------------------------------------------------------------------
#define CTX_CHECK(c)                                                            \
    do {                                                                        \
        if (!(c)) return fail(GS_ERR_INVALID_ARG, "null context");              \
        CK(cudaSetDevice((c)->device));                                         \
    } while (0)

extern "C" {

void gs_config_default(GsConfig* cfg) {
    if (!cfg) return;
    memset(cfg, 0, sizeof *cfg);
    cfg->near_plane = 0.2f;
    cfg->cov_dilation = 0.3f;
    cfg->alpha_max = 0.99f;
    cfg->alpha_min = 1.0f / 255.0f;
    cfg->t_min = 1e-4f;
    cfg->sh_degree = 0;
    cfg->rect_mode = 0;
    cfg->batched = 1;
    cfg->use_graph = 1;
    cfg->device = 0;
    cfg->autotune = 0;
    cfg->raster_batch = 256;
    cfg->raster_ppt = 0;
    cfg->tile_cull = 1;
    cfg->tile_size = GS_TILE;
    cfg->lpt_order = 1;
}

void gs_adam_default(GsAdamConfig* a) {
    if (!a) return;
    a->lr_color = 0.025f;
    a->lr_opacity = 0.05f;
    a->lr_mean = 0.002f;
    a->lr_scale = 0.005f;
    a->lr_rotation = 0.001f;
    a->lr_sh = 0.025f / 20.0f;
    a->beta1 = 0.9f;
    a->beta2 = 0.999f;
    a->eps = 1e-8f;
}

const char* gs_last_error(void) { return g_err.c_str(); }

const char* gs_status_string(int status) {
    switch (status) {
        case GS_OK: return "ok";
        case GS_ERR_INVALID_ARG: return "invalid argument";
        case GS_ERR_CUDA: return "CUDA error";
        case GS_ERR_CAPACITY: return "capacity exceeded";
        case GS_ERR_NO_DEVICE: return "no CUDA device";
        case GS_ERR_STATE: return "call out of order";
        case GS_ERR_NONFINITE: return "non-finite value";
        case GS_ERR_COMM: return "data-parallel exchange failed";
        default: return "unknown status";
    }
}

int gs_param_stride(int sh_degree) {
    if (sh_degree < 0 || sh_degree > 3) return -1;
    return num_planes(sh_degree);
}

const char* gs_stage_name(int32_t stage) {
    if (stage < 0 || stage >= GS_NUM_STAGES) return "";
    return kStageNames[stage];
}

int gs_create(const GsConfig* cfg_in, GsContext** out) {
    GS_TRACE("gs_create");
    if (!out) return fail(GS_ERR_INVALID_ARG, "out is null");
    *out = nullptr;
    GsConfig cfg;
    if (cfg_in) cfg = *cfg_in;
    else gs_config_default(&cfg);
    if (cfg.sh_degree < 0 || cfg.sh_degree > 3) return fail(GS_ERR_INVALID_ARG, "sh_degree must be 0..3");
    if (cfg.rect_mode < 0 || cfg.rect_mode > 1) return fail(GS_ERR_INVALID_ARG, "rect_mode must be 0 or 1");
    if (cfg.raster_batch != 32 && cfg.raster_batch != 64 && cfg.raster_batch != 128 && cfg.raster_batch != 256)
        return fail(GS_ERR_INVALID_ARG, "raster_batch must be 32, 64, 128 or 256");
    if (cfg.tile_size == 0) cfg.tile_size = GS_TILE;
    if (cfg.raster_ppt == 0) cfg.raster_ppt = cfg.tile_size == 8 ? 2 : 4;
    if (cfg.tile_size != 8 && cfg.tile_size != 16 && cfg.tile_size != 32 && cfg.tile_size != 64)
        return fail(GS_ERR_INVALID_ARG, "tile_size must be 8, 16, 32 or 64");
    if (cfg.raster_work_tile == 0) cfg.raster_work_tile = cfg.tile_size == 64 ? 16 : cfg.tile_size;
    if (!raster_variant_ok(cfg.tile_size, cfg.raster_work_tile, cfg.raster_ppt))
        return fail(GS_ERR_INVALID_ARG,
                    "no raster variant with %d pixels per thread and %d-pixel work tiles for %d-pixel tiles "
                    "(8: 2 px, work tile 8; 16: 2, 4 or 8 px, work tile 16; 32: 2, 4 or 8 px, work tile 32 or 16; "
                    "64: 2, 4 or 8 px, work tile 16)",
                    cfg.raster_ppt, cfg.raster_work_tile, cfg.tile_size);
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(GS_ERR_NO_DEVICE, "no CUDA device: %s", e == cudaSuccess ? "count is 0" : cudaGetErrorString(e));
    }
    if (cfg.device < 0 || cfg.device >= count) return fail(GS_ERR_INVALID_ARG, "device %d out of range", cfg.device);
    CK(cudaSetDevice(cfg.device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, cfg.device));
    if (prop.major < 10) return fail(GS_ERR_NO_DEVICE, "device %s is sm_%d%d; this build targets sm_100a", prop.name, prop.major, prop.minor);
    GsContext* c = new GsContext();
    c->cfg = cfg;
    c->device = cfg.device;
    c->num_sms = prop.multiProcessorCount;
    c->device_name = prop.name;
    c->degree = cfg.sh_degree;
    c->planes = num_planes(cfg.sh_degree);
    c->tile = cfg.tile_size;
    c->batch_fwd = c->batch_bwd = cfg.raster_batch;
    c->ppt_fwd = c->ppt_bwd = cfg.raster_ppt;
    c->wt_fwd = c->wt_bwd = cfg.raster_work_tile;
    int rc = GS_OK;
    auto bail = [&](int r) {
        gs_destroy(c);
        return r;
    };
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(GS_ERR_CUDA, "cudaStreamCreate failed"));
    if (loss_prepare() != cudaSuccess) return bail(fail(GS_ERR_CUDA, "loss kernel attributes"));
    if (radix_prepare() != cudaSuccess) return bail(fail(GS_ERR_CUDA, "radix kernel attributes"));
    if ((rc = ensure(c->status, sizeof(DevStatus), c)) != GS_OK) return bail(rc);
    if ((rc = ensure(c->visible, sizeof(unsigned) * (GS_MAX_VIEWS + 1), c)) != GS_OK) return bail(rc);
    if ((rc = ensure(c->acc, sizeof(double) * 2 * (GS_MAX_VIEWS + 1), c)) != GS_OK) return bail(rc);
    if ((rc = ensure(c->totals, 16384, c)) != GS_OK) return bail(rc);
    if ((rc = ensure(c->views_d, sizeof(ViewDesc) * (GS_MAX_VIEWS + 1), c)) != GS_OK) return bail(rc);
    if (cudaMemset(c->status.p, 0, sizeof(DevStatus)) != cudaSuccess) return bail(fail(GS_ERR_CUDA, "memset"));
    if (cudaMallocHost((void**)&c->status_host, sizeof(DevStatus)) != cudaSuccess)
        return bail(fail(GS_ERR_CUDA, "cudaMallocHost failed"));
    memset(c->status_host, 0, sizeof(DevStatus));
    if (cudaEventCreateWithFlags(&c->status_event, cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(GS_ERR_CUDA, "cudaEventCreate failed"));
    for (int k = 0; k < 64; k++)
        if (cudaEventCreate(&c->user_events[k]) != cudaSuccess) return bail(fail(GS_ERR_CUDA, "cudaEventCreate failed"));
    c->ctas_fwd = persistent_ctas(c, false);
    c->ctas_bwd = persistent_ctas(c, true);
    *out = c;
    return GS_OK;
}

int gs_destroy(GsContext* c) {
    GS_TRACE("gs_destroy");
    if (!c) return GS_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graphs(c);
    dp_comm_destroy(c->dp_comm);
    c->dp_comm = nullptr;
    DevBuf* bufs[] = {&c->params, &c->grads, &c->mom1, &c->mom2, &c->views_d, &c->target_u8, &c->target_f32,
                      &c->image, &c->t_final, &c->last, &c->dl, &c->ranges, &c->tile_order, &c->geo0, &c->geo1,
                      &c->rgb, &c->erec, &c->pcount, &c->pkeys, &c->pvals, &c->pkeys_alt, &c->pvals_alt, &c->sg8, &c->sg1,
                      &c->ikeys, &c->ivals, &c->ikeys_alt, &c->ivals_alt, &c->hist, &c->totals, &c->block_sums,
                      &c->pair_offsets, &c->block_first_pair,
                      &c->segs, &c->visible, &c->acc, &c->scratch16, &c->status, &c->stats, &c->dn_scratch,
                      &c->nb_scratch, &c->stage[0], &c->stage[1]};
    for (DevBuf* b : bufs) release(*b);
    for (cudaEvent_t e : c->capture_events) cudaEventDestroy(e);
    for (auto& sl : c->slots)
        for (cudaEvent_t e : sl.ev) cudaEventDestroy(e);
    for (int k = 0; k < 64; k++)
        if (c->user_events[k]) cudaEventDestroy(c->user_events[k]);
    if (c->status_event) cudaEventDestroy(c->status_event);
    for (int k = 0; k < 2; k++) {
        if (c->ev_copied[k]) cudaEventDestroy(c->ev_copied[k]);
        if (c->ev_free[k]) cudaEventDestroy(c->ev_free[k]);
        if (c->ev_done[k]) cudaEventDestroy(c->ev_done[k]);
    }
    if (c->copy_stream) {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamDestroy(c->copy_stream);
    }
    if (c->status_host) cudaFreeHost(c->status_host);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return GS_OK;
}

// ---- scene ------------------------------------------------------------------------
// Sizes every per-Gaussian buffer for n Gaussians and clears gradients, moments and the
// densification statistics; pair buffers, capacities and graphs start over.  The Adam
// step counter is kept when keep_step (densification keeps training's t).
static int resize_scene(GsContext* c, int n, bool keep_step) {
    c->n = n;
    c->n_pad = ((n + 127) / 128) * 128;
    if (c->n_pad == 0) c->n_pad = 128;
    const size_t bytes = (size_t)c->planes * c->n_pad * 4;
    CKI(ensure(c->params, bytes, c));
    CKI(ensure(c->grads, grad_buffer_floats(c) * 4, c));
    CKI(ensure(c->mom1, bytes, c));
    CKI(ensure(c->mom2, bytes, c));
    CKI(ensure(c->stats, (size_t)2 * c->n_pad * 4, c));
    CK(cudaMemsetAsync(c->grads.p, 0, grad_buffer_floats(c) * 4, c->stream));
    CK(cudaMemsetAsync(c->mom1.p, 0, bytes, c->stream));
    CK(cudaMemsetAsync(c->mom2.p, 0, bytes, c->stream));
    CK(cudaMemsetAsync(c->stats.p, 0, (size_t)2 * c->n_pad * 4, c->stream));
    if (keep_step) CK(cudaMemsetAsync(c->status.p, 0, GS_STATUS_FORWARD_BYTES, c->stream));
    else CK(cudaMemsetAsync(c->status.p, 0, sizeof(DevStatus), c->stream));
    CKI(write_segments(c));
    c->pair_cap = 0;  // re-size pair buffers for the new n_pad
    CKI(size_pairs(c, std::max(c->V, 1)));
    c->inst_cap_valid = false;
    c->last_first = -1;
    c->have_loss = false;
    c->grads_pending = false;
    drop_graphs(c);
    return GS_OK;
}

static int upload_planes(GsContext* c, int n, const std::vector<float>& planes_host) {
    CKI(resize_scene(c, n, false));
    CK(cudaMemcpyAsync(c->params.p, planes_host.data(), (size_t)c->planes * c->n_pad * 4, cudaMemcpyHostToDevice,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return GS_OK;
}

int gs_set_gaussians(GsContext* c, int32_t n, const float* params) {
    GS_TRACE("gs_set_gaussians");
    CTX_CHECK(c);
    if (n < 0 || n > (1 << 28) || (n > 0 && !params)) return fail(GS_ERR_INVALID_ARG, "bad Gaussian count or pointer");
    const int P = c->planes;
    const int np = ((n + 127) / 128) * 128 > 0 ? ((n + 127) / 128) * 128 : 128;
    std::vector<float> h((size_t)P * np, 0.f);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < P; k++) h[(size_t)k * np + i] = params[(size_t)i * P + k];
    // Padding Gaussians: unit quaternion so nothing downstream divides by zero.
    for (int i = n; i < np; i++) h[(size_t)6 * np + i] = 1.f;
    return upload_planes(c, n, h);
}

int gs_set_gaussians_packed(GsContext* c, int32_t n, const float* packed) {
    GS_TRACE("gs_set_gaussians_packed");
    CTX_CHECK(c);
    if (n < 0 || n > (1 << 28) || (n > 0 && !packed)) return fail(GS_ERR_INVALID_ARG, "bad Gaussian count or pointer");
    const int P = c->planes;
    const int np = ((n + 127) / 128) * 128 > 0 ? ((n + 127) / 128) * 128 : 128;
    std::vector<float> h((size_t)P * np, 0.f);
    static const int slot_of_plane[14] = {0, 1, 2, 4, 5, 6, 8, 9, 10, 11, 7, 12, 13, 14};
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 14; k++) h[(size_t)k * np + i] = packed[(size_t)i * 16 + slot_of_plane[k]];
    for (int i = n; i < np; i++) h[(size_t)6 * np + i] = 1.f;
    return upload_planes(c, n, h);
}

static int download_planes(GsContext* c, const DevBuf& b, std::vector<float>& h) {
    h.resize((size_t)c->planes * c->n_pad);
    CK(cudaMemcpyAsync(h.data(), b.p, h.size() * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return GS_OK;
}

int gs_get_gaussians(GsContext* c, float* out) {
    CTX_CHECK(c);
    if (!out && c->n > 0) return fail(GS_ERR_INVALID_ARG, "out is null");
    if (c->n == 0) return GS_OK;
    std::vector<float> h;
    CKI(download_planes(c, c->params, h));
    const int P = c->planes;
    for (int i = 0; i < c->n; i++)
        for (int k = 0; k < P; k++) out[(size_t)i * P + k] = h[(size_t)k * c->n_pad + i];
    return GS_OK;
}

int gs_get_gaussians_packed(GsContext* c, float* out) {
    CTX_CHECK(c);
    if (!out && c->n > 0) return fail(GS_ERR_INVALID_ARG, "out is null");
    if (c->n == 0) return GS_OK;
    std::vector<float> h;
    CKI(download_planes(c, c->params, h));
    static const int slot_of_plane[14] = {0, 1, 2, 4, 5, 6, 8, 9, 10, 11, 7, 12, 13, 14};
    for (int i = 0; i < c->n; i++) {
        float* o = out + (size_t)i * 16;
        o[3] = 0.f;
        o[15] = 0.f;
        for (int k = 0; k < 14; k++) o[slot_of_plane[k]] = h[(size_t)k * c->n_pad + i];
    }
    return GS_OK;
}

int32_t gs_num_gaussians(const GsContext* c) { return c ? c->n : 0; }

// ---- views ------------------------------------------------------------------------
int gs_set_views(GsContext* c, int32_t num_views, const GsCamera* cams) {
    GS_TRACE("gs_set_views");
    CTX_CHECK(c);
    if (num_views < 0 || num_views > GS_MAX_VIEWS || (num_views > 0 && !cams))
        return fail(GS_ERR_INVALID_ARG, "num_views must be 0..%d", GS_MAX_VIEWS);
    for (int v = 0; v < num_views; v++)
        if (!valid_camera(cams[v])) return fail(GS_ERR_INVALID_ARG, "camera %d is invalid", v);
    CK(cudaStreamSynchronize(c->stream));
    c->cams.assign(cams, cams + num_views);
    c->V = num_views;
    c->target_kind.assign(num_views, 0);
    CKI(layout(c));
    if (c->n_pad > 0) CKI(size_pairs(c, std::max(num_views, 1)));
    c->inst_cap_valid = false;
    c->last_first = -1;
    c->have_loss = false;
    drop_graphs(c);
    CK(cudaStreamSynchronize(c->stream));
    return GS_OK;
}

static int check_view(GsContext* c, int v) {
    if (v < 0 || v >= c->V) return fail(GS_ERR_INVALID_ARG, "view %d out of range [0, %d)", v, c->V);
    return GS_OK;
}

int gs_set_target_u8(GsContext* c, int32_t view, const uint8_t* rgb) {
    CTX_CHECK(c);
    CKI(check_view(c, view));
    if (!rgb) return fail(GS_ERR_INVALID_ARG, "rgb is null");
    CKI(ensure(c->target_u8, (size_t)c->total_pixels * 3, c));
    const ViewDesc& d = c->vdesc[view];
    CK(cudaMemcpyAsync(c->target_u8.as<uint8_t>() + (size_t)d.pixel_offset * 3, rgb, (size_t)d.width * d.height * 3,
                       cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->target_kind[view] = 1;
    return GS_OK;
}

int gs_set_target_f32(GsContext* c, int32_t view, const float* rgb) {
    CTX_CHECK(c);
    CKI(check_view(c, view));
    if (!rgb) return fail(GS_ERR_INVALID_ARG, "rgb is null");
    CKI(ensure(c->target_f32, (size_t)c->total_pixels * 12, c));
    const ViewDesc& d = c->vdesc[view];
    CK(cudaMemcpyAsync(c->target_f32.as<float>() + (size_t)d.pixel_offset * 3, rgb, (size_t)d.width * d.height * 12,
                       cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->target_kind[view] = 2;
    return GS_OK;
}

// ---- forward / backward ---------------------------------------------------------------
static int check_range(GsContext* c, int first, int count, bool allow_scratch) {
    const int limit = allow_scratch ? (int)c->cams.size() : c->V;
    if (count < 1 || first < 0 || first + count > limit)
        return fail(GS_ERR_INVALID_ARG, "views [%d, %d) out of range [0, %d)", first, first + count, limit);
    if (c->n <= 0) return fail(GS_ERR_STATE, "no Gaussians set");
    return GS_OK;
}

static int run_forward(GsContext* c, int first, int count) {
    CKI(size_pairs(c, count));
    CKI(ensure_capacity(c, first, count));
    for (int tries = 0; tries < 3; tries++) {
        CKI(enqueue_forward(c, first, count, c->cfg.batched != 0));
        CKI(read_status(c));
        if (!c->status_host->overflow) break;
        CKI(grow_instances(c, c->status_host->instances_needed));
    }
    if (c->status_host->overflow) return fail(GS_ERR_CAPACITY, "key instances overflowed");
    c->last_first = first;
    c->last_count = count;
    c->last_batched = c->cfg.batched != 0;
    c->have_loss = false;
    return GS_OK;
}

int gs_forward(GsContext* c, int32_t first, int32_t count, float* images_out) {
    GS_TRACE("gs_forward");
    CTX_CHECK(c);
    CKI(check_range(c, first, count, false));
    CKI(run_forward(c, first, count));
    if (images_out) {
        const ViewDesc& a = c->vdesc[first];
        const ViewDesc& b = c->vdesc[first + count - 1];
        const size_t px = (size_t)(b.pixel_offset + (int64_t)b.width * b.height - a.pixel_offset);
        CK(cudaMemcpyAsync(images_out, c->image.as<float>() + (size_t)a.pixel_offset * 3, px * 12,
                           cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return GS_OK;
}

static int targets_kind(GsContext* c, int first, int count, int* kind) {
    int k = c->target_kind[first];
    for (int v = first; v < first + count; v++)
        if (c->target_kind[v] != k) return fail(GS_ERR_STATE, "views of one step must all have u8 or all f32 targets");
    if (k == 0) return fail(GS_ERR_STATE, "view %d has no target", first);
    *kind = k;
    return GS_OK;
}

static int check_loss(const GsLossConfig* lc) {
    if (!lc) return fail(GS_ERR_INVALID_ARG, "loss config is null");
    if (!(lc->ssim_lambda >= 0.f && lc->ssim_lambda <= 1.f)) return fail(GS_ERR_INVALID_ARG, "ssim_lambda must be in [0, 1]");
    if (lc->window != 0 && lc->window != 1) return fail(GS_ERR_INVALID_ARG, "window must be 0 or 1");
    return GS_OK;
}

int gs_loss(GsContext* c, const GsLossConfig* lc, float* loss_out) {
    GS_TRACE("gs_loss");
    CTX_CHECK(c);
    CKI(check_loss(lc));
    if (c->last_first < 0) return fail(GS_ERR_STATE, "gs_loss needs a forward first");
    int kind;
    CKI(targets_kind(c, c->last_first, c->last_count, &kind));
    CK(cudaMemsetAsync(c->acc.p, 0, sizeof(double) * 2 * (GS_MAX_VIEWS + 1), c->stream));
    if (c->last_batched) {
        CKI(enqueue_loss_view(c, c->last_first, c->last_count, *lc, kind));
    } else {
        for (int v = c->last_first; v < c->last_first + c->last_count; v++) CKI(enqueue_loss_view(c, v, 1, *lc, kind));
    }
    launch_loss_from_acc(c->status.as<DevStatus>(), c->acc.as<double>(), c->views_d.as<ViewDesc>(), c->last_first,
                         c->last_count, lc->ssim_lambda, lc->window, c->stream);
    CK(cudaGetLastError());
    c->have_loss = true;
    if (loss_out) {
        CKI(read_status(c));
        *loss_out = c->status_host->loss;
    }
    return GS_OK;
}

int gs_backward(GsContext* c, const float* dl_dimages) {
    GS_TRACE("gs_backward");
    CTX_CHECK(c);
    if (c->last_first < 0) return fail(GS_ERR_STATE, "gs_backward needs a forward first");
    const int first = c->last_first, count = c->last_count;
    if (dl_dimages) {
        const ViewDesc& a = c->vdesc[first];
        const ViewDesc& b = c->vdesc[first + count - 1];
        const size_t px = (size_t)(b.pixel_offset + (int64_t)b.width * b.height - a.pixel_offset);
        CK(cudaMemcpyAsync(c->dl.as<float>() + (size_t)a.pixel_offset * 3, dl_dimages, px * 12, cudaMemcpyHostToDevice,
                           c->stream));
    } else if (!c->have_loss) {
        return fail(GS_ERR_STATE, "gs_backward without dL/dpixel needs gs_loss first");
    }
    if (c->last_batched) {
        CKI(enqueue_backward_view(c, first, first, count, true, false));
    } else {
        for (int v = first; v < first + count; v++) CKI(enqueue_backward_view(c, v, first, 1, false, v > first));
    }
    CK(cudaStreamSynchronize(c->stream));
    return GS_OK;
}

int gs_get_param_grads(GsContext* c, float* out) {
    CTX_CHECK(c);
    if (!out) return fail(GS_ERR_INVALID_ARG, "out is null");
    std::vector<float> h;
    CKI(download_planes(c, c->grads, h));
    const int P = c->planes;
    for (int i = 0; i < c->n; i++)
        for (int k = 0; k < P; k++) out[(size_t)i * P + k] = h[(size_t)k * c->n_pad + i];
    return GS_OK;
}

static int slot_of(GsContext* c, int view, int* slot) {
    if (c->last_first < 0) return fail(GS_ERR_STATE, "no forward yet");
    if (view < c->last_first || view >= c->last_first + c->last_count)
        return fail(GS_ERR_INVALID_ARG, "view %d was not in the last forward", view);
    *slot = view - c->last_first;
    return GS_OK;
}

int gs_get_screen_grads(GsContext* c, int32_t view, float* out16) {
    CTX_CHECK(c);
    if (!out16) return fail(GS_ERR_INVALID_ARG, "out is null");
    int slot;
    CKI(slot_of(c, view, &slot));
    CKI(ensure(c->scratch16, (size_t)c->n_pad * 64, c));
    launch_screen_grads16(c->sg8.as<float4>() + (size_t)slot * c->n_pad * 2, c->sg1.as<float>() + (size_t)slot * c->n_pad,
                          c->n, c->scratch16.as<float>(), c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out16, c->scratch16.p, (size_t)c->n * 64, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return GS_OK;
}

int gs_get_splats(GsContext* c, int32_t view, float* out12) {
    CTX_CHECK(c);
    if (!out12) return fail(GS_ERR_INVALID_ARG, "out is null");
    int slot;
    CKI(slot_of(c, view, &slot));
    CKI(ensure(c->scratch16, (size_t)c->n_pad * 64, c));
    const size_t off = (size_t)slot * c->n_pad;
    launch_splats12(c->geo0.as<float4>() + off, c->geo1.as<float4>() + off, c->rgb.as<float4>() + off,
                    c->pkeys.as<uint32_t>() + off, c->n, c->scratch16.as<float>(), c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out12, c->scratch16.p, (size_t)c->n * 48, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return GS_OK;
}

int gs_get_tile_lists(GsContext* c, int32_t view, uint32_t* list_out, uint32_t* ranges_out, uint64_t* keys_out,
                      int64_t list_cap, int64_t* count_out) {
    CTX_CHECK(c);
    int slot;
    CKI(slot_of(c, view, &slot));
    if (!ranges_out || !count_out) return fail(GS_ERR_INVALID_ARG, "ranges_out/count_out is null");
    const ViewDesc& d = c->vdesc[view];
    const int tiles = d.tiles_x * d.tiles_y;
    std::vector<uint2> rg(tiles);
    CK(cudaMemcpyAsync(rg.data(), c->ranges.as<uint2>() + d.tile_offset, (size_t)tiles * 8, cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    uint32_t lo = 0xffffffffu, hi = 0;
    for (int t = 0; t < tiles; t++)
        if (rg[t].y > rg[t].x) {
            lo = std::min(lo, rg[t].x);
            hi = std::max(hi, rg[t].y);
        }
    int64_t total = 0;
    for (int t = 0; t < tiles; t++) total += rg[t].y - rg[t].x;
    *count_out = total;
    if (total > list_cap) return fail(GS_ERR_CAPACITY, "list_cap %lld < %lld entries", (long long)list_cap, (long long)total);
    std::vector<uint32_t> pairs;
    std::vector<float4> g1;
    if (total > 0) {
        pairs.resize(hi - lo);
        CK(cudaMemcpyAsync(pairs.data(), c->ivals.as<uint32_t>() + lo, (size_t)(hi - lo) * 4, cudaMemcpyDeviceToHost,
                           c->stream));
        if (keys_out) {
            g1.resize(c->n_pad);
            CK(cudaMemcpyAsync(g1.data(), c->geo1.as<float4>() + (size_t)slot * c->n_pad, (size_t)c->n_pad * 16,
                               cudaMemcpyDeviceToHost, c->stream));
        }
        CK(cudaStreamSynchronize(c->stream));
    }
    int64_t pos = 0;
    for (int t = 0; t < tiles; t++) {
        ranges_out[2 * t] = (uint32_t)pos;
        for (uint32_t k = rg[t].x; k < rg[t].y; k++) {
            const uint32_t pair = pairs[k - lo];
            const uint32_t gi = pair - (uint32_t)slot * (uint32_t)c->n_pad;
            if (list_out) list_out[pos] = gi;
            if (keys_out) {
                uint32_t bits;
                memcpy(&bits, &g1[gi].w, 4);
                keys_out[pos] = ((uint64_t)t << 32) | bits;
            }
            pos++;
        }
        ranges_out[2 * t + 1] = (uint32_t)pos;
    }
    return GS_OK;
}

// ---- one-camera helpers (render, gradients, loss gradient) ------------------------------
int gs_render(GsContext* c, const GsCamera* cam, float* rgb_out, float* state_out) {
    GS_TRACE("gs_render");
    CTX_CHECK(c);
    if (!cam || !rgb_out) return fail(GS_ERR_INVALID_ARG, "null argument");
    if (c->n <= 0) return fail(GS_ERR_STATE, "no Gaussians set");
    CKI(set_scratch_camera(c, *cam));
    const int v = c->V;
    CKI(run_forward(c, v, 1));
    const ViewDesc& d = c->vdesc[v];
    const size_t px = (size_t)d.width * d.height;
    CK(cudaMemcpyAsync(rgb_out, c->image.as<float>() + (size_t)d.pixel_offset * 3, px * 12, cudaMemcpyDeviceToHost,
                       c->stream));
    if (state_out) {
        std::vector<float> T(px);
        std::vector<uint32_t> L(px);
        std::vector<uint2> rg((size_t)d.tiles_x * d.tiles_y);
        CK(cudaMemcpyAsync(T.data(), c->t_final.as<float>() + d.pixel_offset, px * 4, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(L.data(), c->last.as<uint32_t>() + d.pixel_offset, px * 4, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(rg.data(), c->ranges.as<uint2>() + d.tile_offset, rg.size() * 8, cudaMemcpyDeviceToHost,
                           c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (int y = 0; y < d.height; y++)
            for (int x = 0; x < d.width; x++) {
                const size_t p = (size_t)y * d.width + x;
                const uint2 r = rg[(size_t)(y / d.tile) * d.tiles_x + x / d.tile];
                state_out[p * 2] = T[p];
                state_out[p * 2 + 1] = (float)(L[p] - r.x);
            }
    }
    CK(cudaStreamSynchronize(c->stream));
    return GS_OK;
}

int gs_gradients(GsContext* c, const GsCamera* cam, const float* target, float ssim_lambda, float* image_out,
                 float* grads16_out, float* shape10_out) {
    GS_TRACE("gs_gradients");
    CTX_CHECK(c);
    if (!cam || !target) return fail(GS_ERR_INVALID_ARG, "null argument");
    if (c->n <= 0) return fail(GS_ERR_STATE, "no Gaussians set");
    CKI(set_scratch_camera(c, *cam));
    const int v = c->V;
    const ViewDesc& d = c->vdesc[v];
    const size_t px = (size_t)d.width * d.height;
    CKI(ensure(c->target_f32, (size_t)c->total_pixels * 12, c));
    CK(cudaMemcpyAsync(c->target_f32.as<float>() + (size_t)d.pixel_offset * 3, target, px * 12, cudaMemcpyHostToDevice,
                       c->stream));
    c->target_kind[v] = 2;
    CKI(run_forward(c, v, 1));
    GsLossConfig lc{ssim_lambda, 0};
    CKI(gs_loss(c, &lc, nullptr));
    CKI(gs_backward(c, nullptr));
    if (image_out)
        CK(cudaMemcpyAsync(image_out, c->image.as<float>() + (size_t)d.pixel_offset * 3, px * 12, cudaMemcpyDeviceToHost,
                           c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (grads16_out) CKI(gs_get_screen_grads(c, v, grads16_out));
    if (shape10_out) {
        std::vector<float> h;
        CKI(download_planes(c, c->grads, h));
        for (int i = 0; i < c->n; i++)
            for (int k = 0; k < 10; k++) shape10_out[(size_t)i * 10 + k] = h[(size_t)k * c->n_pad + i];
    }
    return GS_OK;
}

int gs_loss_gradient(GsContext* c, const float* image, const float* target, int32_t width, int32_t height,
                     float ssim_lambda, int32_t window, float* grad_out, float* loss_out) {
    GS_TRACE("gs_loss_gradient");
    CTX_CHECK(c);
    if (!image || !target || !grad_out) return fail(GS_ERR_INVALID_ARG, "null argument");
    GsLossConfig lc{ssim_lambda, window};
    CKI(check_loss(&lc));
    GsCamera cam;
    memset(&cam, 0, sizeof cam);
    cam.view[0] = cam.view[5] = cam.view[10] = 1.f;
    cam.fx = cam.fy = 1.f;
    cam.width = width;
    cam.height = height;
    CKI(set_scratch_camera(c, cam));
    const int v = c->V;
    const ViewDesc& d = c->vdesc[v];
    const size_t px = (size_t)width * height;
    CKI(ensure(c->target_f32, (size_t)c->total_pixels * 12, c));
    CK(cudaMemcpyAsync(c->image.as<float>() + (size_t)d.pixel_offset * 3, image, px * 12, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->target_f32.as<float>() + (size_t)d.pixel_offset * 3, target, px * 12, cudaMemcpyHostToDevice,
                       c->stream));
    CK(cudaMemsetAsync(c->acc.p, 0, sizeof(double) * 2 * (GS_MAX_VIEWS + 1), c->stream));
    CKI(enqueue_loss_view(c, v, 1, lc, 2));
    launch_loss_from_acc(c->status.as<DevStatus>(), c->acc.as<double>(), c->views_d.as<ViewDesc>(), v, 1, ssim_lambda,
                         window, c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(grad_out, c->dl.as<float>() + (size_t)d.pixel_offset * 3, px * 12, cudaMemcpyDeviceToHost, c->stream));
    CKI(read_status(c));
    if (loss_out) *loss_out = c->status_host->loss;
    return GS_OK;
}

// ---- training ---------------------------------------------------------------------------
static int check_adam(const GsAdamConfig* a) {
    if (!a) return fail(GS_ERR_INVALID_ARG, "adam config is null");
    if (!(a->beta1 >= 0.f && a->beta1 < 1.f && a->beta2 >= 0.f && a->beta2 < 1.f && a->eps > 0.f))
        return fail(GS_ERR_INVALID_ARG, "bad Adam betas/eps");
    return GS_OK;
}

// Picks up the status of the previous asynchronous step, if it has finished.
static int poll_status(GsContext* c, bool wait) {
    if (!c->status_pending) return GS_OK;
    if (wait) CK(cudaEventSynchronize(c->status_event));
    else if (cudaEventQuery(c->status_event) != cudaSuccess) {
        cudaGetLastError();
        return GS_OK;
    }
    c->status_pending = false;
    if (c->status_host->sort_timeout) return sort_timed_out(c);
    if (c->status_host->overflow) {
        c->skipped_steps++;
        CKI(grow_instances(c, c->status_host->instances_needed));
    }
    return GS_OK;
}

// The whole step on the context's stream: its graph (captured on first use) or the direct
// launches.
static int launch_step(GsContext* c, const GsAdamConfig& ad, const GsLossConfig& lc, int first, int count,
                       bool batched, int kind) {
    if (c->cfg.use_graph) {
        GraphKey key;
        memset(&key, 0, sizeof key);
        key.first = first;
        key.count = count;
        key.batched = batched;
        key.window = lc.window;
        key.kind = kind;
        memcpy(&key.loss_lambda_bits, &lc.ssim_lambda, 4);
        key.adam = ad;
        StepGraph& g = c->graphs[key];
        if (!g.exec || g.generation != c->generation) CKI(capture_step(c, g, ad, lc, first, count, batched, kind));
        CKI(launch_graph(c, g));
    } else {
        CKI(begin_record(c));
        CKI(enqueue_step(c, ad, lc, first, count, batched, kind));
        CKI(end_record(c));
    }
    return GS_OK;
}

static int train_step_impl(GsContext* c, const GsAdamConfig* ad, const GsLossConfig* lc, int first, int count,
                           const uint8_t* host_targets, float* loss_out) {
    CTX_CHECK(c);
    CKI(check_adam(ad));
    CKI(check_loss(lc));
    CKI(check_range(c, first, count, false));
    if (host_targets) {
        CKI(ensure(c->target_u8, (size_t)c->total_pixels * 3, c));
        for (int v = first; v < first + count; v++) c->target_kind[v] = 1;
    }
    int kind;
    CKI(targets_kind(c, first, count, &kind));
    if (c->cfg.autotune && !c->tuned && first == 0 && count == c->V) {
        c->tuned = true;  // timing only: the photos need not be on the device yet
        CKI(poll_status(c, true));
        CKI(gs_autotune(c, nullptr));
    }
    CKI(size_pairs(c, count));
    CKI(poll_status(c, false));
    CKI(ensure_capacity(c, first, count));
    const bool batched = c->cfg.batched != 0;
    for (int attempt = 0; attempt < 3; attempt++) {
        if (host_targets) {
            const ViewDesc& a = c->vdesc[first];
            const ViewDesc& b = c->vdesc[first + count - 1];
            const size_t px = (size_t)(b.pixel_offset + (int64_t)b.width * b.height - a.pixel_offset);
            CK(cudaMemcpyAsync(c->target_u8.as<uint8_t>() + (size_t)a.pixel_offset * 3, host_targets, px * 3,
                               cudaMemcpyHostToDevice, c->stream));
        }
        CKI(launch_step(c, *ad, *lc, first, count, batched, kind));
        CK(cudaMemcpyAsync(c->status_host, c->status.p, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaEventRecord(c->status_event, c->stream));
        c->status_pending = true;
        c->last_first = first;
        c->last_count = count;
        c->last_batched = batched;
        c->have_loss = true;
        if (!loss_out) return GS_OK;
        CKI(poll_status(c, true));
        if (!c->status_host->overflow) {
            *loss_out = c->status_host->loss;
            return GS_OK;
        }
        // The step skipped its update (instances overflowed); the buffer has grown: redo it.
    }
    return fail(GS_ERR_CAPACITY, "key instances kept overflowing");
}

int gs_train_step(GsContext* c, const GsAdamConfig* adam, const GsLossConfig* loss, int32_t first, int32_t count,
                  float* loss_out) {
    GS_TRACE("gs_train_step");
    return train_step_impl(c, adam, loss, first, count, nullptr, loss_out);
}

int gs_train_step_host(GsContext* c, const GsAdamConfig* adam, const GsLossConfig* loss, int32_t first, int32_t count,
                       const uint8_t* targets_u8, float* loss_out) {
    GS_TRACE("gs_train_step_host");
    if (!targets_u8) return fail(GS_ERR_INVALID_ARG, "targets_u8 is null");
    return train_step_impl(c, adam, loss, first, count, targets_u8, loss_out);
}

int gs_step_gradients(GsContext* c, const GsLossConfig* lc, int32_t first, int32_t count, float** grads_device,
                      int64_t* num_floats) {
    GS_TRACE("gs_step_gradients");
    CTX_CHECK(c);
    CKI(check_loss(lc));
    CKI(check_range(c, first, count, false));
    if (!grads_device || !num_floats) return fail(GS_ERR_INVALID_ARG, "null output pointer");
    int kind;
    CKI(targets_kind(c, first, count, &kind));
    CKI(size_pairs(c, count));
    CKI(poll_status(c, false));
    CKI(ensure_capacity(c, first, count));
    const bool batched = c->cfg.batched != 0;
    const GsAdamConfig ad = {};
    if (c->cfg.use_graph) {
        GraphKey key;
        memset(&key, 0, sizeof key);
        key.first = first;
        key.count = count;
        key.batched = batched;
        key.window = lc->window;
        key.kind = kind;
        key.phase = 1;
        memcpy(&key.loss_lambda_bits, &lc->ssim_lambda, 4);
        StepGraph& g = c->graphs[key];
        if (!g.exec || g.generation != c->generation) CKI(capture_step(c, g, ad, *lc, first, count, batched, kind, 1));
        CKI(launch_graph(c, g));
    } else {
        CKI(begin_record(c));
        CKI(enqueue_step(c, ad, *lc, first, count, batched, kind, 1));
        CKI(end_record(c));
    }
    c->last_first = first;
    c->last_count = count;
    c->last_batched = batched;
    c->have_loss = true;
    c->grads_pending = true;
    *grads_device = c->grads.as<float>();
    *num_floats = (int64_t)grad_buffer_floats(c);
    return GS_OK;
}

int gs_step_apply(GsContext* c, const GsAdamConfig* ad, float* loss_out, int32_t* skipped_out) {
    GS_TRACE("gs_step_apply");
    CTX_CHECK(c);
    CKI(check_adam(ad));
    if (!c->grads_pending) return fail(GS_ERR_STATE, "gs_step_apply without gs_step_gradients");
    c->grads_pending = false;
    AdamArgs aa;
    fill_adam_args(c, *ad, aa);
    aa.skip = grad_tail(c) + 1;
    launch_adam(aa, c->stream);
    if (c->stats_on)
        launch_stats_commit(c->stats.as<float>(), step_stats(c), c->n_pad, c->status.as<DevStatus>(),
                            grad_tail(c) + 1, c->stream);
    launch_reduced_step_end(c->status.as<DevStatus>(), grad_tail(c), c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->status_host, c->status.p, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaEventRecord(c->status_event, c->stream));
    c->status_pending = true;
    if (!loss_out && !skipped_out) return GS_OK;
    const DevStatus* h = c->status_host;
    CK(cudaEventSynchronize(c->status_event));
    const float loss = h->loss;
    const int skipped = h->skipped;
    CKI(poll_status(c, true));
    if (loss_out) *loss_out = loss;
    if (skipped_out) *skipped_out = skipped;
    return GS_OK;
}

int gs_get_stream(GsContext* c, void** stream_out) {
    CTX_CHECK(c);
    if (!stream_out) return fail(GS_ERR_INVALID_ARG, "stream_out is null");
    *stream_out = (void*)c->stream;
    return GS_OK;
}

int gs_dp_unique_id(void* id_out, int32_t bytes) {
    GS_TRACE("gs_dp_unique_id");
    if (!id_out || bytes < dp_unique_id_bytes())
        return fail(GS_ERR_INVALID_ARG, "id buffer needs %d bytes", dp_unique_id_bytes());
    char err[256];
    if (!dp_unique_id(id_out, err, sizeof err)) return fail(GS_ERR_COMM, "%s", err);
    return GS_OK;
}

int gs_dp_init(GsContext* c, const void* id, int32_t bytes, int32_t rank, int32_t world) {
    GS_TRACE("gs_dp_init");
    CTX_CHECK(c);
    if (!id || bytes < dp_unique_id_bytes())
        return fail(GS_ERR_INVALID_ARG, "id needs %d bytes", dp_unique_id_bytes());
    if (world < 1 || rank < 0 || rank >= world) return fail(GS_ERR_INVALID_ARG, "rank %d of %d", rank, world);
    if (c->dp_comm) return fail(GS_ERR_STATE, "data parallel already initialised");
    char err[256];
    void* comm = dp_comm_create(id, rank, world, err, sizeof err);
    if (!comm) return fail(GS_ERR_COMM, "%s", err);
    c->dp_comm = comm;
    c->dp_rank = rank;
    c->dp_world = world;
    return GS_OK;
}

int gs_dp_allreduce(GsContext* c) {
    GS_TRACE("gs_dp_allreduce");
    CTX_CHECK(c);
    if (!c->dp_comm) return fail(GS_ERR_STATE, "gs_dp_init first");
    if (!c->grads_pending) return fail(GS_ERR_STATE, "gs_step_gradients first");
    char err[256];
    if (!dp_allreduce_sum(c->dp_comm, c->grads.as<float>(), grad_buffer_floats(c), c->stream, err, sizeof err))
        return fail(GS_ERR_COMM, "%s", err);
    CK(cudaGetLastError());
    return GS_OK;
}

int gs_dp_finalize(GsContext* c) {
    GS_TRACE("gs_dp_finalize");
    CTX_CHECK(c);
    if (c->dp_comm) {
        CK(cudaStreamSynchronize(c->stream));
        dp_comm_destroy(c->dp_comm);
        c->dp_comm = nullptr;
    }
    c->dp_rank = 0;
    c->dp_world = 1;
    return GS_OK;
}

int gs_train_step_host_async(GsContext* c, const GsAdamConfig* ad, const GsLossConfig* lc, int32_t first,
                             int32_t count, const uint8_t* targets_u8, float* loss_out) {
    GS_TRACE("gs_train_step_host_async");
    CTX_CHECK(c);
    CKI(check_adam(ad));
    CKI(check_loss(lc));
    CKI(check_range(c, first, count, false));
    if (!targets_u8 || !loss_out) return fail(GS_ERR_INVALID_ARG, "null targets or loss buffer");
    if (!c->copy_stream) {
        CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        for (int k = 0; k < 2; k++) {
            CK(cudaEventCreateWithFlags(&c->ev_copied[k], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&c->ev_free[k], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&c->ev_done[k], cudaEventDisableTiming));
        }
    }
    const int slot = c->pipe_slot;
    // At most two steps in flight: the one queued two calls ago must be done before its
    // staging buffer and loss slot are reused (its loss is then in the caller's buffer).
    if (c->pipe_pending[slot]) {
        CK(cudaEventSynchronize(c->ev_done[slot]));
        c->pipe_pending[slot] = false;
    }
    CKI(ensure(c->target_u8, (size_t)c->total_pixels * 3, c));
    for (int v = first; v < first + count; v++) c->target_kind[v] = 1;
    int kind;
    CKI(targets_kind(c, first, count, &kind));
    CKI(size_pairs(c, count));
    CKI(poll_status(c, false));
    CKI(ensure_capacity(c, first, count));
    const ViewDesc& va = c->vdesc[first];
    const ViewDesc& vb = c->vdesc[first + count - 1];
    const size_t bytes = (size_t)(vb.pixel_offset + (int64_t)vb.width * vb.height - va.pixel_offset) * 3;
    if (c->stage[slot].bytes < bytes) {
        CK(cudaStreamSynchronize(c->copy_stream));  // the other slot's copy may still read nothing of this one
        CKI(ensure(c->stage[slot], bytes, c));
    }
    // Photos: host -> staging buffer on the copy stream (overlapping the step before),
    // then staging -> target buffer on the compute stream, right before the step.
    CK(cudaStreamWaitEvent(c->copy_stream, c->ev_free[slot], 0));
    CK(cudaMemcpyAsync(c->stage[slot].p, targets_u8, bytes, cudaMemcpyHostToDevice, c->copy_stream));
    CK(cudaEventRecord(c->ev_copied[slot], c->copy_stream));
    CK(cudaStreamWaitEvent(c->stream, c->ev_copied[slot], 0));
    CK(cudaMemcpyAsync(c->target_u8.as<uint8_t>() + (size_t)va.pixel_offset * 3, c->stage[slot].p, bytes,
                       cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaEventRecord(c->ev_free[slot], c->stream));
    CKI(launch_step(c, *ad, *lc, first, count, c->cfg.batched != 0, kind));
    CK(cudaMemcpyAsync(loss_out, &c->status.as<DevStatus>()->loss, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(c->status_host, c->status.p, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaEventRecord(c->status_event, c->stream));
    CK(cudaEventRecord(c->ev_done[slot], c->stream));
    c->status_pending = true;
    c->pipe_pending[slot] = true;
    c->pipe_slot = slot ^ 1;
    c->last_first = first;
    c->last_count = count;
    c->last_batched = c->cfg.batched != 0;
    c->have_loss = true;
    return GS_OK;
}

int gs_train(GsContext* c, int32_t steps, const GsAdamConfig* adam, float* losses_out) {
    GS_TRACE("gs_train");
    CTX_CHECK(c);
    if (steps < 0) return fail(GS_ERR_INVALID_ARG, "steps < 0");
    if (c->V < 1) return fail(GS_ERR_STATE, "no views");
    const GsLossConfig lc{0.f, 0};
    const int saved = c->cfg.batched;
    c->cfg.batched = 0;
    int rc = GS_OK;
    for (int t = 1; t <= steps && rc == GS_OK; t++) {
        float loss = 0.f;
        rc = train_step_impl(c, adam, &lc, (t - 1) % c->V, 1, nullptr, &loss);
        if (rc == GS_OK && losses_out) losses_out[t - 1] = loss;
    }
    c->cfg.batched = saved;
    return rc;
}

int gs_get_step(GsContext* c, int32_t* t_out) {
    CTX_CHECK(c);
    if (!t_out) return fail(GS_ERR_INVALID_ARG, "t_out is null");
    CKI(read_status(c));
    *t_out = c->status_host->step_t;
    return GS_OK;
}

int gs_debug_lookback_wait(GsContext* c, int32_t polls) {
    CTX_CHECK(c);
    if (polls < 0) return fail(GS_ERR_INVALID_ARG, "polls must be >= 0");
    c->debug_wait_host = (unsigned int)polls;
    CK(cudaMemcpyAsync(&c->status.as<DevStatus>()->debug_wait, &c->debug_wait_host, sizeof(unsigned int),
                       cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return GS_OK;
}

// ---- memory, timing, diagnostics --------------------------------------------------------
int gs_host_alloc(size_t bytes, void** out) {
    if (!out) return fail(GS_ERR_INVALID_ARG, "out is null");
    CK(cudaMallocHost(out, bytes ? bytes : 1));
    return GS_OK;
}

int gs_host_free(void* p) {
    if (p) CK(cudaFreeHost(p));
    return GS_OK;
}

int gs_synchronize(GsContext* c) {
    CTX_CHECK(c);
    CK(cudaStreamSynchronize(c->stream));
    CKI(poll_status(c, true));
    return GS_OK;
}

int gs_event_record(GsContext* c, int32_t slot) {
    CTX_CHECK(c);
    if (slot < 0 || slot >= 64) return fail(GS_ERR_INVALID_ARG, "slot out of range");
    CK(cudaEventRecord(c->user_events[slot], c->stream));
    return GS_OK;
}

int gs_event_elapsed(GsContext* c, int32_t a, int32_t b, float* ms) {
    CTX_CHECK(c);
    if (a < 0 || a >= 64 || b < 0 || b >= 64 || !ms) return fail(GS_ERR_INVALID_ARG, "bad slot or pointer");
    CK(cudaEventSynchronize(c->user_events[b]));
    CK(cudaEventElapsedTime(ms, c->user_events[a], c->user_events[b]));
    return GS_OK;
}

int gs_stage_times(GsContext* c, double* ms_out, int64_t* launches_out, int32_t* steps_out) {
    CTX_CHECK(c);
    for (auto& sl : c->slots) CKI(harvest(c, sl));
    for (int s = 0; s < GS_NUM_STAGES; s++) {
        if (ms_out) ms_out[s] = c->stage_ms[s];
        if (launches_out) launches_out[s] = c->stage_launches[s];
    }
    if (steps_out) *steps_out = c->timed_steps;
    return GS_OK;
}

int gs_stage_times_reset(GsContext* c) {
    CTX_CHECK(c);
    for (auto& sl : c->slots) CKI(harvest(c, sl));
    for (int s = 0; s < GS_NUM_STAGES; s++) {
        c->stage_ms[s] = 0.0;
        c->stage_launches[s] = 0;
    }
    c->timed_steps = 0;
    return GS_OK;
}

int gs_set_stage_timing(GsContext* c, int32_t enabled) {
    CTX_CHECK(c);
    for (auto& sl : c->slots) CKI(harvest(c, sl));
    if ((enabled != 0) != c->stage_timing) {
        c->stage_timing = enabled != 0;
        drop_graphs(c);
    }
    return GS_OK;
}

int gs_get_stats(GsContext* c, GsStats* out) {
    CTX_CHECK(c);
    if (!out) return fail(GS_ERR_INVALID_ARG, "out is null");
    CK(cudaStreamSynchronize(c->stream));
    CKI(poll_status(c, true));
    CKI(read_status(c));
    memset(out, 0, sizeof *out);
    out->instances = (int64_t)c->status_host->instances_needed;
    out->instance_capacity = c->inst_cap;
    unsigned vis[GS_MAX_VIEWS + 1];
    CK(cudaMemcpy(vis, c->visible.p, sizeof vis, cudaMemcpyDeviceToHost));
    int64_t v = 0;
    if (c->last_batched) v = vis[0];
    else
        for (int s = 0; s < c->last_count && s < GS_MAX_VIEWS; s++) v += vis[1 + s];
    out->visible_pairs = v;
    if (c->last_first >= 0) {
        const ViewDesc& a = c->vdesc[c->last_first];
        const ViewDesc& b = c->vdesc[c->last_first + c->last_count - 1];
        out->tiles = b.tile_offset + (int64_t)b.tiles_x * b.tiles_y - a.tile_offset;
        out->pixels = b.pixel_offset + (int64_t)b.width * b.height - a.pixel_offset;
    }
    out->kernel_launches_per_step = c->last_step_launches;
    out->raster_batch = c->batch_bwd;
    out->raster_threads = c->wt_bwd * c->wt_bwd / c->ppt_bwd;
    auto wt_code = [](int wt) { return (uint32_t)(wt == 8 ? 3 : (wt == 16 ? 4 : 5)) << 9; };  // log2
    out->raster_variant = (int32_t)(((uint32_t)c->batch_fwd | wt_code(c->wt_fwd) | ((uint32_t)c->ppt_fwd << 12)) |
                                    (((uint32_t)c->batch_bwd | wt_code(c->wt_bwd)) << 16) |
                                    ((uint32_t)c->ppt_bwd << 28));
    out->tile_size = c->tile;
    out->overflow = (int32_t)c->skipped_steps;
    return GS_OK;
}

int gs_get_blend_count(GsContext* c, uint64_t* blends_out) {
    CTX_CHECK(c);
    if (!blends_out) return fail(GS_ERR_INVALID_ARG, "blends_out is null");
    if (c->last_first < 0 || c->last_count < 1) return fail(GS_ERR_STATE, "no forward yet");
    int maxpx = 0;
    for (int v = c->last_first; v < c->last_first + c->last_count; v++)
        maxpx = std::max(maxpx, c->vdesc[v].width * c->vdesc[v].height);
    CKI(ensure(c->scratch16, 64, c));
    CK(cudaMemsetAsync(c->scratch16.p, 0, 8, c->stream));
    launch_blend_count(c->views_d.as<ViewDesc>(), c->last_first, c->last_count, maxpx, c->ranges.as<uint2>(),
                       c->last.as<uint32_t>(), c->scratch16.as<unsigned long long>(), c->stream);
    CK(cudaGetLastError());
    unsigned long long n = 0;
    CK(cudaMemcpyAsync(&n, c->scratch16.p, 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *blends_out = (uint64_t)n;
    return GS_OK;
}

// ---- initialisation from points ---------------------------------------------------------
// Device copies of xyz (and rgb), the neighbour table and the sizes in nb_scratch;
// returns the device sizes.
static int neighbour_sizes_device(GsContext* c, const float* xyz, int count, double mn, double mx, double fb,
                                  const float* rgb, float** d_xyz_out, float** d_rgb_out, float** d_sizes_out) {
    unsigned T = 1024;
    while (T < 2u * (unsigned)count) T <<= 1;
    const size_t n = (size_t)count;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) & ~(size_t)255;
        return o;
    };
    const size_t o_keys = take((size_t)T * 8), o_ids = take((size_t)T * 4), o_cnt = take(64);
    const size_t o_slot = take(n * 4), o_cc = take(n * 4), o_cs = take(n * 4), o_cur = take(n * 4),
                 o_pts = take(n * 4), o_xyz = take(n * 12), o_rgb = take(n * 12), o_sz = take(n * 4);
    CKI(ensure(c->nb_scratch, off, c));
    char* base = c->nb_scratch.as<char>();
    NeighbourArgs a;
    memset(&a, 0, sizeof a);
    a.xyz = reinterpret_cast<float*>(base + o_xyz);
    a.count = count;
    a.keys = reinterpret_cast<unsigned long long*>(base + o_keys);
    a.ids = reinterpret_cast<unsigned*>(base + o_ids);
    a.mask = T - 1;
    a.counters = reinterpret_cast<unsigned*>(base + o_cnt);
    a.point_slot = reinterpret_cast<unsigned*>(base + o_slot);
    a.cell_count = reinterpret_cast<unsigned*>(base + o_cc);
    a.cell_start = reinterpret_cast<unsigned*>(base + o_cs);
    a.cell_cursor = reinterpret_cast<unsigned*>(base + o_cur);
    a.cell_points = reinterpret_cast<unsigned*>(base + o_pts);
    a.sizes = reinterpret_cast<float*>(base + o_sz);
    a.min_size = mn;
    a.max_size = mx;
    a.fallback = fb;
    CK(cudaMemcpyAsync(base + o_xyz, xyz, n * 12, cudaMemcpyHostToDevice, c->stream));
    if (rgb) CK(cudaMemcpyAsync(base + o_rgb, rgb, n * 12, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(a.keys, 0xff, (size_t)T * 8, c->stream));
    CK(cudaMemsetAsync(a.counters, 0, 64, c->stream));
    CK(cudaMemsetAsync(a.cell_count, 0, n * 4, c->stream));
    launch_neighbour_sizes(a, c->stream);
    CK(cudaGetLastError());
    *d_xyz_out = reinterpret_cast<float*>(base + o_xyz);
    if (d_rgb_out) *d_rgb_out = reinterpret_cast<float*>(base + o_rgb);
    *d_sizes_out = a.sizes;
    return GS_OK;
}

int gs_neighbour_sizes(GsContext* c, const float* xyz, int32_t count, double min_size, double max_size,
                       double fallback, float* sizes_out) {
    GS_TRACE("gs_neighbour_sizes");
    CTX_CHECK(c);
    if (count < 0 || count > (1 << 28) || (count > 0 && (!xyz || !sizes_out)))
        return fail(GS_ERR_INVALID_ARG, "bad point count or pointer");
    if (count == 0) return GS_OK;
    float *dx = nullptr, *ds = nullptr;
    CKI(neighbour_sizes_device(c, xyz, count, min_size, max_size, fallback, nullptr, &dx, nullptr, &ds));
    CK(cudaMemcpyAsync(sizes_out, ds, (size_t)count * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return GS_OK;
}

int gs_init_from_points(GsContext* c, const float* xyz, const float* rgb, int32_t count, float size) {
    GS_TRACE("gs_init_from_points");
    CTX_CHECK(c);
    if (count < 0 || count > (1 << 28) || (count > 0 && (!xyz || !rgb)))
        return fail(GS_ERR_INVALID_ARG, "bad point count or pointer");
    if (count == 0) {
        std::vector<float> none((size_t)c->planes * 128, 0.f);
        for (int i = 0; i < 128; i++) none[(size_t)6 * 128 + i] = 1.f;
        return upload_planes(c, 0, none);
    }
    float *dx = nullptr, *drgb = nullptr, *ds = nullptr;
    if (size > 0.f) {
        CKI(ensure(c->nb_scratch, (size_t)count * 24 + 256, c));
        dx = c->nb_scratch.as<float>();
        drgb = dx + (size_t)count * 3 + 64;
        CK(cudaMemcpyAsync(dx, xyz, (size_t)count * 12, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(drgb, rgb, (size_t)count * 12, cudaMemcpyHostToDevice, c->stream));
    } else {
        // neighbourSizes with the reference's defaults (min 0.005, max 0.1, fallback 0.06).
        CKI(neighbour_sizes_device(c, xyz, count, 0.005, 0.1, 0.06, rgb, &dx, &drgb, &ds));
    }
    // resize_scene allocates only the per-Gaussian buffers; the scratch stays valid.
    CKI(resize_scene(c, count, false));
    launch_init_planes(dx, drgb, size > 0.f ? nullptr : ds, size, count, c->n_pad, c->planes, c->params.as<float>(),
                       c->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    return GS_OK;
}

// ---- photo selection -------------------------------------------------------------------
int gs_sharpness(GsContext* c, const uint8_t* images, int32_t count, int32_t width, int32_t height,
                 int32_t channels, double* scores) {
    GS_TRACE("gs_sharpness");
    CTX_CHECK(c);
    if (count < 0 || width < 1 || height < 1 || (channels != 1 && channels != 3) || (count > 0 && (!images || !scores)))
        return fail(GS_ERR_INVALID_ARG, "bad images");
    if (count == 0) return GS_OK;
    const size_t px = (size_t)width * height * count;
    const size_t off_grey = ((px * channels + 255) & ~(size_t)255);
    const size_t off_sums = off_grey + ((px + 255) & ~(size_t)255);
    CKI(ensure(c->nb_scratch, off_sums + (size_t)count * 16, c));
    uint8_t* base = c->nb_scratch.as<uint8_t>();
    CK(cudaMemcpyAsync(base, images, px * channels, cudaMemcpyHostToDevice, c->stream));
    const uint8_t* grey = base;
    if (channels == 3) {
        launch_grey(base, px, base + off_grey, c->stream);
        grey = base + off_grey;
    }
    long long* sums = reinterpret_cast<long long*>(base + off_sums);
    CK(cudaMemsetAsync(sums, 0, (size_t)count * 16, c->stream));
    launch_laplacian_sums(grey, count, width, height, sums, c->stream);
    CK(cudaGetLastError());
    std::vector<long long> h((size_t)count * 2);
    CK(cudaMemcpyAsync(h.data(), sums, (size_t)count * 16, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const long long n = (long long)std::max(0, width - 2) * std::max(0, height - 2);
    for (int k = 0; k < count; k++) {
        if (!n) {
            scores[k] = 0.0;
            continue;
        }
        const double mean = (double)h[2 * k] / (double)n;
        scores[k] = (double)h[2 * k + 1] / (double)n - mean * mean;
    }
    return GS_OK;
}

int gs_choose_sharp(const double* scores, int32_t count, int32_t max_views, int32_t* chosen, int32_t* chosen_count) {
    if (count < 0 || max_views < 1 || (count > 0 && (!scores || !chosen)) || !chosen_count)
        return fail(GS_ERR_INVALID_ARG, "bad arguments");
    // chooseSharp (trainer/sharpness.js:39-55) in the reference's double arithmetic.
    const double step = std::max(1.0, (double)count / (double)max_views);
    std::vector<int> pick;
    for (double start = 0; start < count; start += step) {
        const int from = (int)std::floor(start);
        const int to = (int)std::min((double)count, std::floor(start + step));
        int best = from;
        for (int i = from + 1; i < to; i++)
            if (scores[i] > scores[best]) best = i;
        pick.push_back(best);
    }
    std::vector<double> sorted(scores, scores + count);
    std::stable_sort(sorted.begin(), sorted.end(), [](double a, double b) { return a - b < 0; });
    const double median = count ? sorted[(size_t)((count - 1) / 2)] : 0.0;
    std::vector<int> blurry;
    for (int i : pick)
        if (scores[i] < median * 0.35) blurry.push_back(i);
    std::stable_sort(blurry.begin(), blurry.end(), [&](int a, int b) { return scores[a] - scores[b] < 0; });
    const size_t ndrop = std::min(blurry.size(), (size_t)std::floor(pick.size() * 0.25));
    std::vector<char> drop((size_t)std::max(count, 1), 0);
    for (size_t k = 0; k < ndrop; k++) drop[(size_t)blurry[k]] = 1;
    int m = 0;
    for (int i : pick)
        if (!drop[(size_t)i]) chosen[m++] = i;
    *chosen_count = m;
    return GS_OK;
}

// ---- scene I/O ------------------------------------------------------------------------
int gs_load_ply(GsContext* c, const void* data, int64_t bytes, int32_t* count_out) {
    GS_TRACE("gs_load_ply");
    CTX_CHECK(c);
    if (!data || bytes <= 0) return fail(GS_ERR_INVALID_ARG, "no data");
    PlyHeaderInfo h;
    std::string err;
    if (ply_parse(data, bytes, c->planes, &h, &err) != 0) return fail(GS_ERR_INVALID_ARG, ".ply: %s", err.c_str());
    if (h.count > (1 << 28)) return fail(GS_ERR_INVALID_ARG, ".ply: too many vertices");
    const int n = (int)h.count;
    CKI(resize_scene(c, n, false));
    const size_t body = (size_t)h.count * h.nprops * 4;
    if (body > 0) {
        // The file's body as it is; the kernel transposes it into the parameter planes.
        CKI(ensure(c->dn_scratch, body, c));
        CK(cudaMemcpyAsync(c->dn_scratch.p, static_cast<const char*>(data) + h.header_bytes, body,
                           cudaMemcpyHostToDevice, c->stream));
    }
    launch_ply_to_planes(c->dn_scratch.as<float>(), h, c->n_pad, c->planes, c->params.as<float>(), c->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    if (count_out) *count_out = n;
    return GS_OK;
}

int gs_save_ply(GsContext* c, int32_t with_sh, void* out, int64_t capacity, int64_t* bytes_out) {
    GS_TRACE("gs_save_ply");
    CTX_CHECK(c);
    if (!bytes_out) return fail(GS_ERR_INVALID_ARG, "bytes_out is null");
    const int nk_out = with_sh ? (c->planes - 14) / 3 : 0;
    const std::string header = ply_header(c->n, nk_out);
    const int nprops = 17 + 3 * nk_out;
    const size_t body = (size_t)c->n * nprops * 4;
    const int64_t total = (int64_t)(header.size() + body);
    *bytes_out = total;
    if (!out) return GS_OK;
    if (capacity < total) return fail(GS_ERR_CAPACITY, "buffer holds %lld of %lld bytes", (long long)capacity,
                                      (long long)total);
    memcpy(out, header.data(), header.size());
    if (body > 0) {
        CKI(ensure(c->dn_scratch, body, c));
        launch_planes_to_ply(c->params.as<float>(), c->n, c->n_pad, c->planes, nk_out, c->dn_scratch.as<float>(),
                             c->stream);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(static_cast<char*>(out) + header.size(), c->dn_scratch.p, body, cudaMemcpyDeviceToHost,
                           c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return GS_OK;
}

int gs_save_splat(GsContext* c, void* out, int64_t capacity, int64_t* bytes_out) {
    GS_TRACE("gs_save_splat");
    CTX_CHECK(c);
    if (!bytes_out) return fail(GS_ERR_INVALID_ARG, "bytes_out is null");
    const int n = c->n;
    std::vector<unsigned char> rec((size_t)n * 32), finite((size_t)n);
    std::vector<double> weight((size_t)n);
    if (n > 0) {
        const size_t need = (size_t)n * (32 + 8 + 1) + 64;
        CKI(ensure(c->dn_scratch, need, c));
        unsigned char* d_rec = c->dn_scratch.as<unsigned char>();
        double* d_w = reinterpret_cast<double*>(d_rec + (size_t)n * 32);
        unsigned char* d_f = reinterpret_cast<unsigned char*>(d_w + n);
        launch_splat_records(c->params.as<float>(), n, c->n_pad, d_rec, d_w, d_f, c->stream);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(rec.data(), d_rec, (size_t)n * 32, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(weight.data(), d_w, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(finite.data(), d_f, (size_t)n, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    const std::vector<int> order = splat_order(weight, finite);
    const int64_t total = (int64_t)order.size() * 32;
    *bytes_out = total;
    if (!out) return GS_OK;
    if (capacity < total) return fail(GS_ERR_CAPACITY, "buffer holds %lld of %lld bytes", (long long)capacity,
                                      (long long)total);
    unsigned char* o = static_cast<unsigned char*>(out);
    for (size_t k = 0; k < order.size(); k++) memcpy(o + k * 32, rec.data() + (size_t)order[k] * 32, 32);
    return GS_OK;
}

// ---- densification ------------------------------------------------------------------
int gs_set_densify_stats(GsContext* c, int32_t enable) {
    CTX_CHECK(c);
    const bool on = enable != 0;
    if (on != c->stats_on) {
        c->stats_on = on;
        drop_graphs(c);  // the step graphs hold (or lack) the statistics kernels
    }
    return GS_OK;
}

int gs_reset_densify_stats(GsContext* c) {
    CTX_CHECK(c);
    if (c->stats.p) CK(cudaMemsetAsync(c->stats.p, 0, (size_t)2 * c->n_pad * 4, c->stream));
    return GS_OK;
}

int gs_get_densify_stats(GsContext* c, float* sums, float* counts) {
    CTX_CHECK(c);
    if ((!sums || !counts) && c->n > 0) return fail(GS_ERR_INVALID_ARG, "null output");
    if (c->n == 0) return GS_OK;
    CK(cudaMemcpyAsync(sums, c->stats.p, (size_t)c->n * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(counts, c->stats.as<float>() + c->n_pad, (size_t)c->n * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return GS_OK;
}

void gs_densify_config_default(GsDensifyConfig* d) {
    if (!d) return;
    memset(d, 0, sizeof *d);
    d->grad_threshold = 2e-4;
    d->size_threshold = 0.1;
    d->min_opacity = 0.005;
    d->max_count = 400000;
    d->max_size = INFINITY;
    d->seed = 0;
}

int gs_densify(GsContext* c, const GsDensifyConfig* d, int32_t* new_count) {
    GS_TRACE("gs_densify");
    CTX_CHECK(c);
    if (!d) return fail(GS_ERR_INVALID_ARG, "config is null");
    if (std::isnan(d->grad_threshold) || std::isnan(d->size_threshold) || std::isnan(d->min_opacity) ||
        std::isnan(d->max_size) || d->max_count < 0)
        return fail(GS_ERR_INVALID_ARG, "bad densify config");
    if (c->n == 0) {
        if (new_count) *new_count = 0;
        return GS_OK;
    }
    const int blocks = densify_blocks(c->n);
    CKI(ensure(c->dn_scratch, (size_t)blocks * 8 + 64, c));
    DensifyArgs a;
    memset(&a, 0, sizeof a);
    a.params = c->params.as<float>();
    a.stats = c->stats.as<float>();
    a.n = c->n;
    a.n_pad = c->n_pad;
    a.planes = c->planes;
    a.grad_threshold = d->grad_threshold;
    a.size_threshold = d->size_threshold;
    a.min_opacity = d->min_opacity;
    a.max_size = d->max_size;
    a.log_split = std::log(1.6);
    a.room = (long long)d->max_count - c->n;
    a.seed = d->seed;
    a.block_sums = reinterpret_cast<uint2*>(c->dn_scratch.p);
    a.result = reinterpret_cast<unsigned*>(c->dn_scratch.as<char>() + (size_t)blocks * 8);
    launch_densify_count(a, c->stream);
    CK(cudaGetLastError());
    unsigned res[3] = {0, 0, 0};
    CK(cudaMemcpyAsync(res, a.result, sizeof res, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const int new_n = (int)res[2];
    if (res[2] > (1u << 28)) return fail(GS_ERR_CAPACITY, "densified set too large (%u)", res[2]);
    // The new planes go into the first moment's buffer, which becomes the parameters;
    // the old parameter buffer becomes the first moment (zeroed below).
    const int new_np = new_n > 0 ? ((new_n + 127) / 128) * 128 : 128;
    CKI(ensure(c->mom1, (size_t)c->planes * new_np * 4, c));
    a.out = c->mom1.as<float>();
    a.out_n_pad = new_np;
    launch_densify_scatter(a, new_n, c->stream);
    CK(cudaGetLastError());
    std::swap(c->params, c->mom1);
    c->generation = ++g_generation_counter;
    CKI(resize_scene(c, new_n, true));
    CK(cudaStreamSynchronize(c->stream));
    if (new_count) *new_count = new_n;
    return GS_OK;
}

int gs_reset_opacity(GsContext* c, double max_logit) {
    CTX_CHECK(c);
    if (std::isnan(max_logit)) return fail(GS_ERR_INVALID_ARG, "max_logit is NaN");
    launch_opacity_cap(c->params.as<float>() + (size_t)10 * c->n_pad, c->n, max_logit, c->stream);
    CK(cudaGetLastError());
    return GS_OK;
}

int gs_scene_extent(const GsCamera* cams, int32_t count, float* extent_out) {
    if (!cams || count < 1 || !extent_out) return fail(GS_ERR_INVALID_ARG, "bad cameras");
    // Camera centres -R^T t in double, as the reference's JavaScript does.
    std::vector<double> cx(count), cy(count), cz(count);
    double mx = 0, my = 0, mz = 0;
    for (int k = 0; k < count; k++) {
        const float* m = cams[k].view;
        cx[k] = -((double)m[0] * m[3] + (double)m[4] * m[7] + (double)m[8] * m[11]);
        cy[k] = -((double)m[1] * m[3] + (double)m[5] * m[7] + (double)m[9] * m[11]);
        cz[k] = -((double)m[2] * m[3] + (double)m[6] * m[7] + (double)m[10] * m[11]);
        mx += cx[k];
        my += cy[k];
        mz += cz[k];
    }
    mx /= count;
    my /= count;
    mz /= count;
    double far = 1e-3;
    for (int k = 0; k < count; k++) far = std::max(far, std::hypot(cx[k] - mx, cy[k] - my, cz[k] - mz));
    *extent_out = (float)(1.1 * far);
    return GS_OK;
}

// Switches the context to tiles of `tile` pixels: views re-laid out, the instance
// capacity measured again by the next forward, graphs re-captured.
static int set_tile(GsContext* c, int tile) {
    if (c->tile == tile) return GS_OK;
    c->tile = tile;
    // Keep raster variants that exist for the new tile size.
    for (int* v : {&c->ppt_fwd, &c->ppt_bwd})
        if (tile == 8) *v = 2;
    if (!raster_variant_ok(tile, c->wt_fwd, c->ppt_fwd)) c->wt_fwd = tile == 64 ? 16 : tile;
    if (!raster_variant_ok(tile, c->wt_bwd, c->ppt_bwd)) c->wt_bwd = tile == 64 ? 16 : tile;
    CKI(layout(c));
    // The instance buffers are sized again for this tile size: the sort and emission
    // grids follow their capacity, which another tile size may have grown.
    for (DevBuf* b : {&c->ikeys, &c->ivals, &c->ikeys_alt, &c->ivals_alt, &c->block_first_pair}) release(*b);
    c->inst_cap = 0;
    c->inst_cap_valid = false;
    c->have_loss = false;
    c->last_first = -1;
    c->ctas_fwd = persistent_ctas(c, false);
    c->ctas_bwd = persistent_ctas(c, true);
    drop_graphs(c);
    return GS_OK;
}

// Tuning: for each tile size (16, 8, 32, 64) the persistent forward and backward raster
// kernels are timed for every (work tile, shared-memory batch, pixels per thread)
// variant that exists for it, on all training views after one forward and loss, keeping
// the fastest of each; then the tile size's whole forward + loss + backward (projection,
// binning, blending, loss, their backward; no update) is timed with those variants, and
// the tile size with the fastest is kept.  The choice is cached per device and workload
// in `cache_path` (lines "key|tile fwd_batch fwd_ppt fwd_wt bwd_batch bwd_ppt bwd_wt").
int gs_autotune(GsContext* c, const char* cache_path) {
    GS_TRACE("gs_autotune");
    CTX_CHECK(c);
    if (c->V < 1 || c->n <= 0) return fail(GS_ERR_STATE, "autotune needs Gaussians and views");
    int kind;
    CKI(targets_kind(c, 0, c->V, &kind));
    char key[256];
    snprintf(key, sizeof key, "%s n=%d views=%d px=%lld deg=%d", c->device_name.c_str(), c->n, c->V,
             (long long)c->total_pixels, c->degree);
    auto apply = [&](int tile, int bf, int pf, int wf, int bb, int pb, int wb) -> int {
        CKI(set_tile(c, tile));
        c->batch_fwd = bf;
        c->ppt_fwd = pf;
        c->wt_fwd = wf;
        c->batch_bwd = bb;
        c->ppt_bwd = pb;
        c->wt_bwd = wb;
        c->ctas_fwd = persistent_ctas(c, false);
        c->ctas_bwd = persistent_ctas(c, true);
        drop_graphs(c);
        return GS_OK;
    };
    auto ok_batch = [](int b) { return b == 32 || b == 64 || b == 128 || b == 256; };
    if (cache_path) {
        FILE* f = fopen(cache_path, "r");
        if (f) {
            char line[512];
            while (fgets(line, sizeof line, f)) {
                int t, bf, pf, wf, bb, pb, wb;
                char* bar = strrchr(line, '|');
                if (!bar) continue;
                *bar = 0;
                if (strcmp(line, key) == 0 &&
                    sscanf(bar + 1, "%d %d %d %d %d %d %d", &t, &bf, &pf, &wf, &bb, &pb, &wb) == 7 && ok_batch(bf) &&
                    ok_batch(bb) && raster_variant_ok(t, wf, pf) && raster_variant_ok(t, wb, pb)) {
                    fclose(f);
                    return apply(t, bf, pf, wf, bb, pb, wb);
                }
            }
            fclose(f);
        }
    }
    const int saved_batched = c->cfg.batched;
    DevStatus* st = c->status.as<DevStatus>();
    const int batches[4] = {32, 64, 128, 256};
    const int tiles[4] = {16, 8, 32, 64};
    const GsLossConfig lc{0.2f, 1};
    cudaEvent_t e0 = c->user_events[62], e1 = c->user_events[63];
    float best_total = 1e30f;
    int best[7] = {c->tile, c->batch_fwd, c->ppt_fwd, c->wt_fwd, c->batch_bwd, c->ppt_bwd, c->wt_bwd};
    int64_t inst16 = -1;  // key instances with 16-pixel tiles (measured first)
    for (int ti = 0; ti < 4; ti++) {
        const int tile = tiles[ti];
        if (inst16 >= 0) {
            // A tile size whose instance buffers would not fit is skipped: instances scale
            // about as the inverse tile area (heavy-tailed scenes with splats over hundreds
            // of tiles reach billions of 8-pixel instances).
            size_t free_b = 0, total_b = 0;
            CK(cudaMemGetInfo(&free_b, &total_b));
            const double est = (double)inst16 * (16.0 / tile) * (16.0 / tile) * 1.25;
            const double need = est * 20.0;  // keys, values, their alternates, emission
            if (est > 2.0e9 || need > 0.5 * (double)(free_b + (size_t)c->inst_cap * 16)) continue;
        }
        CKI(set_tile(c, tile));
        c->cfg.batched = 1;
        int rc = run_forward(c, 0, c->V);
        c->cfg.batched = saved_batched;
        CKI(rc);
        if (tile == 16) inst16 = (int64_t)c->status_host->instances_needed;
        CKI(gs_loss(c, &lc, nullptr));
        float best_f = 1e30f, best_b = 1e30f;
        int bf = 0, pf = 0, wf = 0, bb = 0, pb = 0, wb = 0;
        RasterArgs r = raster_args(c, 0, c->V);
        if (c->cfg.lpt_order) r.tile_order = c->tile_order.as<uint32_t>();
        for (int bi = 0; bi < 4; bi++)
            for (int vi = 0; vi < 6; vi++) {
                const int ppt = 2 << (vi % 3), wt = tile == 64 ? (vi < 3 ? 16 : 0) : (vi < 3 ? tile : tile / 2);
                if (!raster_variant_ok(tile, wt, ppt)) continue;
                for (int backward = 0; backward < 2; backward++) {
                    const int ctas =
                        c->num_sms * raster_max_ctas_per_sm(tile, wt, batches[bi], ppt, backward != 0);
                    float total = 0.f;
                    for (int rep = 0; rep < 3; rep++) {
                        CK(cudaMemsetAsync(&st->work_counter, 0, 8, c->stream));
                        if (backward) {
                            CK(cudaMemsetAsync(c->sg8.p, 0, (size_t)c->V * c->n_pad * 32, c->stream));
                            CK(cudaMemsetAsync(c->sg1.p, 0, (size_t)c->V * c->n_pad * 4, c->stream));
                        }
                        CK(cudaEventRecord(e0, c->stream));
                        if (backward) {
                            r.work_counter = &st->work_counter_bwd;
                            launch_raster_bwd(r, tile, wt, batches[bi], ppt, ctas, c->stream);
                        } else {
                            r.work_counter = &st->work_counter;
                            launch_raster_fwd(r, tile, wt, batches[bi], ppt, ctas, c->stream);
                        }
                        CK(cudaEventRecord(e1, c->stream));
                        CK(cudaGetLastError());
                        CK(cudaEventSynchronize(e1));
                        float ms = 0.f;
                        CK(cudaEventElapsedTime(&ms, e0, e1));
                        if (rep > 0) total += ms;
                    }
                    if (backward && total < best_b) {
                        best_b = total;
                        bb = batches[bi];
                        pb = ppt;
                        wb = wt;
                    }
                    if (!backward && total < best_f) {
                        best_f = total;
                        bf = batches[bi];
                        pf = ppt;
                        wf = wt;
                    }
                }
            }
        CKI(apply(tile, bf, pf, wf, bb, pb, wb));
        // The tile size's whole forward, loss and backward with its best variants.
        float total = 0.f;
        for (int rep = 0; rep < 3; rep++) {
            CK(cudaMemsetAsync(c->acc.p, 0, sizeof(double) * 2 * (GS_MAX_VIEWS + 1), c->stream));
            CK(cudaEventRecord(e0, c->stream));
            CKI(enqueue_forward(c, 0, c->V, true));
            CKI(enqueue_loss_view(c, 0, c->V, lc, kind));
            CKI(enqueue_backward_view(c, 0, 0, c->V, true, false));
            CK(cudaEventRecord(e1, c->stream));
            CK(cudaEventSynchronize(e1));
            CKI(read_status(c));
            if (c->status_host->overflow) return fail(GS_ERR_CAPACITY, "key instances overflowed while tuning");
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            if (rep > 0) total += ms;
        }
        if (total < best_total) {
            best_total = total;
            best[0] = tile;
            best[1] = bf;
            best[2] = pf;
            best[3] = wf;
            best[4] = bb;
            best[5] = pb;
            best[6] = wb;
        }
    }
    CKI(apply(best[0], best[1], best[2], best[3], best[4], best[5], best[6]));
    c->have_loss = false;
    c->last_first = -1;
    if (cache_path) {
        FILE* f = fopen(cache_path, "a");
        if (f) {
            fprintf(f, "%s|%d %d %d %d %d %d %d\n", key, best[0], best[1], best[2], best[3], best[4], best[5],
                    best[6]);
            fclose(f);
        }
    }
    return GS_OK;
}

}  // extern "C"
