/*
 * gsb200.h -- C ABI of the B200-native Gaussian-splat training step.
 *
 * This is the boundary a host binding (the Node-API addon behind the trainer's
 * JavaScript module, or the Python ctypes mirror in this repository) calls.  Every
 * entry point takes plain pointers and sizes, copies caller-owned host memory before
 * it returns (unless stated otherwise), and returns an int status: GS_OK (0) or a
 * negative GS_ERR_* code, with a message from gs_last_error().
 *
 * The reference is the WebGPU trainer of barakatiass-alt/home-measure-privacy.  Each
 * entry point names the function of trainer/gpu.js (or trainer/colmap.js) it stands
 * in for.  Device memory is owned by the context and grows on demand, like the
 * reference's pooled scratch buffers (trainer/gpu.js:764-772).  A context is bound to
 * one CUDA device and one stream and is not re-entrant: callers serialise calls on a
 * context (the reference's JS event loop does the same).
 */
#ifndef GSB200_H
#define GSB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GSB200_VERSION 1

#if defined(__GNUC__)
#define GS_API __attribute__((visibility("default")))
#else
#define GS_API
#endif

/* ---- status codes ------------------------------------------------------------- */
#define GS_OK               0
#define GS_ERR_INVALID_ARG -1   /* bad pointer, size or option                     */
#define GS_ERR_CUDA        -2   /* a CUDA runtime call failed                      */
#define GS_ERR_CAPACITY    -3   /* an instance buffer overflowed; step was skipped */
#define GS_ERR_NO_DEVICE   -4   /* no CUDA device visible                          */
#define GS_ERR_STATE       -5   /* call out of order (no scene / no views / ...)   */
#define GS_ERR_NONFINITE   -6   /* a non-finite loss or parameter was detected     */
#define GS_ERR_COMM        -7   /* the data-parallel exchange (NCCL) failed        */

/* ---- plain data types ---------------------------------------------------------- */

/* One pinhole camera.  Same fields as trainerCamera() (trainer/colmap.js:57-64) and the
 * 80-byte camera uniform (trainer/gpu.js:16, :696-701): view = row-major world-to-camera
 * [R | t] (12 floats, trainer/colmap.js:46-54), intrinsics in pixels, size in pixels. */
typedef struct GsCamera {
    float view[12];
    float fx, fy, cx, cy;
    int32_t width, height;
} GsCamera;

/* Per-context options.  Defaults (gs_config_default) are the reference's hard-coded
 * constants: near 0.2 (trainer/gpu.js:36), EWA dilation 0.3 (:45-47), alpha cap 0.99 and
 * floor 1/255 (:100-101), transmittance stop 1e-4 (:124), 16-pixel tiles (:118). */
typedef struct GsConfig {
    float near_plane;      /* cull when camera-space z < near_plane                    */
    float cov_dilation;    /* added to the 2D covariance diagonal                      */
    float alpha_max;       /* alpha clamp                                              */
    float alpha_min;       /* alphas below this are skipped                           */
    float t_min;           /* stop a pixel once T <= t_min                             */
    int32_t sh_degree;     /* 0..3; degree 0 = the reference's raw RGB colour          */
    int32_t rect_mode;     /* 0 = BIN tile rectangle (trainer/gpu.js:632-635, default),
                              1 = tileLists() rectangle (trainer/gpu.js:456-461)        */
    int32_t batched;       /* 1 = one persistent (view, tile) launch for all views;
                              0 = the plain path: one launch per view per stage        */
    int32_t use_graph;     /* 1 = capture each training step in a CUDA graph           */
    int32_t device;        /* CUDA device ordinal                                     */
    int32_t autotune;      /* 1 = run gs_autotune before the first training step over
                              all views                                                 */
    int32_t raster_batch;  /* Gaussians per shared-memory batch: 32, 64, 128 or 256    */
    int32_t lpt_order;     /* 1 = persistent raster takes heavy tiles first           */
    int32_t instance_capacity; /* initial key-instance capacity; 0 = measured by a first
                              forward.  A step that overflows skips its update, the
                              buffer grows and a synchronous step is redone.           */
    int32_t raster_ppt;    /* pixels per raster thread: 2 (128 threads per 16 x 16
                              tile), 4 (64 threads) or 8 (one warp per tile); 8-pixel
                              tiles take 2 only; 0 = 4 (2 for 8-pixel tiles)            */
    int32_t tile_cull;     /* 1 (default) = a tile list holds only splats whose
                              alpha >= alpha_min ellipse reaches the tile: same images
                              and gradients, fewer entries; 0 = the reference's
                              rectangle lists (rect_mode), whose keys match BIN + SORT  */
    int32_t tile_size;     /* tile edge in pixels: 16 (default, the reference's,
                              trainer/gpu.js:118), 8, 32 or 64; 0 = 16.  Images are the
                              same for every size; gs_autotune may change it            */
    int32_t raster_work_tile; /* pixels a raster CTA covers: the whole tile (0 or the
                              tile edge) or, for 32- and 64-pixel tiles, 16 (each 16 x
                              16 part a CTA of its own, walking the tile's list); 64-
                              pixel tiles take 16 only (0 = 16)                        */
} GsConfig;

/* Adam settings.  The per-group learning rates are the reference's (trainer/gpu.js:846,
 * :891); beta1/beta2/eps are fixed in the reference's ADAM kernel (:431-435). lr_sh is
 * the rate for SH bands >= 1, which the reference does not have. */
typedef struct GsAdamConfig {
    float lr_color, lr_opacity, lr_mean, lr_scale, lr_rotation, lr_sh;
    float beta1, beta2, eps;
} GsAdamConfig;

/* Loss settings: (1 - ssim_lambda) * L1 + ssim_lambda * (1 - SSIM), the reference's
 * lossGradient (trainer/gpu.js:742-753).  window 0 = 7x7 box windows fully inside the
 * image (SSIM_COEF, trainer/gpu.js:336-372); window 1 = 11-tap Gaussian, sigma 1.5,
 * windows fully inside the image. */
typedef struct GsLossConfig {
    float ssim_lambda;
    int32_t window;
} GsLossConfig;

typedef struct GsContext GsContext;

/* ---- context -------------------------------------------------------------------- */

/* Fills *cfg with the reference's constants.  Replaces the defaults of
 * createRenderer() (trainer/gpu.js:704). */
GS_API void gs_config_default(GsConfig* cfg);
GS_API void gs_adam_default(GsAdamConfig* adam);   /* trainScene lr defaults, gpu.js:891 */

/* createRenderer() (trainer/gpu.js:704-712): binds a device, builds the kernels' state.
 * Returns GS_ERR_NO_DEVICE when no CUDA device is visible; there is no CPU fallback. */
GS_API int gs_create(const GsConfig* cfg, GsContext** out);
GS_API int gs_destroy(GsContext* ctx);

/* Message of the last failed call on this thread (never NULL). */
GS_API const char* gs_last_error(void);
GS_API const char* gs_status_string(int status);

/* Number of floats one Gaussian takes in the host parameter record at `sh_degree`:
 * 14 + 3 * ((sh_degree + 1)^2 - 1).  Record order: mean[3], logScale[3],
 * rotation[4] (w, x, y, z), opacityLogit, color[3] (the SH DC term, the reference's raw
 * RGB), then the SH bands >= 1 channel-major (R coefficients 1..K-1, then G, then B),
 * which is the order of a 3DGS .ply's f_rest_* properties. */
GS_API int gs_param_stride(int sh_degree);

/* ---- scene ---------------------------------------------------------------------- */

/* Upload n Gaussians in the host record layout above (gs_param_stride floats each).
 * Resets the Adam moments and step counter, as upload() does (trainer/gpu.js:901-908). */
GS_API int gs_set_gaussians(GsContext* ctx, int32_t n, const float* params);

/* Upload n Gaussians in the reference's packed 16-float layout (packGaussians,
 * trainer/gpu.js:5-6, :688-694); SH bands >= 1 are set to zero. */
GS_API int gs_set_gaussians_packed(GsContext* ctx, int32_t n, const float* packed16);

/* Read the current Gaussians back (host record layout, or the reference's packed
 * 16-float layout as unpackGaussians expects, trainer/gpu.js:602-609). */
GS_API int gs_get_gaussians(GsContext* ctx, float* params_out);
GS_API int gs_get_gaussians_packed(GsContext* ctx, float* packed16_out);
GS_API int32_t gs_num_gaussians(const GsContext* ctx);

/* ---- views ---------------------------------------------------------------------- */

/* The training views' cameras (trainer/dataset.js:74 view.cam).  Allocates the
 * per-pixel buffers for all of them; targets are set separately. */
GS_API int gs_set_views(GsContext* ctx, int32_t num_views, const GsCamera* cams);

/* Target photo of one view: RGB bytes, as decoded by loadDataset (trainer/dataset.js:74;
 * divided by 255 on the device, as trainer/gpu.js:921 does on the host), or RGB floats
 * (train(), trainer/gpu.js:852-856).  width * height * 3 values, row-major HWC. */
GS_API int gs_set_target_u8(GsContext* ctx, int32_t view, const uint8_t* rgb);
GS_API int gs_set_target_f32(GsContext* ctx, int32_t view, const float* rgb);

/* ---- the Function pair: forward and backward ------------------------------------- */

/* render() (trainer/gpu.js:815-820): project, bin, sort and blend the current scene
 * from one camera.  rgb_out: width * height * 3 floats, HWC, black background,
 * unclamped.  state_out (optional, width * height * 2): final transmittance and, as a
 * float, how many entries of the pixel's tile list the blend consumed
 * (trainer/gpu.js:133-136, counted from the tile's start). */
GS_API int gs_render(GsContext* ctx, const GsCamera* cam, float* rgb_out, float* state_out);

/* forward() of views [first, first + count) in one batched pass (or one view per
 * launch when cfg.batched == 0).  images_out (optional): the views' images
 * concatenated, each width * height * 3 floats.  The rasteriser state is kept on the
 * device for gs_backward. */
GS_API int gs_forward(GsContext* ctx, int32_t first_view, int32_t num_views, float* images_out);

/* backward() for the views of the last gs_forward.  dl_dimages (host, optional):
 * dLoss/dPixel for every view, laid out like images_out; when NULL the loss gradient
 * of gs_loss (below) is used.  Fills the parameter gradients kept on the device; read
 * them with gs_get_param_grads.  The reference's BACKWARD/BACKWARD_SG + SHAPE
 * (trainer/gpu.js:139-328, :756-761), with the projection chained analytically. */
GS_API int gs_backward(GsContext* ctx, const float* dl_dimages);

/* Loss and dLoss/dPixel of the last gs_forward against the views' targets
 * (lossGradient, trainer/gpu.js:742-753).  loss_out (optional): the mean loss over
 * the views. */
GS_API int gs_loss(GsContext* ctx, const GsLossConfig* loss, float* loss_out);

/* Parameter gradients of the last gs_backward, host record layout. */
GS_API int gs_get_param_grads(GsContext* ctx, float* grads_out);

/* Screen-space gradients of the last gs_backward for one of its views, in the
 * reference's 16-float per-Gaussian layout (trainer/gpu.js:9-10): 0-2 colour,
 * 3 opacity logit, 4-8 (u, v, conicA, conicB, conicC), 9-15 zero. */
GS_API int gs_get_screen_grads(GsContext* ctx, int32_t view, float* grads16_out);

/* gradients() (trainer/gpu.js:826-839) for the current scene and one camera against a
 * float target: image (W*H*3), grads (n*16, as gs_get_screen_grads) and shape
 * (n*10: mean[3], logScale[3], rotation[4]).  Shape gradients are analytic; the
 * reference takes them by finite differences (trainer/gpu.js:297-328). */
GS_API int gs_gradients(GsContext* ctx, const GsCamera* cam, const float* target,
                 float ssim_lambda, float* image_out, float* grads16_out,
                 float* shape10_out);

/* lossGradientOf() (trainer/gpu.js:962-977): dLoss/dPixel of an image against a
 * target, both width * height * 3 floats, with the reference's 7x7 box SSIM
 * (window 0) or the 11-tap Gaussian window (window 1). */
GS_API int gs_loss_gradient(GsContext* ctx, const float* image, const float* target,
                     int32_t width, int32_t height, float ssim_lambda, int32_t window,
                     float* grad_out, float* loss_out);

/* ---- training ------------------------------------------------------------------- */

/* One training step over views [first, first + count): forward, loss, backward and
 * Adam with step counter t + 1, against the targets already on the device.  With
 * cfg.use_graph the whole step is one CUDA graph launch.  loss_out (optional) makes
 * the call wait for the step and return its mean loss; without it the call returns
 * once the step is queued.  The ADAM kernel's rules are kept (trainer/gpu.js:411-443):
 * colour clamped to [0, 1], rotation renormalised. */
GS_API int gs_train_step(GsContext* ctx, const GsAdamConfig* adam, const GsLossConfig* loss,
                  int32_t first_view, int32_t num_views, float* loss_out);

/* The same step, with this step's targets given as host RGB bytes (the views'
 * images concatenated) and copied to the device inside the step, then the loss copied
 * back: the per-step host traffic of trainScene (trainer/gpu.js:918-921, :934-940).
 * Use gs_host_alloc for the target buffer to copy from pinned memory. */
GS_API int gs_train_step_host(GsContext* ctx, const GsAdamConfig* adam, const GsLossConfig* loss,
                       int32_t first_view, int32_t num_views, const uint8_t* targets_u8,
                       float* loss_out);

/* gs_train_step_host, pipelined: the step's photos go host -> device on a separate copy
 * stream while the previous step still runs, and the loss comes back by an asynchronous
 * copy into loss_out when the step completes; the call returns once the step is queued.
 * At most two steps are in flight: a call first waits for the step queued two calls
 * earlier, so after call k returns the loss of step k - 2 is in its buffer and that
 * step's targets_u8 may be reused.  targets_u8 and loss_out should be pinned
 * (gs_host_alloc) for the copies to overlap.  A step whose key instances overflow skips
 * its update; the buffers grow before the next step (no redo).  gs_synchronize waits for
 * all. */
GS_API int gs_train_step_host_async(GsContext* ctx, const GsAdamConfig* adam, const GsLossConfig* loss,
                                    int32_t first_view, int32_t num_views, const uint8_t* targets_u8,
                                    float* loss_out);

/* train() (trainer/gpu.js:846-878): `steps` steps of L1 loss, one view per step in
 * order, through the plain per-pixel path; losses_out[steps] gets each step's mean
 * L1 (the reference reads the image back every step). */
GS_API int gs_train(GsContext* ctx, int32_t steps, const GsAdamConfig* adam, float* losses_out);

/* Data-parallel split of gs_train_step, for replicas that hold the same Gaussians and
 * train on different views (one process per GPU).  The reference trains on one device
 * and has no counterpart; the pair replaces trainScene's step (trainer/gpu.js:915-933)
 * when its views are spread over several GPUs.
 *
 * gs_step_gradients queues forward, loss and backward of views [first, first+count) on
 * the context's stream and leaves the parameter gradients in the context's gradient
 * buffer: num_params x n_pad floats (plane-major, n_pad = n rounded up to 128), then
 * 2 x n_pad floats of this step's densification statistics (zero unless enabled), then
 * GS_GRAD_TAIL_FLOATS floats: [0] the sum over these views of their mean losses,
 * [1] 1 if the step's key instances overflowed their buffer, [2] the view count, rest 0.
 * *grads_device gets the buffer's device address and *num_floats its length.  Sum the
 * whole buffer across replicas (e.g. an NCCL all-reduce on gs_get_stream's stream),
 * then call gs_step_apply.  The address stays valid until the scene changes size. */
#define GS_GRAD_TAIL_FLOATS 64
GS_API int gs_step_gradients(GsContext* ctx, const GsLossConfig* loss, int32_t first_view, int32_t num_views,
                             float** grads_device, int64_t* num_floats);

/* Adam update from the (reduced) gradient buffer, queued on the context's stream.  The
 * update is skipped on every replica when the reduced overflow count is non-zero; the
 * instance buffer of the replica that overflowed grows before its next step, so the
 * caller repeats the step.  loss_out (nullable, waits for the step) gets the mean loss
 * over all reduced views; skipped_out (nullable, waits) gets 1 for a skipped update. */
GS_API int gs_step_apply(GsContext* ctx, const GsAdamConfig* adam, float* loss_out, int32_t* skipped_out);

/* The context's CUDA stream (a cudaStream_t), for work the caller orders with the
 * library's: a collective over gs_step_gradients' buffer, a copy, an event. */
GS_API int gs_get_stream(GsContext* ctx, void** stream_out);

/* Data parallel without a framework: NCCL (opened at run time; a libnccl already loaded
 * in the process is shared) sums the gradient buffer across replicas on the context's
 * stream.  Rank 0 makes an id (gs_dp_unique_id, 128 bytes), every rank receives it by
 * any means (a socket, a file) and calls gs_dp_init with its rank; then each step is
 * gs_step_gradients (own views), gs_dp_allreduce, gs_step_apply.  gs_dp_init waits for
 * all `world` ranks.  GS_ERR_COMM when NCCL is missing or fails.  Replaces the single
 * device of the reference (trainer/gpu.js:915-933: one view per step on one WebGPU
 * device); there is no reference interface for it. */
GS_API int gs_dp_unique_id(void* id_out, int32_t bytes);
GS_API int gs_dp_init(GsContext* ctx, const void* id, int32_t bytes, int32_t rank, int32_t world);
GS_API int gs_dp_allreduce(GsContext* ctx);
GS_API int gs_dp_finalize(GsContext* ctx);

/* ---- Initialisation from a point cloud ----------------------------------------------
 * neighbourSizes (trainer/neighbours.js:13-53): per point, the root mean square distance
 * to its 3 nearest other points within the 27 cubes of 0.1 m around its own, clamped to
 * [min_size, max_size], or `fallback` when there is none.  xyz: count x 3 floats.
 * sizes_out: count floats. */
GS_API int gs_neighbour_sizes(GsContext* ctx, const float* xyz, int32_t count, double min_size, double max_size,
                              double fallback, float* sizes_out);

/* initFromPoints (trainer/gpu.js:507-521): replaces the context's Gaussians with one per
 * point: log-size on all axes (`size` > 0 for all, else neighbourSizes with the
 * reference's defaults 0.005 / 0.1 / 0.06), identity rotation, opacity 0.1, the point's
 * colour (rgb: count x 3 floats in [0, 1]); SH bands zero. */
GS_API int gs_init_from_points(GsContext* ctx, const float* xyz, const float* rgb, int32_t count, float size);

/* ---- Photo selection (trainer/sharpness.js, trainer/dataset.js:35-47) -------------------
 * sharpness(grey, width, height): variance of the 4-neighbour Laplacian over the interior
 * pixels, for `count` images of one size at once (channels = 1: grey bytes; 3: RGB bytes,
 * turned grey as (77 R + 150 G + 29 B) >> 8).  The reference measures it on a 160-pixel-
 * wide copy the browser scales; the caller passes the images at the size to score. */
GS_API int gs_sharpness(GsContext* ctx, const uint8_t* images, int32_t count, int32_t width, int32_t height,
                        int32_t channels, double* scores);

/* chooseSharp(scores, maxViews) (trainer/sharpness.js:39-55): the sharpest photo of
 * each of max_views stretches of the walk, without the blurriest (below 0.35 x the
 * median, at most a quarter).  chosen: room for min(count, max_views) indices.  Host only. */
GS_API int gs_choose_sharp(const double* scores, int32_t count, int32_t max_views, int32_t* chosen,
                           int32_t* chosen_count);

/* ---- Scene files ---------------------------------------------------------------------
 * fromPly (trainer/gpu.js:983-999): replaces the context's Gaussians with a binary
 * little-endian .ply of float vertex properties (x y z, scale_0..2, rot_0..3 w x y z,
 * opacity, f_dc_0..2 required; colour = clamp(f_dc SH0 + 0.5, 0, 1)), and, beyond the
 * reference, the f_rest_* bands up to the context's SH degree (channel-major; missing
 * bands are zero).  The header is looked for in the first 4096 bytes, as the reference
 * does.  The file's body goes to the device unchanged and is transposed there. */
GS_API int gs_load_ply(GsContext* ctx, const void* data, int64_t bytes, int32_t* count_out);

/* toPly (trainer/gpu.js:524-531): with_sh = 0 gives the reference's 17 properties
 * (x y z nx ny nz f_dc_0..2 opacity scale_0..2 rot_0..3, f_dc = (colour - 0.5) / SH0);
 * with_sh = 1 adds f_rest_* after f_dc (the 3DGS order).  out = NULL: *bytes_out gets
 * the size only. */
GS_API int gs_save_ply(GsContext* ctx, int32_t with_sh, void* out, int64_t capacity, int64_t* bytes_out);

/* toSplat (trainer/gpu.js:538-556): 32 bytes per finite Gaussian (position, scales,
 * colour / opacity / rotation bytes), largest exp(sum log-scales) x opacity first, ties
 * in index order.  out = NULL: *bytes_out gets the size only. */
GS_API int gs_save_splat(GsContext* ctx, void* out, int64_t capacity, int64_t* bytes_out);

/* ---- Densification (trainer/gpu.js:484-497 STATS, :564-599 sceneExtent / densify,
 * :902-903 and :944 the opacity reset) --------------------------------------------------
 * The reference reads every Gaussian back to the host each densification, densifies in
 * JavaScript and uploads the result with fresh moments and statistics.  Here all of it
 * stays on the device. */

/* STATS: while enabled, every training step (gs_train_step, gs_train_step_host,
 * gs_step_gradients + gs_step_apply) adds, for each Gaussian and each of the step's
 * views it projects into, |(dL/du, dL/dv)| to its sum and 1 to its count.  A step whose
 * update was skipped (instance overflow) adds nothing.  Off by default. */
GS_API int gs_set_densify_stats(GsContext* ctx, int32_t enable);
GS_API int gs_reset_densify_stats(GsContext* ctx);
/* sums[n], counts[n]: the statistics since the last reset / densify / gs_set_gaussians. */
GS_API int gs_get_densify_stats(GsContext* ctx, float* sums, float* counts);

typedef struct GsDensifyConfig {
    double grad_threshold;   /* average gradient norm that densifies (reference default 2e-4;
                                trainScene passes 2e-4 / (0.5 * width of its first view)) */
    double size_threshold;   /* largest scale up to which a Gaussian is cloned, else split */
    double min_opacity;      /* sigmoid(opacity logit) below this: dropped */
    double max_size;         /* largest scale above this: dropped (INFINITY: never) */
    int32_t max_count;       /* clones and splits stop once the count would pass this */
    int32_t reserved;
    uint64_t seed;           /* split offsets: SplitMix64(seed, index, copy, axis) instead of
                                the reference's Math.random() */
} GsDensifyConfig;
GS_API void gs_densify_config_default(GsDensifyConfig* cfg);

/* densify() on the device: the new set replaces the context's Gaussians in the
 * reference's order (each kept Gaussian in place; a clone is the Gaussian then its copy;
 * a split is its two moved, shrunk copies).  Moments and statistics restart at zero,
 * the Adam step counter continues (as trainScene's t does).  *new_count gets the new
 * number of Gaussians.  Waits for the stream once (to size the new buffers). */
GS_API int gs_densify(GsContext* ctx, const GsDensifyConfig* cfg, int32_t* new_count);

/* Opacity reset: logit = min(logit, max_logit) for every Gaussian (trainScene passes
 * log(0.01 / 0.99)). */
GS_API int gs_reset_opacity(GsContext* ctx, double max_logit);

/* sceneExtent(views): 1.1 x the largest distance of a camera centre from their mean
 * (at least 1e-3).  Host only. */
GS_API int gs_scene_extent(const GsCamera* cams, int32_t count, float* extent_out);

/* Step counter t (number of Adam updates applied since gs_set_gaussians). */
GS_API int gs_get_step(GsContext* ctx, int32_t* t_out);

/* Failure-detection hook (no counterpart in the reference, whose WebGPU kernels never
 * wait on one another).  The radix sort's decoupled look-back is the one place where a
 * block waits for another; each such wait gives up after a bounded number of polls,
 * sets a flag and lets the block finish, the step then skips its Adam update, and the
 * call that reads the step's status returns GS_ERR_CUDA ("look-back wait timed out")
 * and clears the flag so the context goes on.  With polls > 0 every radix pass run on
 * this context first makes one block wait on a device word that nothing writes, giving
 * up after `polls` polls: the same path, on demand, with no fault.  0 turns it off. */
GS_API int gs_debug_lookback_wait(GsContext* ctx, int32_t polls);

/* ---- memory, timing and diagnostics ---------------------------------------------- */

/* Page-locked host memory for per-step uploads (freed with gs_host_free). */
GS_API int gs_host_alloc(size_t bytes, void** out);
GS_API int gs_host_free(void* ptr);

/* Waits for all work queued on the context's stream. */
GS_API int gs_synchronize(GsContext* ctx);

/* CUDA events on the context's stream, for timing from the host binding.
 * gs_event_record(ctx, slot) records event `slot` (0..63); gs_event_elapsed returns
 * the milliseconds between two recorded slots (waits for the later one). */
GS_API int gs_event_record(GsContext* ctx, int32_t slot);
GS_API int gs_event_elapsed(GsContext* ctx, int32_t slot_a, int32_t slot_b, float* ms_out);

/* Per-stage device times of the steps run since the last reset, summed, in
 * milliseconds, recorded with events around each stage (also inside the step's CUDA
 * graph).  names: GS_NUM_STAGES fixed stage names (see gs_stage_name). */
#define GS_NUM_STAGES 10
GS_API const char* gs_stage_name(int32_t stage);
GS_API int gs_stage_times(GsContext* ctx, double* ms_out, int64_t* launches_out,
                   int32_t* steps_out);
GS_API int gs_stage_times_reset(GsContext* ctx);
GS_API int gs_set_stage_timing(GsContext* ctx, int32_t enabled);

/* Statistics of the last forward: key instances emitted (one per (Gaussian, tile)
 * overlap), visible (Gaussian, view) pairs, blends evaluated in the forward
 * (pixel, Gaussian) pairs that contributed. */
typedef struct GsStats {
    int64_t instances;
    int64_t instance_capacity;
    int64_t visible_pairs;
    int64_t tiles;
    int64_t pixels;
    int64_t kernel_launches_per_step;
    int32_t raster_batch;
    int32_t raster_threads;
    int32_t overflow;
    int32_t raster_variant;  /* per kernel (forward in bits 0-15, backward in 16-31): batch
                                (bits 0-8) | log2(work tile edge) << 9 | pixels per
                                thread << 12                                           */
    int32_t tile_size;       /* tile edge in pixels in use (gs_autotune may have changed it) */
} GsStats;
GS_API int gs_get_stats(GsContext* ctx, GsStats* out);

/* Blends of the last forward: the sum over its pixels of the splats each pixel walked
 * through in its tile list until it stopped (the (pixel, splat) pairs of the blend loop,
 * trainer/gpu.js:114-136, which the backward replays).  Waits for the stream. */
GS_API int gs_get_blend_count(GsContext* ctx, uint64_t* blends_out);

/* Sorted tile lists of the last forward for one view, in the reference's terms
 * (tileLists, trainer/gpu.js:450-481): list_out gets the splat indices of every tile
 * of the view, front to back, concatenated in tile order (capacity list_cap);
 * ranges_out (2 per tile) gets each tile's [start, end) in list_out; keys_out
 * (optional, capacity list_cap) gets each entry's 64-bit key
 * (tile index << 32 | float bits of depth).  *count_out = entries written. */
GS_API int gs_get_tile_lists(GsContext* ctx, int32_t view, uint32_t* list_out,
                      uint32_t* ranges_out, uint64_t* keys_out, int64_t list_cap,
                      int64_t* count_out);

/* Projected splat records of the last forward for one view, in the reference's
 * 12-float layout (trainer/gpu.js:7): u, v, conicA, conicB, conicC, opacity, radius,
 * depth, r, g, b, valid. */
GS_API int gs_get_splats(GsContext* ctx, int32_t view, float* splats12_out);

/* Tuning (no counterpart in the reference, whose tile size, workgroup size and batch are
 * fixed): for each tile size (16, 8, 32 and 64 pixels) times the raster kernels'
 * candidate variants (splats per shared-memory batch, pixels per thread, work tile) on
 * the current views and keeps the fastest forward and backward, then times that tile
 * size's whole forward, loss and backward (no update) and keeps the tile size with the
 * fastest.  A tile size whose key instances would not fit in half the free device
 * memory (estimated from the 16-pixel count) is skipped.  Images do not depend on the
 * choice.  The views need targets.  cache_path (optional): a text file
 * that records the choice per device and workload. */
GS_API int gs_autotune(GsContext* ctx, const char* cache_path);

/* ---- loss gradient without allocation ------------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device memory: an
 * engine that hands out all GPU memory from its own pool (memory it did not hand out
 * does not exist for it), or a real-time loop that must not wait on the allocator.  Same result as gs_loss_gradient for each image,
 * but image, target, grad and loss are caller-owned DEVICE buffers and the call only
 * queues work on `stream` (a cudaStream_t; NULL = the legacy default stream): read the
 * outputs after synchronising it.  num_images images of width x height (RGB floats,
 * concatenated) are processed in one launch; loss (optional) gets one mean loss per
 * image.  The kernels' scratch (view descriptors, per-image loss sums) lives in one
 * static device array of GS_NOALLOC_SCRATCH_BYTES that every GPU loading the library
 * keeps until exit, sized for at most GS_NOALLOC_MAX_IMAGES images: more images return
 * GS_ERR_CAPACITY.  Nothing is allocated: no cudaMalloc, cudaFree or allocating library
 * call.  The first call on a device looks up the array's address on that device (and
 * raises the loss kernel's shared-memory limit), so make the first call on each device
 * outside any stream capture.  All calls share the array and it keeps the last call's
 * contents; each call clears the sums it accumulates, and calls that overlap on the GPU
 * (other streams or host threads on the same device) race on it.  A CUDA error already
 * pending on the calling thread (left by the caller's own work) is left pending and the
 * call returns GS_ERR_CUDA without launching anything.  Returns GS_OK or a status code;
 * it does not set gs_last_error. */
#define GS_NOALLOC_MAX_IMAGES 8
#define GS_NOALLOC_SCRATCH_BYTES 4096
GS_API int gs_loss_gradient_noalloc(const float* image, const float* target, int32_t num_images,
                                    int32_t width, int32_t height, float ssim_lambda, int32_t window,
                                    float* grad, float* loss, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GSB200_H */
