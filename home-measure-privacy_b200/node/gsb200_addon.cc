// gsb200_addon.cc -- Node-API binding of libgsb200.so (include/gsb200.h) for the JS
// module gpu_b200.js, which keeps the API of the reference's trainer/gpu.js
// (createRenderer() -> {device, render, gradients, train, trainScene, lossGradientOf},
// trainer/gpu.js:704-980).
//
// Written against the C Node-API (node_api.h, N-API version 8), no C++ wrapper library:
// * a context is a JS external whose finaliser calls gs_destroy (destroy() releases it
//   earlier);
// * calls that touch only host memory or queue little work (setGaussians, setViews,
//   setTarget*, numGaussians, sceneExtent) run synchronously;
// * calls that render, train or read results back run on the libuv thread pool
//   (napi_async_work) and return Promises, as the WebGPU versions do; typed arrays they
//   read or write are kept alive by references until the work completes;
// * a failing status becomes a rejected Promise (or a thrown Error) whose message is
//   gs_last_error() of the thread that made the call and whose `status` property is the
//   GS_ERR_* code (the reference throws Error, trainer/gpu.js:705).
// The library calls cudaSetDevice on entry, so any pool thread may run any context's
// call; gpu_b200.js serialises the calls of one context, which is not re-entrant.
#include <node_api.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "gsb200.h"

namespace {

// ---- errors -----------------------------------------------------------------------------
napi_value make_error(napi_env env, int status, const std::string& msg) {
    napi_value m = nullptr, err = nullptr, code = nullptr;
    napi_create_string_utf8(env, msg.c_str(), msg.size(), &m);
    napi_create_error(env, nullptr, m, &err);
    napi_create_int32(env, status, &code);
    napi_set_named_property(env, err, "status", code);
    return err;
}

napi_value throw_status(napi_env env, int status) {
    napi_throw(env, make_error(env, status, gs_last_error()));
    return nullptr;
}

napi_value throw_msg(napi_env env, const char* msg) {
    napi_throw_error(env, nullptr, msg);
    return nullptr;
}

#define NAPI_OK(call)                                               \
    do {                                                            \
        if ((call) != napi_ok) return throw_msg(env, "gsb200: " #call " failed"); \
    } while (0)

// ---- argument helpers -----------------------------------------------------------------
struct Args {
    size_t argc = 8;
    napi_value argv[8] = {};
};

bool get_args(napi_env env, napi_callback_info info, Args& a, size_t need) {
    if (napi_get_cb_info(env, info, &a.argc, a.argv, nullptr, nullptr) != napi_ok) return false;
    if (a.argc < need) {
        napi_throw_type_error(env, nullptr, "gsb200: too few arguments");
        return false;
    }
    return true;
}

struct Handle {
    GsContext* ctx = nullptr;
};

void finalize_handle(napi_env, void* data, void*) {
    Handle* h = static_cast<Handle*>(data);
    if (h->ctx) gs_destroy(h->ctx);
    delete h;
}

GsContext* get_ctx(napi_env env, napi_value v) {
    void* p = nullptr;
    if (napi_get_value_external(env, v, &p) != napi_ok || !p || !static_cast<Handle*>(p)->ctx) {
        napi_throw_type_error(env, nullptr, "gsb200: not a live renderer context");
        return nullptr;
    }
    return static_cast<Handle*>(p)->ctx;
}

bool get_typed(napi_env env, napi_value v, napi_typedarray_type want, void** data, size_t* len) {
    bool is = false;
    napi_is_typedarray(env, v, &is);
    napi_typedarray_type t;
    napi_value ab;
    size_t off = 0;
    if (!is || napi_get_typedarray_info(env, v, &t, len, data, &ab, &off) != napi_ok || t != want) {
        napi_throw_type_error(env, nullptr,
                              want == napi_uint8_array ? "gsb200: expected a Uint8Array" : "gsb200: expected a Float32Array");
        return false;
    }
    return true;
}

double num(napi_env env, napi_value obj, const char* name, double fallback) {
    bool has = false;
    napi_has_named_property(env, obj, name, &has);
    if (!has) return fallback;
    napi_value v;
    double d = fallback;
    if (napi_get_named_property(env, obj, name, &v) == napi_ok) {
        napi_valuetype t;
        napi_typeof(env, v, &t);
        if (t == napi_number) napi_get_value_double(env, v, &d);
        else if (t == napi_boolean) {
            bool b = false;
            napi_get_value_bool(env, v, &b);
            d = b ? 1.0 : 0.0;
        }
    }
    return d;
}

// A camera of trainerCamera() (trainer/colmap.js:57-64): {view[12], fx, fy, cx, cy,
// width, height}.
bool camera_from_js(napi_env env, napi_value obj, GsCamera* c) {
    memset(c, 0, sizeof *c);
    napi_value view;
    bool is_array = false;
    if (napi_get_named_property(env, obj, "view", &view) != napi_ok) return false;
    napi_is_array(env, view, &is_array);
    bool is_typed = false;
    napi_is_typedarray(env, view, &is_typed);
    if (!is_array && !is_typed) {
        napi_throw_type_error(env, nullptr, "gsb200: camera.view must hold 12 numbers");
        return false;
    }
    for (uint32_t k = 0; k < 12; k++) {
        napi_value e;
        double d = 0.0;
        if (napi_get_element(env, view, k, &e) != napi_ok || napi_get_value_double(env, e, &d) != napi_ok) {
            napi_throw_type_error(env, nullptr, "gsb200: camera.view must hold 12 numbers");
            return false;
        }
        c->view[k] = (float)d;
    }
    c->fx = (float)num(env, obj, "fx", 0.0);
    c->fy = (float)num(env, obj, "fy", c->fx);
    c->width = (int32_t)num(env, obj, "width", 0.0);
    c->height = (int32_t)num(env, obj, "height", 0.0);
    c->cx = (float)num(env, obj, "cx", c->width / 2.0);
    c->cy = (float)num(env, obj, "cy", c->height / 2.0);
    return true;
}

bool cameras_from_js(napi_env env, napi_value arr, std::vector<GsCamera>* out) {
    uint32_t n = 0;
    if (napi_get_array_length(env, arr, &n) != napi_ok) {
        napi_throw_type_error(env, nullptr, "gsb200: expected an array of cameras");
        return false;
    }
    out->resize(n);
    for (uint32_t i = 0; i < n; i++) {
        napi_value e;
        if (napi_get_element(env, arr, i, &e) != napi_ok || !camera_from_js(env, e, &(*out)[i])) return false;
    }
    return true;
}

GsAdamConfig adam_from_js(napi_env env, napi_value obj) {
    GsAdamConfig a;
    gs_adam_default(&a);
    napi_valuetype t = napi_undefined;
    if (obj) napi_typeof(env, obj, &t);
    if (t != napi_object) return a;
    a.lr_color = (float)num(env, obj, "color", a.lr_color);
    a.lr_opacity = (float)num(env, obj, "opacity", a.lr_opacity);
    a.lr_mean = (float)num(env, obj, "mean", a.lr_mean);
    a.lr_scale = (float)num(env, obj, "scale", a.lr_scale);
    a.lr_rotation = (float)num(env, obj, "rotation", a.lr_rotation);
    a.lr_sh = (float)num(env, obj, "sh", a.lr_color / 20.0);
    return a;
}

// A new Float32Array of `count` floats and its data pointer (written by a worker).
napi_value new_f32(napi_env env, size_t count, float** data) {
    napi_value ab = nullptr, arr = nullptr;
    void* p = nullptr;
    if (napi_create_arraybuffer(env, count * sizeof(float), &p, &ab) != napi_ok) return nullptr;
    if (napi_create_typedarray(env, napi_float32_array, count, ab, 0, &arr) != napi_ok) return nullptr;
    *data = static_cast<float*>(p);
    return arr;
}

// ---- asynchronous calls -------------------------------------------------------------------
// One queued call: `run` executes on a pool thread and returns a gs status; `result`
// builds the resolved value on the JS thread.  `keep` holds the JS values the worker
// reads or writes until the call completes.
struct Job {
    napi_async_work work = nullptr;
    napi_deferred deferred = nullptr;
    std::vector<napi_ref> keep;
    std::function<int()> run;
    std::function<napi_value(napi_env)> result;
    int status = GS_OK;
    std::string error;
};

void job_execute(napi_env, void* data) {
    Job* j = static_cast<Job*>(data);
    j->status = j->run();
    if (j->status != GS_OK) j->error = gs_last_error();  // thread-local: read on this thread
}

void job_complete(napi_env env, napi_status st, void* data) {
    Job* j = static_cast<Job*>(data);
    if (st != napi_ok) {
        napi_reject_deferred(env, j->deferred, make_error(env, GS_ERR_STATE, "gsb200: call cancelled"));
    } else if (j->status != GS_OK) {
        napi_reject_deferred(env, j->deferred, make_error(env, j->status, j->error));
    } else {
        napi_value v = nullptr;
        if (j->result) v = j->result(env);
        if (!v) napi_get_undefined(env, &v);
        napi_resolve_deferred(env, j->deferred, v);
    }
    for (napi_ref r : j->keep) napi_delete_reference(env, r);
    napi_delete_async_work(env, j->work);
    delete j;
}

void keep(napi_env env, Job* j, napi_value v) {
    napi_ref r = nullptr;
    if (napi_create_reference(env, v, 1, &r) == napi_ok) j->keep.push_back(r);
}

napi_value queue(napi_env env, Job* j) {
    napi_value promise = nullptr, name = nullptr;
    if (napi_create_promise(env, &j->deferred, &promise) != napi_ok) {
        for (napi_ref r : j->keep) napi_delete_reference(env, r);
        delete j;
        return throw_msg(env, "gsb200: napi_create_promise failed");
    }
    napi_create_string_utf8(env, "gsb200", NAPI_AUTO_LENGTH, &name);
    if (napi_create_async_work(env, nullptr, name, job_execute, job_complete, j, &j->work) != napi_ok ||
        napi_queue_async_work(env, j->work) != napi_ok) {
        napi_reject_deferred(env, j->deferred, make_error(env, GS_ERR_STATE, "gsb200: could not queue the call"));
        for (napi_ref r : j->keep) napi_delete_reference(env, r);
        delete j;
    }
    return promise;
}

// ---- context --------------------------------------------------------------------------------
// create({gpuTiles, shDegree, near, batched, useGraph, device, autotune, tileCull,
//         rasterBatch, rasterPixelsPerThread}) -> context (createRenderer, :704-712)
napi_value Create(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 0)) return nullptr;
    GsConfig cfg;
    gs_config_default(&cfg);
    napi_valuetype t = napi_undefined;
    if (a.argc > 0) napi_typeof(env, a.argv[0], &t);
    if (t == napi_object) {
        napi_value o = a.argv[0];
        cfg.rect_mode = num(env, o, "gpuTiles", 1.0) != 0.0 ? 0 : 1;  // gpuTiles:false -> tileLists rectangle
        cfg.sh_degree = (int32_t)num(env, o, "shDegree", cfg.sh_degree);
        cfg.near_plane = (float)num(env, o, "near", cfg.near_plane);
        cfg.batched = (int32_t)num(env, o, "batched", cfg.batched);
        cfg.use_graph = (int32_t)num(env, o, "useGraph", cfg.use_graph);
        cfg.device = (int32_t)num(env, o, "device", cfg.device);
        cfg.autotune = (int32_t)num(env, o, "autotune", cfg.autotune);
        cfg.tile_cull = (int32_t)num(env, o, "tileCull", cfg.tile_cull);
        cfg.raster_batch = (int32_t)num(env, o, "rasterBatch", cfg.raster_batch);
        cfg.raster_ppt = (int32_t)num(env, o, "rasterPixelsPerThread", cfg.raster_ppt);
        cfg.tile_size = (int32_t)num(env, o, "tileSize", cfg.tile_size);
        cfg.raster_work_tile = (int32_t)num(env, o, "rasterWorkTile", cfg.raster_work_tile);
    }
    GsContext* ctx = nullptr;
    const int rc = gs_create(&cfg, &ctx);
    if (rc != GS_OK) return throw_status(env, rc);
    Handle* h = new Handle{ctx};
    napi_value ext;
    if (napi_create_external(env, h, finalize_handle, nullptr, &ext) != napi_ok) {
        gs_destroy(ctx);
        delete h;
        return throw_msg(env, "gsb200: napi_create_external failed");
    }
    return ext;
}

napi_value Destroy(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 1)) return nullptr;
    void* p = nullptr;
    NAPI_OK(napi_get_value_external(env, a.argv[0], &p));
    Handle* h = static_cast<Handle*>(p);
    if (h && h->ctx) {
        gs_destroy(h->ctx);
        h->ctx = nullptr;
    }
    return nullptr;
}

napi_value ParamStride(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 1)) return nullptr;
    int32_t d = 0;
    NAPI_OK(napi_get_value_int32(env, a.argv[0], &d));
    napi_value v;
    NAPI_OK(napi_create_int32(env, gs_param_stride(d), &v));
    return v;
}

// ---- scene and views (synchronous: host copies) -----------------------------------------------
// setGaussians(ctx, Float32Array records, shDegree)  -- n x paramStride(shDegree) floats
napi_value SetGaussians(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 2)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    void* data = nullptr;
    size_t len = 0;
    if (!get_typed(env, a.argv[1], napi_float32_array, &data, &len)) return nullptr;
    int32_t stride = 0, d = 0;
    if (a.argc > 2 && napi_get_value_int32(env, a.argv[2], &d) == napi_ok) stride = gs_param_stride(d);
    if (stride <= 0) return throw_msg(env, "gsb200: setGaussians needs the SH degree");
    if (len % (size_t)stride) return throw_msg(env, "gsb200: record array length is not a multiple of the stride");
    const int rc = gs_set_gaussians(ctx, (int32_t)(len / (size_t)stride), static_cast<const float*>(data));
    if (rc != GS_OK) return throw_status(env, rc);
    return nullptr;
}

// setGaussiansPacked(ctx, Float32Array packed16)  -- packGaussians layout (:688-694)
napi_value SetGaussiansPacked(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 2)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    void* data = nullptr;
    size_t len = 0;
    if (!get_typed(env, a.argv[1], napi_float32_array, &data, &len)) return nullptr;
    if (len % 16) return throw_msg(env, "gsb200: packed array length is not a multiple of 16");
    const int rc = gs_set_gaussians_packed(ctx, (int32_t)(len / 16), static_cast<const float*>(data));
    if (rc != GS_OK) return throw_status(env, rc);
    return nullptr;
}

napi_value NumGaussians(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 1)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    napi_value v;
    NAPI_OK(napi_create_int32(env, gs_num_gaussians(ctx), &v));
    return v;
}

// getGaussians(ctx, stride) / getGaussiansPacked(ctx) -> Promise<Float32Array>
napi_value GetGaussiansImpl(napi_env env, napi_callback_info info, bool packed) {
    Args a;
    if (!get_args(env, info, a, packed ? 1 : 2)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    int32_t per = 16;
    if (!packed) {
        int32_t d = 0;
        NAPI_OK(napi_get_value_int32(env, a.argv[1], &d));
        per = gs_param_stride(d);
        if (per <= 0) return throw_msg(env, "gsb200: bad SH degree");
    }
    const size_t n = (size_t)gs_num_gaussians(ctx);
    float* out = nullptr;
    napi_value arr = new_f32(env, n * (size_t)per, &out);
    if (!arr) return throw_msg(env, "gsb200: out of memory");
    Job* j = new Job;
    keep(env, j, arr);
    napi_ref ref = j->keep.back();
    j->run = [ctx, out, packed]() { return packed ? gs_get_gaussians_packed(ctx, out) : gs_get_gaussians(ctx, out); };
    j->result = [ref](napi_env e) {
        napi_value v = nullptr;
        napi_get_reference_value(e, ref, &v);
        return v;
    };
    return queue(env, j);
}
napi_value GetGaussians(napi_env env, napi_callback_info info) { return GetGaussiansImpl(env, info, false); }
napi_value GetGaussiansPacked(napi_env env, napi_callback_info info) { return GetGaussiansImpl(env, info, true); }

// setViews(ctx, cameras[])
napi_value SetViews(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 2)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    std::vector<GsCamera> cams;
    if (!cameras_from_js(env, a.argv[1], &cams)) return nullptr;
    const int rc = gs_set_views(ctx, (int32_t)cams.size(), cams.data());
    if (rc != GS_OK) return throw_status(env, rc);
    return nullptr;
}

// setTargetU8(ctx, view, Uint8Array rgb) (dataset.js:74 photo) / setTargetF32(ctx, view, Float32Array)
napi_value SetTargetImpl(napi_env env, napi_callback_info info, bool u8) {
    Args a;
    if (!get_args(env, info, a, 3)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    int32_t view = 0;
    NAPI_OK(napi_get_value_int32(env, a.argv[1], &view));
    void* data = nullptr;
    size_t len = 0;
    if (!get_typed(env, a.argv[2], u8 ? napi_uint8_array : napi_float32_array, &data, &len)) return nullptr;
    const int rc = u8 ? gs_set_target_u8(ctx, view, static_cast<const uint8_t*>(data))
                      : gs_set_target_f32(ctx, view, static_cast<const float*>(data));
    if (rc != GS_OK) return throw_status(env, rc);
    return nullptr;
}
napi_value SetTargetU8(napi_env env, napi_callback_info info) { return SetTargetImpl(env, info, true); }
napi_value SetTargetF32(napi_env env, napi_callback_info info) { return SetTargetImpl(env, info, false); }

// ---- rendering and gradients (asynchronous) -----------------------------------------------------
// render(ctx, cam) -> Promise<Float32Array(W*H*3)>  (render, :815-820, Gaussians already set)
napi_value Render(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 2)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    GsCamera cam;
    if (!camera_from_js(env, a.argv[1], &cam)) return nullptr;
    if (cam.width <= 0 || cam.height <= 0) return throw_msg(env, "gsb200: camera width and height must be positive");
    float* out = nullptr;
    napi_value arr = new_f32(env, (size_t)cam.width * cam.height * 3, &out);
    if (!arr) return throw_msg(env, "gsb200: out of memory");
    Job* j = new Job;
    keep(env, j, arr);
    napi_ref ref = j->keep.back();
    j->run = [ctx, cam, out]() { return gs_render(ctx, &cam, out, nullptr); };
    j->result = [ref](napi_env e) {
        napi_value v = nullptr;
        napi_get_reference_value(e, ref, &v);
        return v;
    };
    return queue(env, j);
}

// gradients(ctx, cam, Float32Array target, ssim) -> Promise<{image, grads(n*16), shape(n*10)}>
// (gradients, :826-839)
napi_value Gradients(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 3)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    GsCamera cam;
    if (!camera_from_js(env, a.argv[1], &cam)) return nullptr;
    void* tgt = nullptr;
    size_t tlen = 0;
    if (!get_typed(env, a.argv[2], napi_float32_array, &tgt, &tlen)) return nullptr;
    const size_t px = (size_t)cam.width * cam.height;
    if (tlen != px * 3) return throw_msg(env, "gsb200: target must hold width * height * 3 floats");
    double ssim = 0.0;
    if (a.argc > 3) napi_get_value_double(env, a.argv[3], &ssim);
    const size_t n = (size_t)gs_num_gaussians(ctx);
    float *img = nullptr, *g16 = nullptr, *s10 = nullptr;
    napi_value ai = new_f32(env, px * 3, &img), ag = new_f32(env, n * 16, &g16), as = new_f32(env, n * 10, &s10);
    if (!ai || !ag || !as) return throw_msg(env, "gsb200: out of memory");
    Job* j = new Job;
    keep(env, j, a.argv[2]);
    keep(env, j, ai);
    keep(env, j, ag);
    keep(env, j, as);
    const napi_ref ri = j->keep[1], rg = j->keep[2], rs = j->keep[3];
    const float* t = static_cast<const float*>(tgt);
    j->run = [ctx, cam, t, ssim, img, g16, s10]() { return gs_gradients(ctx, &cam, t, (float)ssim, img, g16, s10); };
    j->result = [ri, rg, rs](napi_env e) {
        napi_value o = nullptr, v = nullptr;
        napi_create_object(e, &o);
        napi_get_reference_value(e, ri, &v);
        napi_set_named_property(e, o, "image", v);
        napi_get_reference_value(e, rg, &v);
        napi_set_named_property(e, o, "grads", v);
        napi_get_reference_value(e, rs, &v);
        napi_set_named_property(e, o, "shape", v);
        return o;
    };
    return queue(env, j);
}

// lossGradient(ctx, image, target, width, height, lambda, window) -> Promise<Float32Array>
// (lossGradientOf, :962-977; window 0 = the reference's 7x7 box)
napi_value LossGradient(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 6)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    void *img = nullptr, *tgt = nullptr;
    size_t li = 0, lt = 0;
    if (!get_typed(env, a.argv[1], napi_float32_array, &img, &li)) return nullptr;
    if (!get_typed(env, a.argv[2], napi_float32_array, &tgt, &lt)) return nullptr;
    int32_t w = 0, h = 0, window = 0;
    double lambda = 0.0;
    NAPI_OK(napi_get_value_int32(env, a.argv[3], &w));
    NAPI_OK(napi_get_value_int32(env, a.argv[4], &h));
    NAPI_OK(napi_get_value_double(env, a.argv[5], &lambda));
    if (a.argc > 6) napi_get_value_int32(env, a.argv[6], &window);
    if (w <= 0 || h <= 0 || li != (size_t)w * h * 3 || lt != li)
        return throw_msg(env, "gsb200: image and target must hold width * height * 3 floats");
    float* out = nullptr;
    napi_value arr = new_f32(env, li, &out);
    if (!arr) return throw_msg(env, "gsb200: out of memory");
    Job* j = new Job;
    keep(env, j, a.argv[1]);
    keep(env, j, a.argv[2]);
    keep(env, j, arr);
    const napi_ref ro = j->keep[2];
    const float *pi = static_cast<const float*>(img), *pt = static_cast<const float*>(tgt);
    j->run = [ctx, pi, pt, w, h, lambda, window, out]() {
        return gs_loss_gradient(ctx, pi, pt, w, h, (float)lambda, window, out, nullptr);
    };
    j->result = [ro](napi_env e) {
        napi_value v = nullptr;
        napi_get_reference_value(e, ro, &v);
        return v;
    };
    return queue(env, j);
}

// ---- the forward / backward Function pair ---------------------------------------------------------
// forward(ctx, first, count, pixels) -> Promise<Float32Array images>  (all views [first,
// first + count) in one batched launch; the tile lists, final T and last contributor stay
// on the device for backward)
napi_value Forward(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 4)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    int32_t first = 0, count = 0;
    int64_t pixels = 0;
    NAPI_OK(napi_get_value_int32(env, a.argv[1], &first));
    NAPI_OK(napi_get_value_int32(env, a.argv[2], &count));
    NAPI_OK(napi_get_value_int64(env, a.argv[3], &pixels));
    if (pixels <= 0) return throw_msg(env, "gsb200: forward needs the views' pixel count");
    float* out = nullptr;
    napi_value arr = new_f32(env, (size_t)pixels * 3, &out);
    if (!arr) return throw_msg(env, "gsb200: out of memory");
    Job* j = new Job;
    keep(env, j, arr);
    const napi_ref ro = j->keep[0];
    j->run = [ctx, first, count, out]() { return gs_forward(ctx, first, count, out); };
    j->result = [ro](napi_env e) {
        napi_value v = nullptr;
        napi_get_reference_value(e, ro, &v);
        return v;
    };
    return queue(env, j);
}

// loss(ctx, lambda, window) -> Promise<number>: dL/dpixel of the last forward against the
// views' targets, kept on the device for backward(ctx, null)
napi_value Loss(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 3)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    double lambda = 0.0;
    int32_t window = 0;
    NAPI_OK(napi_get_value_double(env, a.argv[1], &lambda));
    NAPI_OK(napi_get_value_int32(env, a.argv[2], &window));
    Job* j = new Job;
    auto loss = std::make_shared<float>(0.f);
    j->run = [ctx, lambda, window, loss]() {
        GsLossConfig lc{(float)lambda, window};
        return gs_loss(ctx, &lc, loss.get());
    };
    j->result = [loss](napi_env e) {
        napi_value v = nullptr;
        napi_create_double(e, *loss, &v);
        return v;
    };
    return queue(env, j);
}

// backward(ctx, Float32Array dL/dimages | null, stride) -> Promise<Float32Array grads
// (n x stride records)>: the reverse replay of the last forward (BACKWARD, :139-202, and
// the projection's chain, SHAPE, :297-328)
napi_value Backward(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 3)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    napi_valuetype t;
    NAPI_OK(napi_typeof(env, a.argv[1], &t));
    const float* dl = nullptr;
    Job* j = new Job;
    if (t != napi_null && t != napi_undefined) {
        void* data = nullptr;
        size_t len = 0;
        if (!get_typed(env, a.argv[1], napi_float32_array, &data, &len)) {
            delete j;
            return nullptr;
        }
        dl = static_cast<const float*>(data);
        keep(env, j, a.argv[1]);
    }
    int32_t d = 0;
    if (napi_get_value_int32(env, a.argv[2], &d) != napi_ok || gs_param_stride(d) <= 0) {
        for (napi_ref r : j->keep) napi_delete_reference(env, r);
        delete j;
        return throw_msg(env, "gsb200: bad SH degree");
    }
    const size_t n = (size_t)gs_num_gaussians(ctx);
    float* out = nullptr;
    napi_value arr = new_f32(env, n * (size_t)gs_param_stride(d), &out);
    if (!arr) {
        for (napi_ref r : j->keep) napi_delete_reference(env, r);
        delete j;
        return throw_msg(env, "gsb200: out of memory");
    }
    keep(env, j, arr);
    const napi_ref ro = j->keep.back();
    j->run = [ctx, dl, out]() {
        int rc = gs_backward(ctx, dl);
        if (rc == GS_OK) rc = gs_get_param_grads(ctx, out);
        return rc;
    };
    j->result = [ro](napi_env e) {
        napi_value v = nullptr;
        napi_get_reference_value(e, ro, &v);
        return v;
    };
    return queue(env, j);
}

// ---- training ----------------------------------------------------------------------------------
// trainStep(ctx, lr, {ssim, window}, first, count, wantLoss) -> Promise<number | undefined>:
// forward, loss, backward and Adam over views [first, first + count) (trainScene's step,
// :915-933, when count = 1).  Without wantLoss the promise resolves once the step is queued.
napi_value TrainStep(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 5)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    const GsAdamConfig ad = adam_from_js(env, a.argv[1]);
    GsLossConfig lc{0.f, 0};
    napi_valuetype t = napi_undefined;
    napi_typeof(env, a.argv[2], &t);
    if (t == napi_object) {
        lc.ssim_lambda = (float)num(env, a.argv[2], "ssim", 0.0);
        lc.window = (int32_t)num(env, a.argv[2], "window", 0.0);
    }
    int32_t first = 0, count = 0;
    NAPI_OK(napi_get_value_int32(env, a.argv[3], &first));
    NAPI_OK(napi_get_value_int32(env, a.argv[4], &count));
    bool want = true;
    if (a.argc > 5) napi_get_value_bool(env, a.argv[5], &want);
    Job* j = new Job;
    auto loss = std::make_shared<float>(NAN);
    j->run = [ctx, ad, lc, first, count, want, loss]() {
        return gs_train_step(ctx, &ad, &lc, first, count, want ? loss.get() : nullptr);
    };
    j->result = [loss, want](napi_env e) {
        napi_value v = nullptr;
        if (want) napi_create_double(e, *loss, &v);
        return v;
    };
    return queue(env, j);
}

// train(ctx, steps, lr) -> Promise<Float32Array losses>  (train, :846-878: L1, one view per
// step in order, targets set with setTargetF32)
napi_value Train(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 2)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    int32_t steps = 0;
    NAPI_OK(napi_get_value_int32(env, a.argv[1], &steps));
    if (steps < 0) return throw_msg(env, "gsb200: steps must be >= 0");
    const GsAdamConfig ad = adam_from_js(env, a.argc > 2 ? a.argv[2] : nullptr);
    float* out = nullptr;
    napi_value arr = new_f32(env, (size_t)steps, &out);
    if (!arr) return throw_msg(env, "gsb200: out of memory");
    Job* j = new Job;
    keep(env, j, arr);
    const napi_ref ro = j->keep[0];
    j->run = [ctx, steps, ad, out]() { return gs_train(ctx, steps, &ad, out); };
    j->result = [ro](napi_env e) {
        napi_value v = nullptr;
        napi_get_reference_value(e, ro, &v);
        return v;
    };
    return queue(env, j);
}

napi_value StepCount(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 1)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    int32_t t = 0;
    const int rc = gs_get_step(ctx, &t);
    if (rc != GS_OK) return throw_status(env, rc);
    napi_value v;
    NAPI_OK(napi_create_int32(env, t, &v));
    return v;
}

// ---- densification (trainScene, :936-946) ---------------------------------------------------------
napi_value SetDensifyStats(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 2)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    bool on = false;
    NAPI_OK(napi_get_value_bool(env, a.argv[1], &on));
    const int rc = gs_set_densify_stats(ctx, on ? 1 : 0);
    if (rc != GS_OK) return throw_status(env, rc);
    return nullptr;
}

// densify(ctx, {gradThreshold, sizeThreshold, minOpacity, maxCount, maxSize, seed})
// -> Promise<new count>  (densify, :575-599, on the device)
napi_value Densify(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 2)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    GsDensifyConfig d;
    gs_densify_config_default(&d);
    napi_value o = a.argv[1];
    d.grad_threshold = num(env, o, "gradThreshold", d.grad_threshold);
    d.size_threshold = num(env, o, "sizeThreshold", d.size_threshold);
    d.min_opacity = num(env, o, "minOpacity", d.min_opacity);
    d.max_size = num(env, o, "maxSize", d.max_size);
    d.max_count = (int32_t)num(env, o, "maxCount", d.max_count);
    d.seed = (uint64_t)num(env, o, "seed", (double)d.seed);
    Job* j = new Job;
    auto count = std::make_shared<int32_t>(0);
    j->run = [ctx, d, count]() { return gs_densify(ctx, &d, count.get()); };
    j->result = [count](napi_env e) {
        napi_value v = nullptr;
        napi_create_int32(e, *count, &v);
        return v;
    };
    return queue(env, j);
}

napi_value ResetOpacity(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 2)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    double m = 0.0;
    NAPI_OK(napi_get_value_double(env, a.argv[1], &m));
    const int rc = gs_reset_opacity(ctx, m);
    if (rc != GS_OK) return throw_status(env, rc);
    return nullptr;
}

// sceneExtent(cameras[]) -> number  (sceneExtent, :564-568)
napi_value SceneExtent(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 1)) return nullptr;
    std::vector<GsCamera> cams;
    if (!cameras_from_js(env, a.argv[0], &cams)) return nullptr;
    float e = 0.f;
    const int rc = gs_scene_extent(cams.data(), (int32_t)cams.size(), &e);
    if (rc != GS_OK) return throw_status(env, rc);
    napi_value v;
    NAPI_OK(napi_create_double(env, e, &v));
    return v;
}

// ---- scene files (fromPly / toPly / toSplat, :983-999, :524-556) ------------------------------------
// loadPly(ctx, Uint8Array bytes) -> Promise<count>
napi_value LoadPly(napi_env env, napi_callback_info info) {
    Args a;
    if (!get_args(env, info, a, 2)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    void* data = nullptr;
    size_t len = 0;
    if (!get_typed(env, a.argv[1], napi_uint8_array, &data, &len)) return nullptr;
    Job* j = new Job;
    keep(env, j, a.argv[1]);
    auto count = std::make_shared<int32_t>(0);
    j->run = [ctx, data, len, count]() { return gs_load_ply(ctx, data, (int64_t)len, count.get()); };
    j->result = [count](napi_env e) {
        napi_value v = nullptr;
        napi_create_int32(e, *count, &v);
        return v;
    };
    return queue(env, j);
}

// savePly(ctx, withSh) / saveSplat(ctx) -> Promise<ArrayBuffer>
napi_value SaveImpl(napi_env env, napi_callback_info info, bool splat) {
    Args a;
    if (!get_args(env, info, a, 1)) return nullptr;
    GsContext* ctx = get_ctx(env, a.argv[0]);
    if (!ctx) return nullptr;
    bool with_sh = false;
    if (!splat && a.argc > 1) napi_get_value_bool(env, a.argv[1], &with_sh);
    Job* j = new Job;
    auto bytes = std::make_shared<std::vector<unsigned char>>();
    j->run = [ctx, splat, with_sh, bytes]() {
        int64_t size = 0;
        int rc = splat ? gs_save_splat(ctx, nullptr, 0, &size) : gs_save_ply(ctx, with_sh ? 1 : 0, nullptr, 0, &size);
        if (rc != GS_OK) return rc;
        bytes->resize((size_t)size);
        return splat ? gs_save_splat(ctx, bytes->data(), size, &size)
                     : gs_save_ply(ctx, with_sh ? 1 : 0, bytes->data(), size, &size);
    };
    j->result = [bytes](napi_env e) {
        napi_value ab = nullptr;
        void* p = nullptr;
        if (napi_create_arraybuffer(e, bytes->size(), &p, &ab) == napi_ok && !bytes->empty())
            memcpy(p, bytes->data(), bytes->size());
        return ab;
    };
    return queue(env, j);
}
napi_value SavePly(napi_env env, napi_callback_info info) { return SaveImpl(env, info, false); }
napi_value SaveSplat(napi_env env, napi_callback_info info) { return SaveImpl(env, info, true); }

napi_value Init(napi_env env, napi_value exports) {
    const struct {
        const char* name;
        napi_callback fn;
    } fns[] = {
        {"create", Create},
        {"destroy", Destroy},
        {"paramStride", ParamStride},
        {"setGaussians", SetGaussians},
        {"setGaussiansPacked", SetGaussiansPacked},
        {"getGaussians", GetGaussians},
        {"getGaussiansPacked", GetGaussiansPacked},
        {"numGaussians", NumGaussians},
        {"setViews", SetViews},
        {"setTargetU8", SetTargetU8},
        {"setTargetF32", SetTargetF32},
        {"render", Render},
        {"gradients", Gradients},
        {"lossGradient", LossGradient},
        {"forward", Forward},
        {"loss", Loss},
        {"backward", Backward},
        {"trainStep", TrainStep},
        {"train", Train},
        {"stepCount", StepCount},
        {"setDensifyStats", SetDensifyStats},
        {"densify", Densify},
        {"resetOpacity", ResetOpacity},
        {"sceneExtent", SceneExtent},
        {"loadPly", LoadPly},
        {"savePly", SavePly},
        {"saveSplat", SaveSplat},
    };
    for (const auto& f : fns) {
        napi_value v;
        if (napi_create_function(env, f.name, NAPI_AUTO_LENGTH, f.fn, nullptr, &v) != napi_ok ||
            napi_set_named_property(env, exports, f.name, v) != napi_ok)
            return nullptr;
    }
    return exports;
}

}  // namespace

NAPI_MODULE(NODE_GYP_MODULE_NAME, Init)
