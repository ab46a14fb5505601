// Data-parallel exchange without PyTorch: NCCL, loaded at run time, sums the gradient
// buffer of a step across replicas in place on the context's own stream.
//
// The reference trains on one device (trainer/gpu.js:915-933); spreading a step's views
// over GPUs adds exactly one exchange per step: every rank computes the gradients of
// its own views (gs_step_gradients), the ranks sum the buffer -- parameter gradients,
// densification statistics and the tail holding loss sum, overflow flag and view count
// -- and every rank applies the same Adam update (gs_step_apply).  The sum runs on the
// library's stream, so it orders after the backward and before the update with no host
// wait; NCCL takes NVLink / NVSwitch between GPUs of one node.
//
// NCCL is opened with dlopen when the first communicator is made: a process that already
// holds a libnccl (a framework loaded before this library) shares it, and a process that
// never trains data-parallel never loads it.  Only nccl.h's types and the five entry
// points below are used.
#include <dlfcn.h>
#include <nccl.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "internal.h"

namespace gs {

namespace {

struct NcclApi {
    void* handle = nullptr;
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*all_reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                               cudaStream_t) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;
    char load_error[256] = {0};
};

NcclApi g_nccl;
std::once_flag g_nccl_once;

void load_nccl() {
    const char* names[] = {"libnccl.so.2", "libnccl.so"};
    for (const char* nm : names) {
        // An already loaded NCCL first (RTLD_NOLOAD), then the loader's search path.
        g_nccl.handle = dlopen(nm, RTLD_NOW | RTLD_NOLOAD);
        if (!g_nccl.handle) g_nccl.handle = dlopen(nm, RTLD_NOW | RTLD_LOCAL);
        if (g_nccl.handle) break;
    }
    if (!g_nccl.handle) {
        const char* e = dlerror();
        snprintf(g_nccl.load_error, sizeof g_nccl.load_error, "NCCL not found (%s)", e ? e : "dlopen failed");
        return;
    }
    auto sym = [](const char* name) { return dlsym(g_nccl.handle, name); };
    g_nccl.get_unique_id = reinterpret_cast<decltype(g_nccl.get_unique_id)>(sym("ncclGetUniqueId"));
    g_nccl.comm_init_rank = reinterpret_cast<decltype(g_nccl.comm_init_rank)>(sym("ncclCommInitRank"));
    g_nccl.all_reduce = reinterpret_cast<decltype(g_nccl.all_reduce)>(sym("ncclAllReduce"));
    g_nccl.comm_destroy = reinterpret_cast<decltype(g_nccl.comm_destroy)>(sym("ncclCommDestroy"));
    g_nccl.error_string = reinterpret_cast<decltype(g_nccl.error_string)>(sym("ncclGetErrorString"));
    if (!g_nccl.get_unique_id || !g_nccl.comm_init_rank || !g_nccl.all_reduce || !g_nccl.comm_destroy ||
        !g_nccl.error_string) {
        snprintf(g_nccl.load_error, sizeof g_nccl.load_error, "NCCL library lacks an entry point");
        g_nccl.get_unique_id = nullptr;
    }
}

bool nccl_ready(char* err, size_t n) {
    std::call_once(g_nccl_once, load_nccl);
    if (g_nccl.get_unique_id) return true;
    snprintf(err, n, "%s", g_nccl.load_error);
    return false;
}

void nccl_error(ncclResult_t r, const char* what, char* err, size_t n) {
    snprintf(err, n, "%s: %s", what, g_nccl.error_string ? g_nccl.error_string(r) : "NCCL error");
}

}  // namespace

int dp_unique_id_bytes() { return (int)sizeof(ncclUniqueId); }

bool dp_unique_id(void* out, char* err, size_t n) {
    if (!nccl_ready(err, n)) return false;
    ncclUniqueId id;
    const ncclResult_t r = g_nccl.get_unique_id(&id);
    if (r != ncclSuccess) {
        nccl_error(r, "ncclGetUniqueId", err, n);
        return false;
    }
    memcpy(out, &id, sizeof id);
    return true;
}

void* dp_comm_create(const void* id, int rank, int world, char* err, size_t n) {
    if (!nccl_ready(err, n)) return nullptr;
    ncclUniqueId uid;
    memcpy(&uid, id, sizeof uid);
    ncclComm_t comm = nullptr;
    const ncclResult_t r = g_nccl.comm_init_rank(&comm, world, uid, rank);
    if (r != ncclSuccess) {
        nccl_error(r, "ncclCommInitRank", err, n);
        return nullptr;
    }
    return comm;
}

bool dp_allreduce_sum(void* comm, float* buf, size_t count, cudaStream_t s, char* err, size_t n) {
    const ncclResult_t r =
        g_nccl.all_reduce(buf, buf, count, ncclFloat32, ncclSum, static_cast<ncclComm_t>(comm), s);
    if (r != ncclSuccess) {
        nccl_error(r, "ncclAllReduce", err, n);
        return false;
    }
    return true;
}

void dp_comm_destroy(void* comm) {
    if (comm && g_nccl.comm_destroy) g_nccl.comm_destroy(static_cast<ncclComm_t>(comm));
}

}  // namespace gs
