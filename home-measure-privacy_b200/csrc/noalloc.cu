// Loss gradient that allocates nothing: gs_loss_gradient_noalloc (include/gsb200.h).
//
// Some callers cannot allocate device memory: an engine that owns every byte of the
// GPU through its own pool, or a real-time loop that must not stall on the allocator.  They pass device buffers for the inputs and outputs; the little scratch
// the loss kernel needs besides them -- the images' view descriptors and the per-image
// sums of |x - y| and SSIM -- lives in the file-scope array below, sized for at most
// GS_NOALLOC_MAX_IMAGES images per call.  Every GPU that loads the library holds the
// array until the process exits.
//
// Host code must not use the array's name as a device address: the address is looked up
// once per device with cudaGetSymbolAddress and passed to the kernels.  All calls share
// the array and it keeps the last call's contents, so every call clears what must start
// at zero, and calls that overlap on the GPU (different streams, or different host
// threads on one device) race on it.
#include <atomic>

#include "../../include/gsb200.h"
#include "internal.h"

namespace gs {

struct NoallocScratch {
    ViewDesc views[GS_NOALLOC_MAX_IMAGES];
    double acc[2 * GS_NOALLOC_MAX_IMAGES];
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[GS_NOALLOC_SCRATCH_BYTES];
static_assert(sizeof(NoallocScratch) <= GS_NOALLOC_SCRATCH_BYTES, "scratch array too small");

struct NoallocViews {
    ViewDesc v[GS_NOALLOC_MAX_IMAGES];
};

// Writes the view descriptors (passed by value) and zeroes the loss sums.
__global__ void noalloc_setup_kernel(NoallocScratch* s, NoallocViews views, int count) {
    const int t = threadIdx.x;
    if (t < count) s->views[t] = views.v[t];
    if (t < 2 * GS_NOALLOC_MAX_IMAGES) s->acc[t] = 0.0;
}

// Per-image mean loss (1 - lambda) L1 + lambda (1 - mean SSIM) from the sums.
__global__ void noalloc_loss_kernel(const NoallocScratch* s, int count, float lambda, int window, float* loss) {
    const int i = threadIdx.x;
    if (i >= count) return;
    const int R = window == 0 ? 3 : 5;
    const ViewDesc& vw = s->views[i];
    const double n = (double)vw.width * vw.height * 3.0;
    const int wx = vw.width - 2 * R, wy = vw.height - 2 * R;
    const double windows = (wx > 0 && wy > 0) ? (double)wx * wy * 3.0 : 0.0;
    const double l1 = s->acc[2 * i] / n;
    const double ssim = windows > 0.0 ? s->acc[2 * i + 1] / windows : 1.0;
    loss[i] = (float)((1.0 - lambda) * l1 + (lambda > 0.f ? lambda * (1.0 - ssim) : 0.0));
}

}  // namespace gs

using namespace gs;

// Device address of the array, per device ordinal; looked up on the first call on each
// device.  Threads racing on that first call store the same address.
constexpr int GS_NOALLOC_MAX_DEVICES = 64;
static std::atomic<NoallocScratch*> g_scratch_addr[GS_NOALLOC_MAX_DEVICES];

extern "C" GS_API int gs_loss_gradient_noalloc(const float* image, const float* target, int32_t num_images,
                                               int32_t width, int32_t height, float ssim_lambda, int32_t window,
                                               float* grad, float* loss, void* stream) {
    if (!image || !target || !grad) return GS_ERR_INVALID_ARG;
    if (num_images < 1 || num_images > GS_NOALLOC_MAX_IMAGES) return GS_ERR_CAPACITY;
    if (width < 1 || height < 1 || width > 16384 || height > 16384) return GS_ERR_INVALID_ARG;
    if ((long long)width * height * num_images * 3 > 0x7fffffffLL) return GS_ERR_CAPACITY;
    if (!(ssim_lambda >= 0.f && ssim_lambda <= 1.f) || (window != 0 && window != 1)) return GS_ERR_INVALID_ARG;
    // An error the caller's own work left pending stays the caller's: report it without
    // clearing it, before launching anything.
    if (cudaPeekAtLastError() != cudaSuccess) return GS_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return GS_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= GS_NOALLOC_MAX_DEVICES) return GS_ERR_INVALID_ARG;
    // Once per device, with that device current: the array's device address.
    NoallocScratch* s = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!s) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return GS_ERR_CUDA;
        }
        if (loss_prepare() != cudaSuccess) {
            cudaGetLastError();
            return GS_ERR_CUDA;
        }
        s = reinterpret_cast<NoallocScratch*>(p);
        g_scratch_addr[dev].store(s, std::memory_order_release);
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    NoallocViews views;
    memset(&views, 0, sizeof views);
    int blocks = 0;
    for (int i = 0; i < num_images; i++) {
        ViewDesc& d = views.v[i];
        d.width = width;
        d.height = height;
        d.tiles_x = (width + GS_TILE - 1) / GS_TILE;
        d.tiles_y = (height + GS_TILE - 1) / GS_TILE;
        d.pixel_offset = i * width * height;
        d.loss_blocks_x = (width + loss_block_w() - 1) / loss_block_w();
        d.loss_blocks_y = (height + loss_block_h() - 1) / loss_block_h();
        d.loss_block_offset = blocks;
        blocks += d.loss_blocks_x * d.loss_blocks_y;
    }
    noalloc_setup_kernel<<<1, 2 * GS_NOALLOC_MAX_IMAGES, 0, st>>>(s, views, num_images);
    LossArgs la;
    memset(&la, 0, sizeof la);
    la.views = s->views;
    la.view_first = 0;
    la.num_views = num_images;
    la.block_first = 0;
    la.num_blocks = blocks;
    la.image = image;
    la.target_f32 = target;
    la.dl = grad;
    la.lambda = ssim_lambda;
    la.window = window;
    la.acc = s->acc;
    launch_loss(la, st);
    if (loss) noalloc_loss_kernel<<<1, GS_NOALLOC_MAX_IMAGES, 0, st>>>(s, num_images, ssim_lambda, window, loss);
    if (cudaGetLastError() != cudaSuccess) return GS_ERR_CUDA;
    return GS_OK;
}
