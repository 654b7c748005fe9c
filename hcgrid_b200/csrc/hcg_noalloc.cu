// Single-channel gridding that allocates nothing (hcg_grid_noalloc).
//
// Who needs it: callers that cannot allocate device memory at the time they
// grid. A real-time pipeline (a telescope backend gridding each scan as it
// lands) reserves its device memory when it starts and must not meet an
// allocation failure, or the device-wide stall of cudaMalloc/cudaFree, in the
// middle of an observation; a host application whose own allocator already
// holds the GPU's memory lends the library only the inputs and outputs.
// hcg_grid takes its per-pixel scratch from the context's pool, which may
// have to grow; this entry point takes it from a fixed array compiled into
// the library instead.
//
// The scratch is the per-pixel setup (ring range and the phi half of the
// window arithmetic, 96 bytes a pixel) in a file-scope __device__ array of
// kNoAllocMaxPixels entries: 131072 pixels, 12 MiB, held by every GPU that
// loads the library until the process exits. Host code may not pass the
// array's name to a kernel (on the host it names a stand-in, not device
// memory), so its device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, on the first call for the
// device; make that first call before any stream capture. Every call shares
// the array and overwrites the entries of its pixels before reading them
// (nothing in it has to start at zero); calls whose work overlaps on the GPU
// (other streams or contexts on the same device) race on it, so issue them
// one after another.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "hcg_internal.h"
#include "hcg_kernels.cuh"

namespace hcg {
namespace {

constexpr uint64_t kNoAllocMaxPixels = 131072;

static __device__ __align__(256) PixPrep g_noalloc_prep[kNoAllocMaxPixels];

__global__ void k_noalloc_prep(HpxParams h, uint64_t firstring, uint64_t usedrings, double disc, uint64_t npix,
                               const double *__restrict__ X, const double *__restrict__ Y, PixPrep *prep,
                               DevStats *stats) {
    uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (p < npix) prep_item(h, firstring, usedrings, disc, X, Y, prep, stats, p);
}

template <bool GEN>  // fields whose kernel is not GAUSS1D
__global__ void __launch_bounds__(256) k_noalloc_grid(GridArgs a, uint64_t npix, const float *__restrict__ data,
                                                      uint32_t cstride, float *__restrict__ out,
                                                      float *__restrict__ wout) {
    uint64_t p = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    if (p < npix) grid1_item<GEN>(a, data, cstride, out, wout, p);
}

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
PixPrep *g_prep_addr[kMaxDevices] = {};

// Device (or managed) memory that kernels on `device` may write.
bool is_device_memory(const void *p, int device) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (at.type == cudaMemoryTypeManaged) return true;
    return at.type == cudaMemoryTypeDevice && at.device == device;
}

}  // namespace
}  // namespace hcg

using namespace hcg;

extern "C" hcg_status hcg_grid_noalloc(hcg_context *ctx, const hcg_field *field, const hcg_target *target,
                                       float *cube, float *weights_out) {
    if (!ctx || !field || !target || !cube) return HCG_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (!field->d_spec || field->nchan != 1) {
        ctx->err = "hcg_grid_noalloc grids single-channel fields that have spectra";
        return field->d_spec ? HCG_EINVAL : HCG_ESTATE;
    }
    const uint64_t P = (uint64_t)target->nx * target->ny;
    if (P > kNoAllocMaxPixels) {
        ctx->err = "hcg_grid_noalloc: target has " + std::to_string(P) + " pixels; its fixed scratch holds at most " +
                   std::to_string(kNoAllocMaxPixels) + " (use hcg_grid)";
        return HCG_EINVAL;
    }
    if (field->ctx->device != ctx->device || target->ctx->device != ctx->device) {
        ctx->err = "hcg_grid_noalloc: field or target lives on another device than the context";
        return HCG_EINVAL;
    }
    if (!is_device_memory(cube, ctx->device) || (weights_out && !is_device_memory(weights_out, ctx->device))) {
        ctx->err = "hcg_grid_noalloc writes device buffers of the context's device only";
        return HCG_EINVAL;
    }
    if (ctx->device < 0 || ctx->device >= kMaxDevices) {
        ctx->err = "hcg_grid_noalloc supports device ordinals below " + std::to_string(kMaxDevices);
        return HCG_EINVAL;
    }
    PixPrep *prep;
    {
        std::lock_guard<std::mutex> g(g_setup_mu);
        if (!g_prep_addr[ctx->device]) {
            // once per device, with that device current
            void *addr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_prep);
            if (e != cudaSuccess || !addr) {
                cudaGetLastError();
                ctx->err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
                return HCG_EDEVICE;
            }
            g_prep_addr[ctx->device] = (PixPrep *)addr;
        }
        prep = g_prep_addr[ctx->device];
    }
    cudaStream_t s = ctx->stream;
    // every counter hcg_get_stats reports starts at zero, as in hcg_grid
    cudaError_t e = cudaMemsetAsync(ctx->d_stats, 0, offsetof(DevStats, invalid_input), s);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(&ctx->d_stats->timeouts, 0, 2 * sizeof(unsigned long long), s);
    if (e == cudaSuccess) {
        cudaEventRecord(ctx->ev0, s);
        k_noalloc_prep<<<(unsigned)((P + 255) / 256), 256, 0, s>>>(field->hpx, field->firstring, field->usedrings,
                                                                    field->disc_size, P, target->d_x, target->d_y,
                                                                    prep, ctx->d_stats);
        e = coarsen_prep(prep, target->nx, P, ctx->factor, s);
        for (auto &ev : ctx->evp) cudaEventRecord(ev, s);
        const GridArgs a = grid_args(field, prep, ctx->d_stats);
        const unsigned nblk = (unsigned)((P * 32 + 255) / 256);
        if (field->kernel_type == HCG_GAUSS1D)
            k_noalloc_grid<false><<<nblk, 256, 0, s>>>(a, P, field->d_spec, field->cstride, cube, weights_out);
        else
            k_noalloc_grid<true><<<nblk, 256, 0, s>>>(a, P, field->d_spec, field->cstride, cube, weights_out);
        cudaEventRecord(ctx->ev1, s);
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        ctx->err = std::string("hcg_grid_noalloc: ") + cudaGetErrorString(e);
        return HCG_EDEVICE;
    }
    return HCG_OK;
}
