// C ABI of the gridder (declared in include/hcgrid_c.h).
//
// Host-side setup mirrors the reference's _prepare_grid_kernel
// (HCGrid/gmap.cpp:64-99) and HEALPix initialisation (HCGrid/healpix.cu:42-65,
// HCGrid/helpers.cu:98-114) with the same expressions, so nside,
// disc_size and the transformed kernel parameter are bit-identical; all
// sample and pixel work runs on the device.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <chrono>
#include <new>
#include <string>
#include <vector>

#include "hcg_internal.h"
#include "hcg_wcs.cuh"

using namespace hcg;

namespace {

struct Guard {
    hcg_context *c;
    std::lock_guard<std::mutex> lk;
    explicit Guard(hcg_context *ctx) : c(ctx), lk(ctx->mu) { cudaSetDevice(ctx->device); }
};

hcg_status fail(hcg_context *ctx, hcg_status s, const std::string &msg) {
    if (ctx) ctx->err = msg;
    return s;
}

hcg_status cuda_fail(hcg_context *ctx, cudaError_t e, const char *where, const std::string &why = "") {
    cudaGetLastError();
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    if (!why.empty()) m += " (" + why + ")";
    if (e == cudaErrorMemoryAllocation) return fail(ctx, HCG_ENOMEM, m);
    if (e == cudaErrorInvalidValue && !why.empty()) return fail(ctx, HCG_EINVAL, m);
    return fail(ctx, HCG_EDEVICE, m);
}

#define CK(ctx, x, where)                                        \
    do {                                                         \
        cudaError_t e_ = (x);                                    \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where); \
    } while (0)

// helpers.cu:40-64
uint64_t ilog2_u64(uint64_t arg) {
    uint64_t r = 0;
    while (arg > 1) { arg >>= 1; ++r; }
    return r;
}

// helpers.cu:98-102 and healpix.cu:52-65, same expressions as the reference.
void healpix_params(double hpx_max_res, HpxParams &h) {
    const double PI = 3.1415926535897932384626433832;
    double target_res = (PI / 180.) * hpx_max_res;
    uint64_t nside = (uint64_t)(sqrt(PI / 3.) / target_res + 0.5);
    nside = 1ULL << (ilog2_u64(nside) + 1);
    h.nside = nside;
    h.order = ilog2_u64(nside);
    uint64_t npface = nside * nside;
    h.ncap = (npface - nside) << 1;
    h.npix = 12 * npface;
    h.fact2 = 4. / h.npix;
    h.fact1 = (nside << 1) * h.fact2;
    double omega = 4. * PI / h.npix;
    h.resolution = sqrt(omega);
}

// Device buffers of a field (caller holds the context lock). The sorted
// geometry is freed with the last field that shares it.
void release_field(hcg_field *f, cudaStream_t s) {
    if (f->d_spec) cudaFreeAsync(f->d_spec, s);
    free_split(f, s);
    if (f->geom_refs && --*f->geom_refs > 0) return;
    void *ps[] = {f->d_keys, f->d_perm, f->d_inv, f->d_l2,    f->d_b2,
                  f->d_cb2,  f->d_w,    f->d_half, f->d_lut, f->d_rings, f->d_ptab};
    for (void *p : ps)
        if (p) cudaFreeAsync(p, s);
    delete f->geom_refs;
}

}  // namespace

void *hcg::Scratch::get(int slot, size_t bytes, cudaStream_t s, cudaError_t &err) {
    if (slot >= (int)ptr.size()) {
        ptr.resize(slot + 1, nullptr);
        size.resize(slot + 1, 0);
    }
    if (bytes == 0) bytes = 16;
    if (size[slot] < bytes) {
        if (ptr[slot]) cudaFreeAsync(ptr[slot], s);
        size_t want = bytes + bytes / 4;
        void *p = nullptr;
        cudaError_t e = dalloc(&p, want, s, pool);
        if (e != cudaSuccess) {
            ptr[slot] = nullptr;
            size[slot] = 0;
            err = e;
            return nullptr;
        }
        ptr[slot] = p;
        size[slot] = want;
    }
    return ptr[slot];
}

void hcg::Scratch::release(cudaStream_t s) {
    for (auto &p : ptr)
        if (p) cudaFreeAsync(p, s);
    ptr.clear();
    size.clear();
}

// An output buffer that kernels on `device` may write: its device memory,
// managed memory, or page-locked host memory mapped into the address space.
// Pageable host memory and another device's memory are refused before any
// launch (a kernel writing there would fault).
static bool writable_on(const void *p, int device) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (at.type == cudaMemoryTypeManaged) return true;
    if (at.type == cudaMemoryTypeHost) return at.devicePointer != nullptr;
    return at.type == cudaMemoryTypeDevice && at.device == device;
}

uint64_t hcg::job_pixels(const hcg_job &job) {
    return job.target ? (uint64_t)job.target->nx * job.target->ny : 0;
}

int hcg::device_sms(int device) {
    int n = 0;
    return cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device) == cudaSuccess ? n : 0;
}

// A job whose channel sums fill the GPU by themselves: at least 2^20 target
// pixels, or a multi-channel job with at least one (tile, 256-channel block)
// item per SM.
bool hcg::job_fills_gpu(const hcg_job &job, int nsm) {
    if (!job.target || !job.field) return false;
    if (job_pixels(job) >= kBatchMaxPixels) return true;
    if (job.field->nchan <= 1) return false;
    const uint64_t tiles = (uint64_t)((job.target->nx + 15) / 16) * ((job.target->ny + 7) / 8);  // 16 x 8-pixel tiles
    return tiles * ((job.field->nchan + 255) / 256) >= (uint64_t)(nsm > 0 ? nsm : 148);
}

// hcg_grid after its argument checks; the caller holds the context lock.
static hcg_status grid_checked(hcg_context *ctx, const hcg_field *field, const hcg_target *target, float *cube,
                               int layout, float *weights_out, int mem, int engine) {
    if (!field->d_spec && !field->xfmt) return fail(ctx, HCG_ESTATE, "field has no spectra (hcg_field_set_spectra)");
    if (layout != HCG_LAYOUT_SAMPLE_MAJOR && layout != HCG_LAYOUT_CHANNEL_MAJOR)
        return fail(ctx, HCG_EINVAL, "unknown layout");
    if (engine < HCG_ENGINE_AUTO || engine > HCG_ENGINE_TC_F16) return fail(ctx, HCG_EINVAL, "unknown engine");
    if (!fp32_weights_fit(field))
        return fail(ctx, HCG_EINVAL,
                    "weights up to " + std::to_string(field->wbound) +
                        " (sample weights times the kernel's bound) exceed the FP32 weights of the multi-channel "
                        "engines");
    if (engine == HCG_ENGINE_AUTO) engine = auto_engine(field);
    const bool tc = engine != HCG_ENGINE_FP32 && field->nchan > 1;
    if (tc && field->xfmt != engine)
        return fail(ctx, HCG_ESTATE, "the tensor-core engine needs hcg_field_split_spectra with the same engine");
    if (tc && field->xnonfinite)
        return fail(ctx, HCG_EINVAL,
                    std::to_string(field->xnonfinite) + " non-finite spectrum values: grid with HCG_ENGINE_FP32");
    if (tc && !tc_weights_fit(field))
        return fail(ctx, HCG_EINVAL,
                    "weights up to " + std::to_string(field->wbound) +
                        " (sample weights times the kernel's bound) exceed the tensor-core range: grid with "
                        "HCG_ENGINE_FP32");
    if (!tc && !field->d_spec)
        return fail(ctx, HCG_ESTATE, "the FP32 spectra were dropped by hcg_field_split_spectra");
    cudaStream_t s = ctx->stream;
    const size_t P = (size_t)target->nx * target->ny;
    const size_t cube_bytes = P * field->nchan * sizeof(float);
    float *dc = cube, *dw = weights_out;
    if (mem == HCG_MEM_HOST) {
        cudaError_t e = cudaSuccess;
        dc = (float *)ctx->scratch.get(16, cube_bytes, s, e);
        if (weights_out) dw = (float *)ctx->scratch.get(17, P * sizeof(float), s, e);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "output buffers");
    }
    CK(ctx, cudaMemsetAsync(ctx->d_stats, 0, offsetof(DevStats, invalid_input), s), "stats reset");
    std::string why;
    cudaError_t e = grid_field(ctx, field, target, dc, layout, dw, engine, why);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "grid", why);
    if (tc || field->nchan > 1) {
        unsigned long long to = 0;
        CK(ctx, cudaMemcpyAsync(&to, &ctx->d_stats->timeouts, sizeof(to), cudaMemcpyDeviceToHost, s), "timeouts");
        CK(ctx, cudaStreamSynchronize(s), "grid");
        if (to)
            return fail(ctx, HCG_ETIMEOUT, std::to_string(to) + (tc ? " tensor-core" : " FP32 staging") +
                                                " pipeline waits ran out");
    }
    if (mem == HCG_MEM_HOST) {
        CK(ctx, cudaMemcpyAsync(cube, dc, cube_bytes, cudaMemcpyDeviceToHost, s), "cube download");
        if (weights_out)
            CK(ctx, cudaMemcpyAsync(weights_out, dw, P * sizeof(float), cudaMemcpyDeviceToHost, s), "weights download");
        CK(ctx, cudaStreamSynchronize(s), "grid");
    }
    return HCG_OK;
}

// One server job on a lane's context (the field carries its kernel
// parameters; lane contexts are not prepared themselves).
hcg_status hcg::grid_job(hcg_context *ctx, const hcg_job &job) {
    if (!ctx || !job.field || !job.target || !job.cube) return HCG_EINVAL;
    Guard g(ctx);
    if (job.field->ctx->device != ctx->device || job.target->ctx->device != ctx->device)
        return fail(ctx, HCG_EINVAL, "job lives on another device");
    if (!writable_on(job.cube, ctx->device) || (job.weights && !writable_on(job.weights, ctx->device)))
        return fail(ctx, HCG_EINVAL, "job outputs are not device memory of the lane's device");
    return grid_checked(ctx, job.field, job.target, job.cube, job.layout, job.weights, HCG_MEM_DEVICE,
                        HCG_ENGINE_AUTO);
}

extern "C" {

const char *hcg_status_string(hcg_status s) {
    switch (s) {
        case HCG_OK: return "ok";
        case HCG_EINVAL: return "invalid argument";
        case HCG_ENOMEM: return "out of memory";
        case HCG_ETIMEOUT: return "device wait timed out";
        case HCG_EDEVICE: return "CUDA error";
        case HCG_EIO: return "I/O error";
        case HCG_EUNSUPPORTED: return "unsupported";
        case HCG_ESTATE: return "call out of order";
    }
    return "unknown status";
}

hcg_status hcg_context_create(int device, void *stream, hcg_context **out) {
    if (!out) return HCG_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return HCG_EDEVICE;
    }
    hcg_context *c = new (std::nothrow) hcg_context();
    if (!c) return HCG_ENOMEM;
    c->device = device;
    cudaSetDevice(device);
    if (stream) {
        c->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return HCG_EDEVICE;
        }
        c->own_stream = true;
    }
    // the context's memory pool: freed buffers stay mapped for the next call
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    uint64_t keep = UINT64_MAX;
    if (cudaMemPoolCreate(&c->pool, &props) != cudaSuccess ||
        cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
        cudaGetLastError();
        if (c->pool) cudaMemPoolDestroy(c->pool);
        c->pool = nullptr;  // the device's default pool then
    }
    c->scratch.pool = c->pool;
    bool up = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) == cudaSuccess;
    for (auto &ev : c->evu) up = up && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess;
    if (!up) {  // host spectra then go up in one copy
        cudaGetLastError();
        if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
        c->copy_stream = nullptr;
    }
    if (cudaMalloc(&c->d_stats, sizeof(DevStats)) != cudaSuccess || cudaMemset(c->d_stats, 0, sizeof(DevStats)) ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaEventCreate(&c->evp[0]) != cudaSuccess || cudaEventCreate(&c->evp[1]) != cudaSuccess ||
        cudaEventCreate(&c->evp[2]) != cudaSuccess || cudaEventCreate(&c->evp[3]) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return HCG_EDEVICE;
    }
    *out = c;
    return HCG_OK;
}

// A context lives until it was destroyed and every field and target made on
// it has been released.
static void ctx_teardown(hcg_context *ctx) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    batch_release(ctx);
    ctx->scratch.release(ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->d_stats);
    cudaEventDestroy(ctx->ev0);
    cudaEventDestroy(ctx->ev1);
    for (auto &ev : ctx->evp) cudaEventDestroy(ev);
    for (auto &ev : ctx->evu)
        if (ev) cudaEventDestroy(ev);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    // every buffer of the pool was freed above or with its field or target
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    delete ctx;
}

static void ctx_release(hcg_context *ctx) {
    if (ctx->refs.fetch_sub(1) == 1) ctx_teardown(ctx);
}

hcg_status hcg_context_destroy(hcg_context *ctx) {
    if (!ctx) return HCG_EINVAL;
    {
        Guard g(ctx);
        if (ctx->closed) return HCG_ESTATE;
        ctx->closed = true;
        cudaStreamSynchronize(ctx->stream);
    }
    ctx_release(ctx);
    return HCG_OK;
}

const char *hcg_last_error(const hcg_context *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

hcg_status hcg_prepare_grid_kernel(hcg_context *ctx, uint32_t kernel_type, double *kernel_params,
                                   double sphere_radius, double hpx_max_res) {
    if (!ctx) return HCG_EINVAL;
    Guard g(ctx);
    if (!kernel_params) return fail(ctx, HCG_EINVAL, "kernel_params is NULL");
    if (!(sphere_radius > 0) || !(hpx_max_res > 0)) return fail(ctx, HCG_EINVAL, "sphere_radius and hpx_max_res must be > 0");
    // gmap.cpp:69-80; HCG_TAPER_FIX is TAPERED_SINC's only flag
    const bool taper_fix = (kernel_type & HCG_TAPER_FIX) != 0;
    kernel_type &= ~HCG_TAPER_FIX;
    if (taper_fix && kernel_type != HCG_TAPERED_SINC) return fail(ctx, HCG_EINVAL, "HCG_TAPER_FIX needs TAPERED_SINC");
    if (kernel_type == HCG_GAUSS1D) {
        kernel_params[0] = 0.5 / pow(kernel_params[0], 2.);
        ctx->bearing = false;
    } else if (kernel_type == HCG_GAUSS2D) {
        ctx->bearing = true;
    } else if (kernel_type == HCG_TAPERED_SINC) {
        ctx->bearing = false;
    } else {
        return fail(ctx, HCG_EINVAL, "unknown kernel type");
    }
    ctx->kernel_type = kernel_type;
    ctx->taper_fix = taper_fix;
    memcpy(ctx->kparams, kernel_params, 3 * sizeof(double));
    // gmap.cpp:89-95: rebuild HEALPix only when the sphere moved by > 3e-5
    if (!ctx->prepared || fabs(ctx->last_r - sphere_radius) > 3e-5 || fabs(ctx->last_res - hpx_max_res) > 3e-5) {
        healpix_params(hpx_max_res, ctx->hpx);
        ctx->last_r = sphere_radius;
        ctx->last_res = hpx_max_res;
    }
    ctx->sphere_radius = sphere_radius;
    const double PI = 3.1415926535897932384626433832;
    ctx->disc_size = ((PI / 180.) * sphere_radius + ctx->hpx.resolution);
    ctx->prepared = true;
    return HCG_OK;
}

hcg_status hcg_get_info(const hcg_context *ctx, const hcg_field *field, hcg_info *out) {
    if (!ctx || !out) return HCG_EINVAL;
    const HpxParams &h = field ? field->hpx : ctx->hpx;
    out->nside = h.nside;
    out->npix = h.npix;
    out->firstring = field ? field->firstring : 0;
    out->usedrings = field ? field->usedrings : 0;
    out->resolution = h.resolution;
    out->disc_size = ctx->disc_size;
    out->kernel_param0 = ctx->kparams[0];
    out->sphere_radius = ctx->sphere_radius;
    return HCG_OK;
}

hcg_status hcg_field_create(hcg_context *ctx, uint64_t n, const double *lon, const double *lat,
                            const double *weights, int mem, hcg_field **out) {
    if (!ctx || !out) return HCG_EINVAL;
    Guard g(ctx);
    *out = nullptr;
    if (!ctx->prepared) return fail(ctx, HCG_ESTATE, "hcg_prepare_grid_kernel must come first");
    if (n == 0 || n >= 0xffffffffULL) return fail(ctx, HCG_EINVAL, "sample count must be in [1, 2^32-2]");
    if (!lon || !lat) return fail(ctx, HCG_EINVAL, "lon/lat are NULL");
    cudaStream_t s = ctx->stream;
    hcg_field *f = new (std::nothrow) hcg_field();
    if (!f) return fail(ctx, HCG_ENOMEM, "host allocation");
    f->ctx = ctx;
    f->n = n;
    f->hpx = ctx->hpx;
    f->sphere_radius = ctx->sphere_radius;
    f->kparam0 = ctx->kparams[0];
    memcpy(f->kparams, ctx->kparams, sizeof f->kparams);
    f->disc_size = ctx->disc_size;
    f->kernel_type = ctx->kernel_type;
    f->taper_fix = ctx->taper_fix;
    f->geom_refs = new (std::nothrow) int(1);
    if (!f->geom_refs) { delete f; return fail(ctx, HCG_ENOMEM, "host allocation"); }
    const double *dl = lon, *db = lat, *dw = weights;
    double *tmp = nullptr;
    if (mem == HCG_MEM_HOST) {
        size_t nb = n * sizeof(double);
        cudaError_t e = dalloc(&tmp, 3 * nb, s, ctx->pool);
        if (e != cudaSuccess) { delete f; return cuda_fail(ctx, e, "field upload"); }
        cudaMemcpyAsync(tmp, lon, nb, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(tmp + n, lat, nb, cudaMemcpyHostToDevice, s);
        if (weights) cudaMemcpyAsync(tmp + 2 * n, weights, nb, cudaMemcpyHostToDevice, s);
        dl = tmp;
        db = tmp + n;
        dw = weights ? tmp + 2 * n : nullptr;
    }
    std::string why;
    cudaError_t e = build_field(ctx, f, dl, db, dw, why);
    if (tmp) cudaFreeAsync(tmp, s);
    // |kernel| <= 1 except for the reference's TAPERED_SINC taper, whose
    // exp(+(pi d / (sigma a))^2) grows to its value at d = sphere_radius
    double kbound = 1.0;
    if (f->kernel_type == HCG_TAPERED_SINC && !f->taper_fix) {
        const double t = 3.1415926535897932384626433832 * f->sphere_radius / (f->kparams[0] * f->kparams[1]);
        kbound = exp(t * t);
    }
    f->wbound = f->wmax * kbound;
    if (e != cudaSuccess) {
        hcg_status st = cuda_fail(ctx, e, "field build", why);
        cudaStreamSynchronize(s);
        release_field(f, s);  // the context lock is already held here
        delete f;
        return st;
    }
    ctx->refs.fetch_add(1);
    *out = f;
    return HCG_OK;
}

hcg_status hcg_field_set_spectra(hcg_field *field, uint32_t nchan, const float *values, int layout, int mem) {
    if (!field) return HCG_EINVAL;
    hcg_context *ctx = field->ctx;
    Guard g(ctx);
    if (nchan == 0 || !values) return fail(ctx, HCG_EINVAL, "need nchan >= 1 and values");
    if (layout != HCG_LAYOUT_SAMPLE_MAJOR && layout != HCG_LAYOUT_CHANNEL_MAJOR)
        return fail(ctx, HCG_EINVAL, "unknown layout");
    cudaStream_t s = ctx->stream;
    const float *dv = values;
    float *tmp = nullptr;
    if (mem == HCG_MEM_HOST && ctx->copy_stream && field->n * (uint64_t)nchan * 4 > 2 * kUploadChunk) {
        // large host spectra: chunked copies overlapped with the scatter into sorted order
        free_split(field, s);
        cudaError_t e = upload_spectra(ctx, field, values, nchan, layout);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "spectra upload");
        return HCG_OK;
    }
    if (mem == HCG_MEM_HOST) {
        size_t nb = field->n * (size_t)nchan * sizeof(float);
        cudaError_t e = dalloc(&tmp, nb, s, ctx->pool);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "spectra upload");
        CK(ctx, cudaMemcpyAsync(tmp, values, nb, cudaMemcpyHostToDevice, s), "spectra upload");
        dv = tmp;
    }
    free_split(field, s);  // the split, if any, described the previous spectra
    cudaError_t e = permute_spectra(ctx, field, dv, nchan, layout);
    if (tmp) cudaFreeAsync(tmp, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "spectra permute");
    return HCG_OK;
}

hcg_status hcg_field_split_spectra(hcg_field *field, int engine, int keep_fp32) {
    if (!field) return HCG_EINVAL;
    hcg_context *ctx = field->ctx;
    Guard g(ctx);
    if (engine != HCG_ENGINE_TC_BF16 && engine != HCG_ENGINE_TC_F16)
        return fail(ctx, HCG_EINVAL, "split engine must be HCG_ENGINE_TC_BF16 or HCG_ENGINE_TC_F16");
    if (!field->d_spec) return fail(ctx, HCG_ESTATE, "field has no FP32 spectra (hcg_field_set_spectra)");
    std::string why;
    cudaError_t e = split_spectra(ctx, field, engine, why);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "spectra split", why);
    if (!keep_fp32) {
        cudaFreeAsync(field->d_spec, ctx->stream);
        field->d_spec = nullptr;
    }
    return HCG_OK;
}

hcg_status hcg_field_sorted(const hcg_field *field, uint64_t *keys, uint32_t *perm, uint32_t *lut) {
    if (!field) return HCG_EINVAL;
    hcg_context *ctx = field->ctx;
    Guard g(ctx);
    cudaStream_t s = ctx->stream;
    if (keys) CK(ctx, cudaMemcpyAsync(keys, field->d_keys, (field->n + 1) * 8, cudaMemcpyDeviceToHost, s), "keys");
    if (perm) CK(ctx, cudaMemcpyAsync(perm, field->d_perm, field->n * 4, cudaMemcpyDeviceToHost, s), "perm");
    if (lut) CK(ctx, cudaMemcpyAsync(lut, field->d_lut, (field->usedrings + 1) * 4, cudaMemcpyDeviceToHost, s), "lut");
    CK(ctx, cudaStreamSynchronize(s), "sorted readback");
    return HCG_OK;
}

hcg_status hcg_field_share(const hcg_field *src, hcg_field **out) {
    if (!src || !out) return HCG_EINVAL;
    hcg_context *ctx = src->ctx;
    Guard g(ctx);
    hcg_field *f = new (std::nothrow) hcg_field(*src);
    if (!f) return fail(ctx, HCG_ENOMEM, "host allocation");
    f->d_spec = nullptr;
    f->nchan = f->cstride = 0;
    f->d_xhi = f->d_xlo = nullptr;
    f->d_xinv = nullptr;
    f->xcpad = 0;
    f->xfmt = 0;
    f->xnonfinite = 0;
    ++*f->geom_refs;
    ctx->refs.fetch_add(1);
    *out = f;
    return HCG_OK;
}

hcg_status hcg_field_destroy(hcg_field *f) {
    if (!f) return HCG_EINVAL;
    hcg_context *ctx = f->ctx;
    {
        Guard g(ctx);
        release_field(f, ctx->stream);
    }
    delete f;
    ctx_release(ctx);
    return HCG_OK;
}

static hcg_status make_target(hcg_context *ctx, uint32_t nx, uint32_t ny, const double *x, const double *y,
                              cudaMemcpyKind kind, hcg_target **out) {
    cudaStream_t s = ctx->stream;
    hcg_target *t = new (std::nothrow) hcg_target();
    if (!t) return fail(ctx, HCG_ENOMEM, "host allocation");
    t->ctx = ctx;
    t->nx = nx;
    t->ny = ny;
    size_t nb = (size_t)nx * ny * sizeof(double);
    cudaError_t e = dalloc(&t->d_x, nb, s, ctx->pool);
    if (e == cudaSuccess) e = dalloc(&t->d_y, nb, s, ctx->pool);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t->d_x, x, nb, kind, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t->d_y, y, nb, kind, s);
    if (e == cudaSuccess && kind == cudaMemcpyHostToDevice) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        if (t->d_x) cudaFreeAsync(t->d_x, s);
        if (t->d_y) cudaFreeAsync(t->d_y, s);
        delete t;
        return cuda_fail(ctx, e, "target upload");
    }
    ctx->refs.fetch_add(1);
    *out = t;
    return HCG_OK;
}

hcg_status hcg_target_create(hcg_context *ctx, uint32_t nx, uint32_t ny, const double *xwcs, const double *ywcs,
                             int mem, hcg_target **out) {
    if (!ctx || !out) return HCG_EINVAL;
    Guard g(ctx);
    *out = nullptr;
    if (nx == 0 || ny == 0 || !xwcs || !ywcs) return fail(ctx, HCG_EINVAL, "empty target");
    return make_target(ctx, nx, ny, xwcs, ywcs,
                       mem == HCG_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, out);
}

hcg_status hcg_target_from_header(hcg_context *ctx, const char *header, size_t len, hcg_target **out) {
    if (!ctx || !out || !header) return HCG_EINVAL;
    Guard g(ctx);
    *out = nullptr;
    uint32_t nx, ny;
    SinWcs w;
    std::string why;
    int st = parse_sin_header(header, len, nx, ny, w, why);
    if (st != HCG_OK) return fail(ctx, (hcg_status)st, why);
    if (nx == 0 || ny == 0) return fail(ctx, HCG_EINVAL, "empty target");
    cudaStream_t s = ctx->stream;
    hcg_target *t = new (std::nothrow) hcg_target();
    if (!t) return fail(ctx, HCG_ENOMEM, "host allocation");
    t->ctx = ctx;
    t->nx = nx;
    t->ny = ny;
    size_t nb = (size_t)nx * ny * sizeof(double);
    cudaError_t e = dalloc(&t->d_x, nb, s, ctx->pool);
    if (e == cudaSuccess) e = dalloc(&t->d_y, nb, s, ctx->pool);
    if (e == cudaSuccess) e = sin_coords_device(w, nx, ny, t->d_x, t->d_y, s);  // pixel centres on the device
    if (e != cudaSuccess) {
        if (t->d_x) cudaFreeAsync(t->d_x, s);
        if (t->d_y) cudaFreeAsync(t->d_y, s);
        delete t;
        return cuda_fail(ctx, e, "target");
    }
    ctx->refs.fetch_add(1);
    *out = t;
    return HCG_OK;
}

hcg_status hcg_target_coords(const hcg_target *t, uint32_t *nx, uint32_t *ny, double *xwcs, double *ywcs) {
    if (!t) return HCG_EINVAL;
    hcg_context *ctx = t->ctx;
    Guard g(ctx);
    if (nx) *nx = t->nx;
    if (ny) *ny = t->ny;
    size_t nb = (size_t)t->nx * t->ny * sizeof(double);
    if (xwcs) CK(ctx, cudaMemcpyAsync(xwcs, t->d_x, nb, cudaMemcpyDeviceToHost, ctx->stream), "coords");
    if (ywcs) CK(ctx, cudaMemcpyAsync(ywcs, t->d_y, nb, cudaMemcpyDeviceToHost, ctx->stream), "coords");
    CK(ctx, cudaStreamSynchronize(ctx->stream), "coords");
    return HCG_OK;
}

hcg_status hcg_header_coords(const char *header, size_t len, uint32_t *nx, uint32_t *ny, double *xwcs,
                             double *ywcs) {
    if (!header || !nx || !ny) return HCG_EINVAL;
    uint32_t w, h;
    std::vector<double> x, y;
    std::string why;
    int st = sin_target_coords(header, len, w, h, x, y, why);
    if (st != HCG_OK) return (hcg_status)st;
    *nx = w;
    *ny = h;
    if (xwcs) memcpy(xwcs, x.data(), x.size() * sizeof(double));
    if (ywcs) memcpy(ywcs, y.data(), y.size() * sizeof(double));
    return HCG_OK;
}

hcg_status hcg_target_destroy(hcg_target *t) {
    if (!t) return HCG_EINVAL;
    hcg_context *ctx = t->ctx;
    {
        Guard g(ctx);
        if (t->d_x) cudaFreeAsync(t->d_x, ctx->stream);
        if (t->d_y) cudaFreeAsync(t->d_y, ctx->stream);
    }
    delete t;
    ctx_release(ctx);
    return HCG_OK;
}

hcg_status hcg_grid(hcg_context *ctx, const hcg_field *field, const hcg_target *target, float *cube, int layout,
                    float *weights_out, int mem, int engine) {
    if (!ctx || !field || !target || !cube) return HCG_EINVAL;
    Guard g(ctx);
    if (!ctx->prepared) return fail(ctx, HCG_ESTATE, "hcg_prepare_grid_kernel must come first");
    if (field->ctx->device != ctx->device || target->ctx->device != ctx->device)
        return fail(ctx, HCG_EINVAL, "field or target lives on another device than the context");
    if (mem == HCG_MEM_DEVICE && (!writable_on(cube, ctx->device) || (weights_out && !writable_on(weights_out, ctx->device))))
        return fail(ctx, HCG_EINVAL, "HCG_MEM_DEVICE outputs must be device memory of the context's device "
                                     "(or managed or mapped host memory)");
    return grid_checked(ctx, field, target, cube, layout, weights_out, mem, engine);
}

hcg_status hcg_grid_planes(hcg_context *ctx, const hcg_field *geometry, const hcg_target *target,
                           const float *planes, uint32_t nchan, float *cube, int layout, float *weights_out,
                           int engine, uint32_t block) {
    if (!ctx || !geometry || !target || !planes || !cube || nchan == 0) return HCG_EINVAL;
    Guard g(ctx);
    if (!ctx->prepared) return fail(ctx, HCG_ESTATE, "hcg_prepare_grid_kernel must come first");
    if (geometry->ctx->device != ctx->device || target->ctx->device != ctx->device)
        return fail(ctx, HCG_EINVAL, "field or target lives on another device than the context");
    if (layout != HCG_LAYOUT_SAMPLE_MAJOR && layout != HCG_LAYOUT_CHANNEL_MAJOR)
        return fail(ctx, HCG_EINVAL, "unknown layout");
    if (block == 0) block = kPlaneBlock;
    if (block % 64) return fail(ctx, HCG_EINVAL, "block must be a multiple of 64 channels");
    if (engine == HCG_ENGINE_AUTO) engine = nchan > 1 ? HCG_ENGINE_TC_F16 : HCG_ENGINE_FP32;
    if (engine < HCG_ENGINE_FP32 || engine > HCG_ENGINE_TC_F16) return fail(ctx, HCG_EINVAL, "unknown engine");
    cudaStream_t s = ctx->stream, cs = ctx->copy_stream, us = nullptr, dl = nullptr;
    if (!cs) return fail(ctx, HCG_EDEVICE, "the context has no copy stream");
    const uint64_t n = geometry->n;
    const size_t P = (size_t)target->nx * target->ny;
    const uint32_t nblk = (nchan + block - 1) / block;
    // events: chunk copied (2), staging buffer free (2), block uploaded (2),
    // block cube downloaded (2), block gridded, buffers ready
    cudaEvent_t ev[10] = {};
    cudaEvent_t *ev_copied = ev, *ev_free = ev + 2, *ev_up = ev + 4, *ev_dl = ev + 6;
    cudaEvent_t &ev_grid = ev[8], &ev_ready = ev[9];
    hcg_field *fb[2] = {nullptr, nullptr};
    uint64_t chunks = 0;
    const char *where = "plane pipeline";
    cudaError_t e = cudaSuccess;
    auto run = [&]() -> hcg_status {
        // earlier uploads on the copy stream have ended before its staging buffers are reused
        if ((e = cudaStreamSynchronize(cs)) != cudaSuccess) return cuda_fail(ctx, e, where);
        if ((e = cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&dl, cudaStreamNonBlocking)) != cudaSuccess)
            return cuda_fail(ctx, e, where);
        for (auto &x : ev)
            if ((e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming)) != cudaSuccess)
                return cuda_fail(ctx, e, where);
        // staging (two chunks of whole planes), two block cubes, the weights
        const uint64_t per = std::max<uint64_t>(1, kUploadChunk / std::max<uint64_t>(1, n * 4));
        const uint64_t stage_bytes = std::min<uint64_t>(per, block) * n * 4;
        float *stage[2], *dcube[2], *dw = nullptr;
        for (int b = 0; b < 2; ++b) {
            stage[b] = (float *)ctx->scratch.get(19 + b, stage_bytes, s, e);
            dcube[b] = (float *)ctx->scratch.get(22 + b, (size_t)std::min(block, nchan) * P * sizeof(float), s, e);
        }
        if (weights_out) dw = (float *)ctx->scratch.get(24, P * sizeof(float), s, e);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "plane pipeline buffers");
        if ((e = cudaEventRecord(ev_ready, s)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(cs, ev_ready, 0)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(us, ev_ready, 0)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(dl, ev_ready, 0)) != cudaSuccess)
            return cuda_fail(ctx, e, where);
        for (int b = 0; b < 2 && b < (int)nblk; ++b) {
            fb[b] = new (std::nothrow) hcg_field(*geometry);
            if (!fb[b]) return fail(ctx, HCG_ENOMEM, "host allocation");
            fb[b]->d_spec = nullptr;
            fb[b]->nchan = fb[b]->cstride = 0;
            fb[b]->d_xhi = fb[b]->d_xlo = nullptr;
            fb[b]->d_xinv = nullptr;
            fb[b]->xcpad = 0;
            fb[b]->xfmt = 0;
            fb[b]->xnonfinite = 0;
            ++*fb[b]->geom_refs;
        }
        auto upload = [&](uint32_t b) -> cudaError_t {
            const uint32_t c0 = b * block, nb = std::min(block, nchan - c0);
            cudaError_t u = upload_plane_block(ctx, fb[b & 1], planes + (size_t)c0 * n, nb, cs, us, stage, stage_bytes,
                                               ev_copied, ev_free, chunks);
            return u != cudaSuccess ? u : cudaEventRecord(ev_up[b & 1], us);
        };
        if ((e = upload(0)) != cudaSuccess) return cuda_fail(ctx, e, "spectra upload");
        for (uint32_t b = 0; b < nblk; ++b) {
            // the next block's copies go out before this block's gridding holds the host
            if (b + 1 < nblk && (e = upload(b + 1)) != cudaSuccess) return cuda_fail(ctx, e, "spectra upload");
            const uint32_t c0 = b * block, nb = std::min(block, nchan - c0);
            hcg_field *f = fb[b & 1];
            const bool tc = engine != HCG_ENGINE_FP32 && nb > 1;
            if ((e = cudaStreamWaitEvent(s, ev_up[b & 1], 0)) != cudaSuccess) return cuda_fail(ctx, e, where);
            if (tc) {
                std::string why;
                if ((e = split_spectra(ctx, f, engine, why)) != cudaSuccess) return cuda_fail(ctx, e, "spectra split", why);
                cudaFreeAsync(f->d_spec, s);
                f->d_spec = nullptr;
            }
            if (b >= 2 && (e = cudaStreamWaitEvent(s, ev_dl[b & 1], 0)) != cudaSuccess) return cuda_fail(ctx, e, where);
            hcg_status st = grid_checked(ctx, f, target, dcube[b & 1], layout, b == 0 ? dw : nullptr, HCG_MEM_DEVICE,
                                         tc ? engine : HCG_ENGINE_FP32);
            if (st != HCG_OK) return st;
            free_split(f, s);
            if (f->d_spec) cudaFreeAsync(f->d_spec, s);
            f->d_spec = nullptr;
            if ((e = cudaEventRecord(ev_grid, s)) != cudaSuccess ||
                (e = cudaStreamWaitEvent(dl, ev_grid, 0)) != cudaSuccess)
                return cuda_fail(ctx, e, where);
            if (layout == HCG_LAYOUT_CHANNEL_MAJOR)
                e = cudaMemcpyAsync(cube + (size_t)c0 * P, dcube[b & 1], (size_t)nb * P * sizeof(float),
                                    cudaMemcpyDeviceToHost, dl);
            else
                e = cudaMemcpy2DAsync(cube + c0, (size_t)nchan * sizeof(float), dcube[b & 1], (size_t)nb * sizeof(float),
                                      (size_t)nb * sizeof(float), P, cudaMemcpyDeviceToHost, dl);
            if (e == cudaSuccess && b == 0 && weights_out)
                e = cudaMemcpyAsync(weights_out, dw, P * sizeof(float), cudaMemcpyDeviceToHost, dl);
            if (e != cudaSuccess || (e = cudaEventRecord(ev_dl[b & 1], dl)) != cudaSuccess)
                return cuda_fail(ctx, e, "cube download");
        }
        if ((e = cudaStreamSynchronize(dl)) != cudaSuccess) return cuda_fail(ctx, e, "cube download");
        return HCG_OK;
    };
    hcg_status st = run();
    // wind down: nothing queued outlives the buffers and fields below
    cudaStreamSynchronize(cs);
    if (us) cudaStreamSynchronize(us);
    if (dl) cudaStreamSynchronize(dl);
    cudaStreamSynchronize(s);
    for (auto &f : fb)
        if (f) {
            release_field(f, s);
            delete f;
        }
    for (auto &x : ev)
        if (x) cudaEventDestroy(x);
    if (us) cudaStreamDestroy(us);
    if (dl) cudaStreamDestroy(dl);
    return st;
}

hcg_status hcg_tc_set_config(hcg_context *ctx, int channel_class, int config) {
    if (!ctx) return HCG_EINVAL;
    Guard g(ctx);
    if (config < -1 || config >= kTcConfigCount || channel_class < -1 || channel_class >= kTcClasses)
        return fail(ctx, HCG_EINVAL, "unknown tensor-core pipeline shape or channel class");
    for (int c = 0; c < kTcClasses; ++c)
        if (channel_class < 0 || c == channel_class) ctx->tc_config[c] = config;
    return HCG_OK;
}

hcg_status hcg_tc_set_weights(hcg_context *ctx, int mode) {
    if (!ctx) return HCG_EINVAL;
    Guard g(ctx);
    if (mode < HCG_TC_WEIGHTS_AUTO || mode > HCG_TC_WEIGHTS_DIRECT)
        return fail(ctx, HCG_EINVAL, "unknown tensor-core weight mode");
    ctx->tc_weights = mode;
    return HCG_OK;
}

hcg_status hcg_tc_set_pipeline(hcg_context *ctx, int channel_class, int prefetch, int strip) {
    if (!ctx) return HCG_EINVAL;
    Guard g(ctx);
    if (channel_class < -1 || channel_class >= kTcClasses || prefetch < -1 || prefetch > 64 || strip < -1 ||
        strip > 4096)
        return fail(ctx, HCG_EINVAL, "prefetch must be -1..64 chunks and strip -1..4096 tiles");
    for (int c = 0; c < kTcClasses; ++c)
        if (channel_class < 0 || c == channel_class) {
            ctx->tc_pf[c] = prefetch;
            ctx->tc_strip[c] = strip;
        }
    return HCG_OK;
}

// Best and worst of `reps` timed gridding runs (after one warm-up) with the
// context's current settings.
static hcg_status tune_time(hcg_context *ctx, const hcg_field *field, const hcg_target *target, int reps, float *cube,
                            float *wts, float &best, float &worst) {
    best = 3.4e38f;
    worst = 0.f;
    for (int r = 0; r < reps + 1; ++r) {
        hcg_status st = hcg_grid(ctx, field, target, cube, ctx->tune_layout, wts, HCG_MEM_DEVICE, field->xfmt);
        if (st != HCG_OK) return st;
        Guard g(ctx);
        CK(ctx, cudaStreamSynchronize(ctx->stream), "autotune");
        float m = 0.f;
        if (cudaEventElapsedTime(&m, ctx->ev0, ctx->ev1) != cudaSuccess) cudaGetLastError();
        if (r > 0) {
            best = m < best ? m : best;
            worst = m > worst ? m : worst;
        }
    }
    return HCG_OK;
}

hcg_status hcg_autotune_layout(hcg_context *ctx, int layout) {
    if (!ctx) return HCG_EINVAL;
    Guard g(ctx);
    if (layout != HCG_LAYOUT_SAMPLE_MAJOR && layout != HCG_LAYOUT_CHANNEL_MAJOR)
        return fail(ctx, HCG_EINVAL, "unknown layout");
    ctx->tune_layout = layout;
    return HCG_OK;
}

hcg_status hcg_autotune_ex(hcg_context *ctx, const hcg_field *field, const hcg_target *target, int reps,
                           hcg_tuning *out) {
    if (!ctx || !field || !target || reps < 1) return HCG_EINVAL;
    int cls;
    {
        Guard g(ctx);
        if (!field->xfmt || field->nchan < 2)
            return fail(ctx, HCG_ESTATE, "autotune needs a multi-channel field with split spectra");
        cls = tc_class_of(field->xcpad);
    }
    const size_t P = (size_t)target->nx * target->ny;
    float *cube = nullptr, *wts = nullptr;
    {
        Guard g(ctx);
        cudaError_t e = cudaSuccess;
        cube = (float *)ctx->scratch.get(16, P * field->nchan * sizeof(float), ctx->stream, e);
        wts = (float *)ctx->scratch.get(17, P * sizeof(float), ctx->stream, e);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "autotune buffers");
    }
    hcg_tuning t = {};
    const int pfs[5] = HCG_TUNE_PREFETCH, strips[5] = HCG_TUNE_STRIP;
    auto set = [&](int shape, int pf, int strip) {
        Guard g(ctx);
        ctx->tc_config[cls] = shape;
        ctx->tc_pf[cls] = pf;
        ctx->tc_strip[cls] = strip;
    };
    float best, worst, spread = 0.f;
    hcg_status st;
    t.shape = 0;
    for (int c = 0; c < kTcConfigCount; ++c) {  // shapes, with the default depth and walk
        set(c, -1, -1);
        if ((st = tune_time(ctx, field, target, reps, cube, wts, best, worst)) != HCG_OK) return st;
        t.ms_shape[c] = best;
        if (best < t.ms_shape[t.shape]) t.shape = c;
    }
    t.prefetch = -1;
    float cur = t.ms_shape[t.shape];
    for (int i = 0; i < 5; ++i) {  // prefetch distance with the best shape
        set(t.shape, pfs[i], -1);
        if ((st = tune_time(ctx, field, target, reps, cube, wts, best, worst)) != HCG_OK) return st;
        t.ms_prefetch[i] = best;
        if (best < cur) {
            cur = best;
            t.prefetch = pfs[i];
        }
    }
    t.strip = -1;
    for (int i = 0; i < 5; ++i) {  // tile walk with the best shape and prefetch
        set(t.shape, t.prefetch, strips[i]);
        if ((st = tune_time(ctx, field, target, reps, cube, wts, best, worst)) != HCG_OK) return st;
        t.ms_strip[i] = best;
        if (best < cur) {
            cur = best;
            t.strip = strips[i];
        }
    }
    set(t.shape, t.prefetch, t.strip);
    if ((st = tune_time(ctx, field, target, reps, cube, wts, best, worst)) != HCG_OK) return st;
    spread = best > 0.f ? (worst - best) / best : 0.f;
    t.ms_best = best;
    t.spread = spread;
    if (t.prefetch < 0) t.prefetch = kTcDefaultPrefetch;
    if (t.strip < 0) t.strip = kTcDefaultStrip;
    if (out) *out = t;
    return HCG_OK;
}

hcg_status hcg_autotune(hcg_context *ctx, const hcg_field *field, const hcg_target *target, int reps, int *best,
                        float *ms) {
    hcg_tuning t;
    hcg_status st = hcg_autotune_ex(ctx, field, target, reps, &t);
    if (st != HCG_OK) return st;
    if (best) *best = t.shape;
    if (ms)
        for (int c = 0; c < kTcConfigCount; ++c) ms[c] = t.ms_shape[c];
    return HCG_OK;
}

hcg_status hcg_batch_set_shape(hcg_context *ctx, int channel_class, int shape) {
    if (!ctx) return HCG_EINVAL;
    Guard g(ctx);
    if (channel_class < -1 || channel_class >= kTcClasses || shape < -1 || shape >= kKbShapes)
        return fail(ctx, HCG_EINVAL, "channel class must be -1..7 and shape -1..3");
    for (int c = 0; c < kTcClasses; ++c)
        if (channel_class < 0 || c == channel_class) ctx->kb_shape[c] = shape;
    return HCG_OK;
}

hcg_status hcg_autotune_batch(hcg_context *ctx, uint32_t njobs, const hcg_job *jobs, int reps, uint32_t max_out,
                              hcg_batch_tuning *out, uint32_t *nout) {
    if (!ctx || !jobs || njobs == 0 || reps < 1 || (max_out && !out)) return HCG_EINVAL;
    // the jobs the batch pass takes on the tensor cores, by channel class
    std::vector<std::vector<hcg_job>> by(kTcClasses);
    {
        Guard g(ctx);
        for (uint32_t i = 0; i < njobs; ++i) {
            const hcg_job &j = jobs[i];
            if (!j.field || !j.target || !j.cube) return fail(ctx, HCG_EINVAL, "job " + std::to_string(i) + " incomplete");
            if (auto_engine(j.field) == HCG_ENGINE_FP32 || j.field->kernel_type != HCG_GAUSS1D ||
                job_pixels(j) >= kBatchMaxPixels)
                continue;
            by[tc_class_of(j.field->xcpad)].push_back(j);
        }
    }
    uint32_t n = 0;
    for (int cls = 0; cls < kTcClasses; ++cls) {
        if (by[cls].empty()) continue;
        hcg_batch_tuning t = {};
        t.channel_class = cls;
        t.jobs = (uint32_t)by[cls].size();
        t.shape = kKbDefaultShape;
        for (int sh = 0; sh < kKbShapes; ++sh) {
            {
                Guard g(ctx);
                ctx->kb_shape[cls] = sh;
            }
            float best = 3.4e38f, worst = 0.f;
            for (int r = 0; r < reps + 1; ++r) {  // run 0 warms up
                const auto t0 = std::chrono::steady_clock::now();
                hcg_status st = hcg_grid_batch(ctx, t.jobs, by[cls].data());
                if (st != HCG_OK) return st;
                const float ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
                if (r > 0) {
                    best = ms < best ? ms : best;
                    worst = ms > worst ? ms : worst;
                }
            }
            t.ms[sh] = best;
            if (sh == 0 || best < t.ms[t.shape]) {
                t.shape = sh;
                t.spread = best > 0.f ? (worst - best) / best : 0.f;
            }
        }
        {
            Guard g(ctx);
            ctx->kb_shape[cls] = t.shape;
        }
        if (n < max_out) out[n] = t;
        ++n;
    }
    if (nout) *nout = n < max_out ? n : max_out;
    return HCG_OK;
}

hcg_status hcg_grid_batch(hcg_context *ctx, uint32_t njobs, const hcg_job *jobs) {
    if (!ctx || (njobs && !jobs)) return HCG_EINVAL;
    Guard g(ctx);
    if (njobs == 0) return HCG_OK;
    for (uint32_t i = 0; i < njobs; ++i) {
        const hcg_job &j = jobs[i];
        if (!j.field || !j.target || !j.cube) return fail(ctx, HCG_EINVAL, "job " + std::to_string(i) + " incomplete");
        if (j.field->ctx->device != ctx->device || j.target->ctx->device != ctx->device)
            return fail(ctx, HCG_EINVAL, "job " + std::to_string(i) + " lives on another device");
        if (!writable_on(j.cube, ctx->device) || (j.weights && !writable_on(j.weights, ctx->device)))
            return fail(ctx, HCG_EINVAL, "job " + std::to_string(i) + ": outputs are not device memory of the "
                                         "context's device");
        if (!j.field->d_spec && auto_engine(j.field) == HCG_ENGINE_FP32)
            return fail(ctx, HCG_ESTATE, "job " + std::to_string(i) + ": field has no spectra for its engine");
        if (!fp32_weights_fit(j.field))
            return fail(ctx, HCG_EINVAL, "job " + std::to_string(i) + ": weights exceed the FP32 weights of the "
                                         "multi-channel engines");
        if (j.layout != HCG_LAYOUT_SAMPLE_MAJOR && j.layout != HCG_LAYOUT_CHANNEL_MAJOR)
            return fail(ctx, HCG_EINVAL, "unknown layout");
    }
    CK(ctx, cudaMemsetAsync(ctx->d_stats, 0, offsetof(DevStats, invalid_input), ctx->stream), "stats reset");
    // The batch kernels evaluate GAUSS1D; jobs with the other kernels run on
    // their own after the batch, as do the jobs the batch routes out. Jobs of
    // at least kBatchMaxPixels target pixels fill the GPU by themselves and go
    // straight to the single-job path (its persistent kernels), without a
    // pass through the batch's geometry graph.
    auto alone_now = [&](const hcg_job &j) {
        return j.field->kernel_type != HCG_GAUSS1D || ctx->factor > 1 || job_pixels(j) >= kBatchMaxPixels;
    };
    std::vector<hcg_job> shared;
    std::vector<uint32_t> index;  // shared job -> caller's job
    for (uint32_t i = 0; i < njobs; ++i) {
        // coarsened runs grid on the single-job path
        if (alone_now(jobs[i])) continue;
        shared.push_back(jobs[i]);
        index.push_back(i);
    }
    std::vector<char> fallback;
    std::string why;
    cudaError_t e = cudaSuccess;
    if (!shared.empty()) e = grid_batch(ctx, (uint32_t)shared.size(), shared.data(), fallback, why);
    if (e == cudaErrorTimeout) return fail(ctx, HCG_ETIMEOUT, why);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "grid batch", why);
    std::vector<char> alone(njobs, 0);
    for (uint32_t k = 0; k < shared.size(); ++k) alone[index[k]] = fallback[k];
    for (uint32_t i = 0; i < njobs; ++i) alone[i] |= alone_now(jobs[i]);
    for (uint32_t i = 0; i < njobs; ++i) {
        if (!alone[i]) continue;
        e = grid_field(ctx, jobs[i].field, jobs[i].target, jobs[i].cube, jobs[i].layout, jobs[i].weights,
                       auto_engine(jobs[i].field), why);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "grid batch fallback", why);
        if (batch_trace()) {
            float ms = 0.f;
            cudaStreamSynchronize(ctx->stream);
            cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
            fprintf(stderr, "[hcg batch] job %u on its own (%llu samples, %u channels, %ux%u pixels): %.3f ms\n", i,
                    (unsigned long long)jobs[i].field->n, jobs[i].field->nchan, jobs[i].target->nx, jobs[i].target->ny,
                    ms);
        }
    }
    CK(ctx, cudaStreamSynchronize(ctx->stream), "grid batch");
    return HCG_OK;
}

hcg_status hcg_get_stats(hcg_context *ctx, hcg_stats *out) {
    if (!ctx || !out) return HCG_EINVAL;
    Guard g(ctx);
    DevStats d;
    CK(ctx, cudaMemcpyAsync(&d, ctx->d_stats, sizeof d, cudaMemcpyDeviceToHost, ctx->stream), "stats");
    CK(ctx, cudaStreamSynchronize(ctx->stream), "stats");
    out->pairs_candidate = d.pairs_candidate;
    out->pairs_within = d.pairs_within;
    out->ring_skips = d.ring_skips;
    out->hard_roundings = d.hard_roundings;
    out->tc_macs = d.tc_macs;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) != cudaSuccess) {
        cudaGetLastError();
        ms = 0.f;
    }
    out->ms_total = ms;
    // phases: ev0 | prep | evp0 | count+scan | evp1 | weights | evp2 | channel sums | ev1
    cudaEvent_t marks[5] = {ctx->ev0, ctx->evp[0], ctx->evp[1], ctx->evp[2], ctx->ev1};
    for (int i = 0; i < 4; ++i) {
        float m = 0.f;
        if (cudaEventElapsedTime(&m, marks[i], marks[i + 1]) != cudaSuccess) {
            cudaGetLastError();
            m = 0.f;
        }
        out->ms_phase[i] = m;
    }
    return HCG_OK;
}

hcg_status hcg_set_entry_budget(hcg_context *ctx, uint64_t bytes) {
    if (!ctx || bytes < 4096) return HCG_EINVAL;
    Guard g(ctx);
    ctx->entry_budget = bytes;
    return HCG_OK;
}

hcg_status hcg_set_coarsening_factor(hcg_context *ctx, uint32_t factor) {
    if (!ctx) return HCG_EINVAL;
    Guard g(ctx);
    if (factor < 1 || factor > 3)
        return fail(ctx, HCG_EINVAL, "coarsening factor must be 1, 2 or 3 (the reference's kernel holds 3 pixels)");
    ctx->factor = factor;
    return HCG_OK;
}

hcg_status hcg_context_trim(hcg_context *ctx) {
    if (!ctx) return HCG_EINVAL;
    Guard g(ctx);
    CK(ctx, cudaStreamSynchronize(ctx->stream), "trim");
    if (ctx->pool) CK(ctx, cudaMemPoolTrimTo(ctx->pool, 0), "trim");
    return HCG_OK;
}

hcg_status hcg_synchronize(hcg_context *ctx) {
    if (!ctx) return HCG_EINVAL;
    Guard g(ctx);
    CK(ctx, cudaStreamSynchronize(ctx->stream), "synchronize");
    return HCG_OK;
}

}  // extern "C"
