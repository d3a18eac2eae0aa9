// context.cu -- context, density, spectrum and CCCS-kernel handles.
#include <cstring>
#include <mutex>

#include "fd2_internal.cuh"

namespace fd2 {

int ctx_buffer(fd2_context* ctx, int slot, size_t bytes, cudaStream_t st, void** out) {
    FD2_REQUIRE(slot >= 0 && slot < kBufCount, FD2_ERR_INVALID_ARGUMENT, "ctx_buffer: slot %d", slot);
    // The buffer lives in the order of the stream of its last use.  A use on
    // another stream first waits for the device: the earlier use may still be
    // running (and the stream it ran on may no longer exist).
    if (ctx->buf[slot] && ctx->buf_stream[slot] != st) FD2_CHECK_CUDA(cudaDeviceSynchronize());
    if (bytes > ctx->buf_bytes[slot]) {
        // the larger buffer replaces the old one in this stream's order: work
        // already enqueued on it reads the old buffer first
        if (ctx->buf[slot]) FD2_CHECK_CUDA(cudaFreeAsync(ctx->buf[slot], st));
        ctx->buf[slot] = nullptr;
        ctx->buf_bytes[slot] = 0;
        FD2_CHECK_CUDA(cudaMallocFromPoolAsync(&ctx->buf[slot], bytes, ctx->pool, st));
        ctx->buf_bytes[slot] = bytes;
    }
    ctx->buf_stream[slot] = st;
    *out = ctx->buf[slot];
    return FD2_OK;
}

void ctx_graphs_free(fd2_context* ctx) {
    for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
    ctx->graphs.clear();
    for (int i = 0; i < 2; i++) {
        if (ctx->stage_free[i]) {
            cudaEventSynchronize(ctx->stage_free[i]);
            cudaEventDestroy(ctx->stage_free[i]);
        }
        if (ctx->h_stage[i]) cudaFreeHost(ctx->h_stage[i]);
        ctx->stage_free[i] = nullptr;
        ctx->h_stage[i] = nullptr;
        ctx->h_stage_bytes[i] = 0;
    }
}

// One pool per device for the densities of fd2_density_create: created on
// first use and kept until the process ends, so a density may be freed after
// the context it was made with; freed memory is kept for the next density.
int density_pool(int device, cudaMemPool_t* out) {
    static std::mutex mu;
    static cudaMemPool_t pools[kMaxDevices] = {};
    FD2_REQUIRE(device >= 0 && device < kMaxDevices, FD2_ERR_INVALID_ARGUMENT, "density pool: device %d", device);
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[device]) {
        cudaMemPoolProps pp = {};
        pp.allocType = cudaMemAllocationTypePinned;
        pp.handleTypes = cudaMemHandleTypeNone;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = device;
        const uint64_t keep = ~0ull;
        cudaMemPool_t p = nullptr;
        FD2_CHECK_CUDA(cudaMemPoolCreate(&p, &pp));
        if (cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, (void*)&keep) != cudaSuccess) {
            cudaMemPoolDestroy(p);
            fd2::set_error("density pool: cannot set its release threshold");
            return FD2_ERR_CUDA;
        }
        pools[device] = p;
    }
    *out = pools[device];
    return FD2_OK;
}

int density_create_pooled(fd2_context* ctx, const float* host_density, const fd2_volume_t* volume,
                          fd2_density** out) {
    FD2_REQUIRE(ctx && host_density && volume && out, FD2_ERR_INVALID_ARGUMENT, "density_create: null argument");
    const size_t nv = (size_t)volume->dim[0] * volume->dim[1] * volume->dim[2];
    FD2_REQUIRE(nv > 0, FD2_ERR_INVALID_ARGUMENT, "density_create: empty volume");
    FD2_REQUIRE(volume->voxel_size[0] > 0 && volume->voxel_size[1] > 0 && volume->voxel_size[2] > 0,
                FD2_ERR_INVALID_ARGUMENT, "density_create: voxel size must be positive");
    void* p = nullptr;
    FD2_CHECK_CUDA(cudaMallocFromPoolAsync(&p, nv * sizeof(float), ctx->pool, ctx->stream));
    const cudaError_t e = cudaMemcpyAsync(p, host_density, nv * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) {
        cudaFreeAsync(p, ctx->stream);
        FD2_CHECK_CUDA(e);
    }
    auto* d = new fd2_density();
    d->ctx = ctx;
    d->vol = *volume;
    d->d_density = (float*)p;
    d->device = ctx->device;
    d->pooled = true;
    *out = d;
    return FD2_OK;
}

}  // namespace fd2

extern "C" {

int fd2_context_create(int device, fd2_context** out) {
    FD2_REQUIRE(out, FD2_ERR_INVALID_ARGUMENT, "context_create: null out");
    *out = nullptr;
    int n = 0;
    FD2_CHECK_CUDA(cudaGetDeviceCount(&n));
    FD2_REQUIRE(device >= 0 && device < n, FD2_ERR_INVALID_ARGUMENT, "no CUDA device %d (%d present)", device, n);
    FD2_CHECK_CUDA(cudaSetDevice(device));
    auto* c = new fd2_context();
    c->device = device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        delete c;
        fd2::set_error("cudaGetDeviceProperties failed");
        return FD2_ERR_CUDA;
    }
    c->sm_count = prop.multiProcessorCount;
    cudaMemPoolProps pp = {};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.handleTypes = cudaMemHandleTypeNone;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = device;
    const uint64_t keep = ~0ull;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&c->d_status, sizeof(fd2::DeviceStatus)) != cudaSuccess ||
        cudaMemset(c->d_status, 0, sizeof(fd2::DeviceStatus)) != cudaSuccess ||
        cudaMemPoolCreate(&c->pool, &pp) != cudaSuccess ||
        cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, (void*)&keep) != cudaSuccess) {
        fd2::set_error("context_create: stream/status/pool allocation failed");
        if (c->stream) cudaStreamDestroy(c->stream);
        if (c->d_status) cudaFree(c->d_status);
        if (c->pool) cudaMemPoolDestroy(c->pool);
        delete c;
        return FD2_ERR_CUDA;
    }
    *out = c;
    return FD2_OK;
}

int fd2_context_destroy(fd2_context* c) {
    if (!c) return FD2_OK;
    cudaSetDevice(c->device);
    cudaDeviceSynchronize();  // no work of any stream still uses the context's memory
    fd2::ctx_graphs_free(c);
    for (void* b : c->buf)
        if (b) cudaFreeAsync(b, c->stream);
    if (c->d_status) cudaFree(c->d_status);
    if (c->stream) {
        cudaStreamSynchronize(c->stream);
        cudaStreamDestroy(c->stream);
    }
    if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
    if (c->pool) {
        cudaDeviceSynchronize();  // stream-ordered frees on other streams complete first
        cudaMemPoolDestroy(c->pool);
    }
    delete c;
    return FD2_OK;
}

int fd2_context_release(fd2_context* c) {
    FD2_REQUIRE(c, FD2_ERR_INVALID_ARGUMENT, "null context");
    FD2_CHECK_CUDA(cudaDeviceSynchronize());  // no work of any stream still uses the buffers
    fd2::ctx_graphs_free(c);  // the graphs name the buffers freed below
    for (int i = 0; i < fd2::kBufCount; i++) {
        if (c->buf[i]) FD2_CHECK_CUDA(cudaFreeAsync(c->buf[i], c->stream));
        c->buf[i] = nullptr;
        c->buf_bytes[i] = 0;
        c->buf_stream[i] = nullptr;
    }
    FD2_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    FD2_CHECK_CUDA(cudaMemPoolTrimTo(c->pool, 0));
    return FD2_OK;
}

int fd2_context_graph_counts(fd2_context* c, uint64_t* launches, uint64_t* instantiations, uint64_t* updates) {
    FD2_REQUIRE(c, FD2_ERR_INVALID_ARGUMENT, "null context");
    if (launches) *launches = c->graph_launches;
    if (instantiations) *instantiations = c->graph_instantiations;
    if (updates) *updates = c->graph_updates;
    return FD2_OK;
}

int fd2_context_synchronize(fd2_context* c) {
    FD2_REQUIRE(c, FD2_ERR_INVALID_ARGUMENT, "null context");
    FD2_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    return FD2_OK;
}

int fd2_context_set_timing(fd2_context* c, int on) {
    FD2_REQUIRE(c, FD2_ERR_INVALID_ARGUMENT, "null context");
    c->timing = on ? 1 : 0;
    return FD2_OK;
}

int fd2_context_stage_times(fd2_context* c, double* ms, int n) {
    FD2_REQUIRE(c && ms, FD2_ERR_INVALID_ARGUMENT, "null argument");
    for (int i = 0; i < n && i < FD2_STAGE_COUNT; i++) ms[i] = c->stage_ms[i];
    for (int i = 0; i < FD2_STAGE_COUNT; i++) c->stage_ms[i] = 0.0;
    return FD2_OK;
}

uint64_t fd2_context_launch_count(const fd2_context* c) { return c ? c->launches : 0; }

int fd2_context_tuned_schedules(const fd2_context* c, size_t cap, uint64_t* keys, int32_t* schedules, size_t* n,
                                uint64_t* runs) {
    FD2_REQUIRE(c && n && runs && (cap == 0 || (keys && schedules)), FD2_ERR_INVALID_ARGUMENT,
                "tuned_schedules: bad argument");
    size_t i = 0;
    for (const auto& kv : c->cccs_schedule) {
        if (i < cap) {
            keys[i] = kv.first;
            schedules[i] = kv.second;
        }
        i++;
    }
    *n = i;
    *runs = c->tuning_runs;
    return FD2_OK;
}

int fd2_density_create(fd2_context* ctx, const float* host_density, const fd2_volume_t* volume, fd2_density** out) {
    FD2_REQUIRE(ctx && host_density && volume && out, FD2_ERR_INVALID_ARGUMENT, "density_create: null argument");
    size_t nv = (size_t)volume->dim[0] * volume->dim[1] * volume->dim[2];
    FD2_REQUIRE(nv > 0, FD2_ERR_INVALID_ARGUMENT, "density_create: empty volume");
    FD2_REQUIRE(volume->voxel_size[0] > 0 && volume->voxel_size[1] > 0 && volume->voxel_size[2] > 0,
                FD2_ERR_INVALID_ARGUMENT, "density_create: voxel size must be positive");
    // The device copy comes from the library's density pool of this device
    // (no cudaMalloc / cudaFree per plan: those driver calls now and then took
    // tens to hundreds of ms), and is complete when this returns, so any
    // stream may read it.
    cudaMemPool_t pool = nullptr;
    FD2_TRY(fd2::density_pool(ctx->device, &pool));
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, nv * sizeof(float), pool, ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        fd2::set_error("density_create: allocation of %zu bytes failed", nv * sizeof(float));
        return FD2_ERR_OUT_OF_MEMORY;
    }
    if (cudaMemcpyAsync(p, host_density, nv * sizeof(float), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaFreeAsync(p, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
        fd2::set_error("density_create: copy failed");
        return FD2_ERR_CUDA;
    }
    auto* d = new fd2_density();
    d->ctx = ctx;
    d->vol = *volume;
    d->d_density = (float*)p;
    d->device = ctx->device;
    *out = d;
    return FD2_OK;
}

int fd2_density_destroy(fd2_density* d) {
    if (!d) return FD2_OK;
    if (d->d_density) {
        if (d->pooled) {
            cudaFreeAsync(d->d_density, d->ctx->stream);
        } else {
            // A density made by fd2_density_create may be read by work on any
            // stream, and may outlive its context: like cudaFree, wait for the
            // device, then return the memory to the library's density pool,
            // which lives as long as the process, on the default stream.
            int cur = -1;
            cudaGetDevice(&cur);
            if (cur != d->device) cudaSetDevice(d->device);
            cudaDeviceSynchronize();
            cudaFreeAsync(d->d_density, cudaStreamLegacy);
            cudaGetLastError();  // nothing a later launch check should see
            if (cur >= 0 && cur != d->device) cudaSetDevice(cur);
        }
    }
    delete d;
    return FD2_OK;
}

const float* fd2_density_device_ptr(const fd2_density* d) { return d ? d->d_density : nullptr; }

int fd2_spectrum_create(fd2_context* ctx, int n, const float* energy, const float* fluence, const float* mu,
                        const float* mu_en, fd2_spectrum** out) {
    FD2_REQUIRE(ctx && energy && fluence && mu && out, FD2_ERR_INVALID_ARGUMENT, "spectrum_create: null argument");
    FD2_REQUIRE(n > 0 && n <= fd2::kMaxSpectrum, FD2_ERR_INVALID_ARGUMENT,
                "spectrum_create: %d bins (1..%d supported, MAX_KERNEL_NUM)", n, fd2::kMaxSpectrum);
    auto* s = new fd2_spectrum();
    s->ctx = ctx;
    s->n = n;
    for (int i = 0; i < n; i++) {
        s->energy[i] = energy[i];
        s->fluence[i] = fluence[i];
        s->mu[i] = mu[i];
        s->mu_en[i] = mu_en ? mu_en[i] : 0.0f;
    }
    *out = s;
    return FD2_OK;
}

int fd2_spectrum_destroy(fd2_spectrum* s) {
    delete s;
    return FD2_OK;
}

int fd2_kernel_create(fd2_context* ctx, int n_theta, const float* theta, const float* A, const float* a,
                      const float* B, const float* b, int n_phi, const float* phi, fd2_cccs_kernel** out) {
    FD2_REQUIRE(ctx && theta && A && a && B && b && phi && out, FD2_ERR_INVALID_ARGUMENT,
                "kernel_create: null argument");
    FD2_REQUIRE(n_theta > 0 && n_theta <= fd2::kMaxAngles && n_phi > 0 && n_phi <= fd2::kMaxAngles,
                FD2_ERR_INVALID_ARGUMENT, "kernel_create: nTheta=%d nPhi=%d (1..%d supported)", n_theta, n_phi,
                fd2::kMaxAngles);
    for (int i = 0; i < n_theta; i++)
        FD2_REQUIRE(a[i] > 0 && b[i] > 0, FD2_ERR_INVALID_ARGUMENT, "kernel_create: a and b must be positive");
    auto* k = new fd2_cccs_kernel();
    k->ctx = ctx;
    k->n_theta = n_theta;
    k->n_phi = n_phi;
    for (int i = 0; i < n_theta; i++) {
        k->theta[i] = theta[i]; k->A[i] = A[i]; k->a[i] = a[i]; k->B[i] = B[i]; k->b[i] = b[i];
    }
    for (int i = 0; i < n_phi; i++) k->phi[i] = phi[i];
    *out = k;
    return FD2_OK;
}

int fd2_kernel_destroy(fd2_cccs_kernel* k) {
    delete k;
    return FD2_OK;
}

}  // extern "C"
