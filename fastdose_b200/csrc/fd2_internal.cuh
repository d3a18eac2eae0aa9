// fd2_internal.cuh -- shared internals of libfd2 (not part of the ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/fd2.h"
#include "../../include/fd2_imrt.h"

namespace fd2 {

// ---------------------------------------------------------------- errors
void set_error(const char* fmt, ...);

#define FD2_CHECK_CUDA(call)                                                              \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            ::fd2::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
            return e_ == cudaErrorMemoryAllocation ? FD2_ERR_OUT_OF_MEMORY : FD2_ERR_CUDA;  \
        }                                                                                  \
    } while (0)

#define FD2_REQUIRE(cond, code, ...)       \
    do {                                   \
        if (!(cond)) {                     \
            ::fd2::set_error(__VA_ARGS__); \
            return (code);                 \
        }                                  \
    } while (0)

#define FD2_TRY(call)              \
    do {                           \
        int s_ = (call);           \
        if (s_ != FD2_OK) return s_; \
    } while (0)

// Maximum table sizes, the reference's MAX_KERNEL_NUM / MAX_THETA_ANGLES
// (FastDoseLib/include/spectrum.cuh:7, kernel.cuh:7).
constexpr int kMaxSpectrum = 24;
constexpr int kMaxAngles = 24;

// Device-side status word written by kernels whose loops are bounded by an
// iteration cap: 0 = fine, otherwise an FD2 status code (negative).
struct DeviceStatus {
    int code;
    int where;
};

}  // namespace fd2

// ---------------------------------------------------------------- handles
struct fd2_context {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;          // internal work stream
    fd2::DeviceStatus* d_status = nullptr;  // device status word
    // reusable grow-only device buffers (fd2::ctx_buffer slots), kept between calls
    void* buf[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    size_t buf_bytes[5] = {0, 0, 0, 0, 0};
    cudaStream_t buf_stream[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // stream of each buffer's last use
    // second work stream of the construction: the column stage of one batch
    // runs on it beside the next batch's Terma and CCCS (created on first use)
    cudaStream_t aux_stream = nullptr;
    // stream-ordered pool for batch buffers and dose-matrix storage; it keeps
    // freed memory (release threshold = max) so repeated plans reuse it
    cudaMemPool_t pool = nullptr;
    // instrumentation: kernels launched, and (when enabled) device time per stage
    uint64_t launches = 0;
    int timing = 0;
    double stage_ms[FD2_STAGE_COUNT] = {0};
    // autotuned CCCS schedule (0 or 1) per batch shape, measured on first use
    std::unordered_map<uint64_t, int> cccs_schedule;
    uint64_t tuning_runs = 0;  // batches on which both schedules were timed
    // graph-captured construction (fd2_dosemat_params_t.graph): one executable
    // graph per batch shape, updated in place for each batch; the batch's small
    // tables go up from pinned staging (two slots, each reused once the graph
    // that read it has run)
    std::unordered_map<uint64_t, cudaGraphExec_t> graphs;
    void* h_stage[2] = {nullptr, nullptr};
    size_t h_stage_bytes[2] = {0, 0};
    cudaEvent_t stage_free[2] = {nullptr, nullptr};
    int stage_slot = 0;
    uint64_t graph_launches = 0, graph_instantiations = 0, graph_updates = 0;
};

namespace fd2 {
// Brackets one stage of work on a stream with CUDA events when the context's
// timing is on; the elapsed time is added to ctx->stage_ms[stage] at finish().
struct StageTimer {
    fd2_context* ctx;
    cudaStream_t st;
    int stage;
    cudaEvent_t a = nullptr, b = nullptr;
    StageTimer(fd2_context* c, cudaStream_t s, int stg) : ctx(c), st(s), stage(stg) {
        if (ctx->timing) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, st);
        }
    }
    void stop() {
        if (ctx->timing && b) cudaEventRecord(b, st);
    }
    ~StageTimer() {
        if (ctx->timing && a && b) {
            float ms = 0.0f;
            if (cudaEventSynchronize(b) == cudaSuccess && cudaEventElapsedTime(&ms, a, b) == cudaSuccess)
                ctx->stage_ms[stage] += ms;
        }
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};
}  // namespace fd2

struct fd2_density {
    fd2_context* ctx = nullptr;
    fd2_volume_t vol{};
    float* d_density = nullptr;  // float[z][y][x], from the context's pool
    int device = 0;
    bool pooled = false;         // a service density: used and freed in the context stream's order only
};

struct fd2_spectrum {
    fd2_context* ctx = nullptr;
    int n = 0;
    float energy[fd2::kMaxSpectrum];
    float fluence[fd2::kMaxSpectrum];
    float mu[fd2::kMaxSpectrum];
    float mu_en[fd2::kMaxSpectrum];
};

struct fd2_cccs_kernel {
    fd2_context* ctx = nullptr;
    int n_theta = 0, n_phi = 0;
    float theta[fd2::kMaxAngles], A[fd2::kMaxAngles], a[fd2::kMaxAngles], B[fd2::kMaxAngles],
        b[fd2::kMaxAngles], phi[fd2::kMaxAngles];
};

namespace fd2 {

// Grow-only device buffers owned by a context, one per use, from the
// context's pool.  A buffer is reused by every later call on the context
// (calls on one context are serialised: one host thread, work in stream
// order); growing it replaces the old one in the order of stream `st`, and
// waits for the device only when the previous use was on another stream.
enum CtxBuffer { kBufCccs = 0, kBufBev = 1, kBufColumns = 2, kBufBatch = 3, kBufBev2 = 4, kBufCount = 5 };
int ctx_buffer(fd2_context* ctx, int slot, size_t bytes, cudaStream_t st, void** out);
inline int ctx_scratch(fd2_context* ctx, size_t bytes, cudaStream_t st, void** out) {
    return ctx_buffer(ctx, kBufCccs, bytes, st, out);
}

// A density whose device copy comes from the context's pool in the order of
// the context's stream, and returns to it the same way on destroy: no call
// that waits for the whole device.  Only for work issued on ctx->stream (a
// service worker's requests); the public fd2_density_create allocates plainly.
constexpr int kMaxDevices = 64;
int density_pool(int device, cudaMemPool_t* out);
int density_create_pooled(fd2_context* ctx, const float* host_density, const fd2_volume_t* volume,
                          fd2_density** out);

// Spectrum table passed by value to kernels (lives in the kernel parameter
// space, not in process-global __constant__ memory).
struct SpectrumParams {
    int n;
    float fluence_energy_mu[kMaxSpectrum];  // fluence * energy * mu per bin
    float mu[kMaxSpectrum];
};

// Per-cone constants of the CCCS march, one entry per (theta, phi) pair,
// directions precomputed on the host (see cccs.cu).
struct ConeParams {
    int n_theta_fwd;        // forward zenith bins actually used
    int n_phi;
    float a[kMaxAngles], b[kMaxAngles];      // attenuation per used zenith bin
    float A_a[kMaxAngles], B_b[kMaxAngles];  // A/a and B/b
};

// Forward zenith bins and azimuths of a CCCS kernel (the angles the cone
// directions are made from).
struct ConeAngles {
    int n_theta_fwd;
    int n_phi;
    float theta[kMaxAngles];
    float phi[kMaxAngles];
};

// Device table of cone directions, float4 [beam][theta_fwd][phi] (cccs_dirs.cu).
int launch_cone_dirs(const fd2_beam_t* d_beams, size_t n_beams, const ConeAngles& ang, float4* d_out,
                     cudaStream_t stream);

// Bytes of context scratch launch_cccs_host needs for a batch (the direction
// table, and the per-zenith planes of schedule 1), so a caller can size the
// scratch before a stream capture.
size_t cccs_scratch_bytes(size_t n_beams, const fd2_beam_t* h_beams, const fd2_cccs_kernel* k, int schedule);

// Graph state of a context: executable graphs, pinned staging, events.
void ctx_graphs_free(fd2_context* ctx);

// Launchers used by the plan-level code (dosemat.cu).
int launch_terma(fd2_context* ctx, size_t fmap_npixels, size_t n_beams, const fd2_beam_t* d_beams,
                 const float* const* d_fluence, float* const* d_terma, float* const* d_dens,
                 const fd2_density* density, const fd2_spectrum* spectrum, int fluence_skip,
                 cudaStream_t stream);

}  // namespace fd2
