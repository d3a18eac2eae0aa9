// dosemat.cu -- dose-loading-matrix construction (IMRT::DoseMatConstruction,
// IMRTOpt/src/IMRTDoseMat.cu:14-301), the CSR ensemble with its on-disk layout
// (IMRT::MatCSREnsemble, IMRTOpt/src/IMRTSparseMatEns.cu), BEV->PVCS entry points
// and beamlet flagging (IMRT::beamletFlagInit, IMRTOpt/src/IMRTBeamBundle.cu:130-316).
//
// Pipeline per batch of beamlets (a batch holds whole beams and is sized by a
// BEV-scratch memory budget instead of the reference's one beam per iteration):
//   Terma (one launch) -> CCCS (one launch) -> column count -> column values
//   -> row gather into the growing device CSR.
// Two small device->host reads per batch (row capacities, row nnz) size the
// buffers; there is no dense beamlets x voxels matrix.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <functional>
#include <numeric>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "fd2_internal.cuh"
#include "resample.cuh"

struct fd2_csr_ensemble {
    fd2_context* ctx = nullptr;
    uint64_t n_cols = 0;
    int value_type = FD2_VALUES_F32;
    std::vector<uint64_t> mat_rows;  // [n_mats + 1]
    uint64_t n_rows = 0, nnz = 0;
    int64_t* d_row_off = nullptr;    // [n_rows + 1]
    int32_t* d_col = nullptr;        // [cap]
    void* d_val = nullptr;           // [cap]
    float* d_scale = nullptr;        // [n_rows] (16-bit formats)
    cudaStream_t stream = nullptr;   // the arrays are allocated, grown and freed in this stream's order
    bool verbose = false;            // per-batch progress on stdout
    uint64_t nnz_bound = 0;          // host-side upper bound of nnz while batches are in flight
    uint64_t row_cap = 0, nnz_cap = 0;
};

namespace fd2 {

namespace {

size_t value_bytes(int vt) { return vt == FD2_VALUES_F32 ? 4 : 2; }

void rot_axis_d(const double p[3], const double r[3], double t, double o[3]) {
    double s = std::sin(t), c = std::cos(t);
    double k = (1 - c) * (p[0] * r[0] + p[1] * r[1] + p[2] * r[2]);
    double a = k * r[0] + c * p[0] + s * (r[1] * p[2] - r[2] * p[1]);
    double b = k * r[1] + c * p[1] + s * (r[2] * p[0] - r[0] * p[2]);
    double d = k * r[2] + c * p[2] + s * (r[0] * p[1] - r[1] * p[0]);
    o[0] = a; o[1] = b; o[2] = d;
}

// Grows the ensemble's device arrays (amortised growth), from the context's
// pool and in the order of the ensemble's stream: the old contents are copied
// and the old arrays freed asynchronously.
__global__ void offsets_shift_kernel(const int64_t* __restrict__ src, uint64_t n, int64_t shift,
                                     int64_t* __restrict__ dst) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = src[i] + shift;
}

// dst[i] = src[i] + shift for i < n (row offsets of a part moved after the parts before it)
int launch_offsets_shift(const int64_t* src, uint64_t n, int64_t shift, int64_t* dst, cudaStream_t st) {
    const unsigned blocks = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 148 * 8));
    offsets_shift_kernel<<<blocks, 256, 0, st>>>(src, n, shift, dst);
    FD2_CHECK_CUDA(cudaGetLastError());
    return FD2_OK;
}

int ensemble_reserve(fd2_csr_ensemble* e, uint64_t rows, uint64_t nnz) {
    cudaStream_t st = e->stream;
    cudaMemPool_t pool = e->ctx->pool;
    if (rows + 1 > e->row_cap) {
        uint64_t cap = std::max<uint64_t>(rows + 1, e->row_cap * 2);
        int64_t* p;
        FD2_CHECK_CUDA(cudaMallocFromPoolAsync((void**)&p, cap * sizeof(int64_t), pool, st));
        if (e->d_row_off) {
            FD2_CHECK_CUDA(cudaMemcpyAsync(p, e->d_row_off, (e->n_rows + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice,
                                           st));
            FD2_CHECK_CUDA(cudaFreeAsync(e->d_row_off, st));
        } else {
            FD2_CHECK_CUDA(cudaMemsetAsync(p, 0, sizeof(int64_t), st));
        }
        e->d_row_off = p;
        if (e->value_type != FD2_VALUES_F32) {
            float* sc;
            FD2_CHECK_CUDA(cudaMallocFromPoolAsync((void**)&sc, cap * sizeof(float), pool, st));
            if (e->d_scale) {
                FD2_CHECK_CUDA(cudaMemcpyAsync(sc, e->d_scale, e->n_rows * sizeof(float), cudaMemcpyDeviceToDevice, st));
                FD2_CHECK_CUDA(cudaFreeAsync(e->d_scale, st));
            }
            e->d_scale = sc;
        }
        e->row_cap = cap;
    }
    if (nnz > e->nnz_cap) {
        uint64_t cap = std::max<uint64_t>(nnz, e->nnz_cap + e->nnz_cap / 2);
        int32_t* c;
        void* v;
        FD2_CHECK_CUDA(cudaMallocFromPoolAsync((void**)&c, cap * sizeof(int32_t), pool, st));
        FD2_CHECK_CUDA(cudaMallocFromPoolAsync(&v, cap * value_bytes(e->value_type), pool, st));
        if (e->d_col) {
            FD2_CHECK_CUDA(cudaMemcpyAsync(c, e->d_col, e->nnz * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
            FD2_CHECK_CUDA(
                cudaMemcpyAsync(v, e->d_val, e->nnz * value_bytes(e->value_type), cudaMemcpyDeviceToDevice, st));
            FD2_CHECK_CUDA(cudaFreeAsync(e->d_col, st));
            FD2_CHECK_CUDA(cudaFreeAsync(e->d_val, st));
        }
        e->d_col = c;
        e->d_val = v;
        e->nnz_cap = cap;
    }
    return FD2_OK;
}

template <typename T>
int upload(const std::vector<T>& h, T** d, cudaMemPool_t pool, cudaStream_t st) {
    FD2_CHECK_CUDA(cudaMallocFromPoolAsync((void**)d, std::max<size_t>(1, h.size()) * sizeof(T), pool, st));
    if (!h.empty()) FD2_CHECK_CUDA(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return FD2_OK;
}

}  // namespace

void make_column_info(const fd2_beam_t& b, const fd2_volume_t* vol, ColumnInfo& ci) {
    std::memset(&ci, 0, sizeof(ci));
    // PVCS -> BEV (rotateBeamAtOriginRHS, FastDoseLib/src/geom.cu:36-44) applied to unit vectors
    const double th = b.angles[0], ph = b.angles[1], co = b.angles[2];
    const double axis[3] = {std::sin(-ph), 0.0, std::cos(-ph)}, yax[3] = {0, 1, 0};
    for (int c = 0; c < 3; c++) {
        double e[3] = {0, 0, 0}, t[3], o[3];
        e[c] = 1;
        rot_axis_d(e, axis, -th, t);
        rot_axis_d(t, yax, ph + co, o);
        for (int r = 0; r < 3; r++) ci.R[r * 3 + c] = (float)o[r];
    }
    for (int i = 0; i < 3; i++) ci.src[i] = b.source[i];
    ci.bsx = b.beamlet_size[0];
    ci.bsy = b.beamlet_size[1];
    ci.fx = (int)b.fmap_size[0];
    ci.fy = (int)b.fmap_size[1];
    ci.hx = 0.5f * ci.fx;
    ci.hy = 0.5f * ci.fy;
    ci.inv_sad = 1.0f / b.sad;
    ci.lim_min = b.lim_min;
    ci.ls = b.long_spacing;
    ci.inv_ls = 1.0f / b.long_spacing;
    ci.L = (int)b.long_dim;
    if (!vol) return;
    // frustum corners in BEV (x lateral, y depth, z lateral) -> PVCS box
    const double vx = vol->voxel_size[0], vy = vol->voxel_size[1], vz = vol->voxel_size[2];
    const double hdiag = 0.5 * std::sqrt(vx * vx + vy * vy + vz * vz);
    const double y0 = std::max(1e-3, (double)b.lim_min - hdiag), y1 = (double)b.lim_min + ci.L * (double)ci.ls + hdiag;
    double lo[3] = {1e30, 1e30, 1e30}, hi[3] = {-1e30, -1e30, -1e30};
    for (int k = 0; k < 8; k++) {
        double y = (k & 1) ? y1 : y0;
        double x = ((k & 2) ? 1 : -1) * (ci.hx * ci.bsx * y / b.sad);
        double z = ((k & 4) ? 1 : -1) * (ci.hy * ci.bsy * y / b.sad);
        // BEV -> PVCS is the transpose of R
        for (int r = 0; r < 3; r++) {
            double p = ci.R[0 * 3 + r] * x + ci.R[1 * 3 + r] * y + ci.R[2 * 3 + r] * z + ci.src[r];
            lo[r] = std::min(lo[r], p);
            hi[r] = std::max(hi[r], p);
        }
    }
    const double vsz[3] = {vx, vy, vz};
    for (int r = 0; r < 3; r++) {
        double a = (lo[r] - hdiag) / vsz[r] - 0.5, c = (hi[r] + hdiag) / vsz[r] - 0.5;
        long i0 = (long)std::floor(a) - 1, i1 = (long)std::ceil(c) + 2;
        i0 = std::max(0L, i0);
        i1 = std::min((long)vol->dim[r], i1);
        if (i1 < i0) i1 = i0;
        ci.box[r] = (int)i0;
        ci.box[3 + r] = (int)i1;
    }
}

// The CCCS march of a batch under the context's tuned schedule.  Batches are
// keyed by shape (beamlets to the nearest power of two, map pixels, cone
// counts); the first batch of a shape runs both schedules -- one block per
// beamlet over all zenith bins, and one block per (beamlet, zenith bin) -- and
// keeps the faster for the shape.  The two give bitwise identical doses, so
// the batch keeps the second run's result (its dose buffer is cleared in
// between).
static int tuned_cccs(fd2_context* ctx, size_t nb, int P, const fd2_cccs_kernel* k, cudaStream_t st,
                      const std::function<int(int)>& run, float* dD, size_t n_dose) {
    int bucket = 0;
    while (((size_t)1 << (bucket + 1)) <= nb) bucket++;
    const uint64_t key = (uint64_t)bucket | (uint64_t)P << 8 | (uint64_t)k->n_phi << 24 | (uint64_t)k->n_theta << 40;
    auto it = ctx->cccs_schedule.find(key);
    if (it != ctx->cccs_schedule.end()) return run(it->second);
    cudaEvent_t ev[3];
    for (auto& e : ev) FD2_CHECK_CUDA(cudaEventCreate(&e));
    int rc = FD2_OK;
    float ms[2] = {0.0f, 0.0f};
    if (cudaEventRecord(ev[0], st) != cudaSuccess) rc = FD2_ERR_CUDA;
    if (!rc) rc = run(0);
    if (!rc && cudaEventRecord(ev[1], st) != cudaSuccess) rc = FD2_ERR_CUDA;
    if (!rc && cudaMemsetAsync(dD, 0, n_dose * sizeof(float), st) != cudaSuccess) rc = FD2_ERR_CUDA;
    cudaEvent_t mid = nullptr;
    if (!rc && cudaEventCreate(&mid) == cudaSuccess) cudaEventRecord(mid, st);
    if (!rc) rc = run(1);
    if (!rc && cudaEventRecord(ev[2], st) != cudaSuccess) rc = FD2_ERR_CUDA;
    if (!rc && cudaEventSynchronize(ev[2]) != cudaSuccess) rc = FD2_ERR_CUDA;
    if (!rc) {
        cudaEventElapsedTime(&ms[0], ev[0], ev[1]);
        cudaEventElapsedTime(&ms[1], mid ? mid : ev[1], ev[2]);
        ctx->cccs_schedule[key] = ms[1] < ms[0] ? 1 : 0;
        ctx->tuning_runs++;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (mid) cudaEventDestroy(mid);
    return rc;
}

// Candidate voxels of each beamlet (the capacity of its row): geometry only,
// so it runs before the beamlets' dose exists.
static int column_counts(fd2_context* ctx, const ColumnInfo* d_infos, size_t nb, const fd2_volume_t& vol, float extent,
                         cudaStream_t st, std::vector<uint32_t>& cnt) {
    cnt.assign(nb, 0);
    if (!nb) return FD2_OK;
    uint32_t* d_cnt = nullptr;
    FD2_CHECK_CUDA(cudaMallocFromPoolAsync((void**)&d_cnt, nb * sizeof(uint32_t), ctx->pool, st));
    int rc = launch_column_count(d_infos, nb, d_cnt, vol, extent, st);
    cudaError_t e = rc ? cudaSuccess : cudaMemcpyAsync(cnt.data(), d_cnt, nb * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d_cnt, st);
    if (!rc && e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (rc) return rc;
    FD2_CHECK_CUDA(e);
    ctx->launches += 1;
    return FD2_OK;
}

// The exact nonzero count, read back from the last row offset.
static int ensemble_sync_nnz(fd2_csr_ensemble* e) {
    int64_t v = 0;
    FD2_CHECK_CUDA(cudaMemcpyAsync(&v, e->d_row_off + e->n_rows, sizeof(int64_t), cudaMemcpyDeviceToHost, e->stream));
    FD2_CHECK_CUDA(cudaStreamSynchronize(e->stream));
    e->nnz = e->nnz_bound = (uint64_t)v;
    return FD2_OK;
}

// Column emission of a batch of beamlets whose BEV dose is in `aD` (device
// array of device pointers, [L][P] each) and whose candidate counts are `cnt`:
// values into the context's column buffer at capacity offsets, row offsets and
// scales by a device scan, then the rows gathered into the ensemble -- all in
// stream order, without waiting for the device (the exact nonzero count is
// read when the matrix is complete, or when the capacity bound runs out).
// Scratch of one batch's column stage: the candidate offsets (already on the
// device), row nonzero counts, row maxima and inverse row scales.  Direct
// launches take them from the pool; a graph-captured batch passes them in
// the context's batch buffer, since nothing may be allocated under capture.
struct ColumnScratch {
    uint64_t* cap_off = nullptr;
    uint32_t* nnz = nullptr;
    float* max = nullptr;
    float* iscale = nullptr;
};

static int append_columns(fd2_csr_ensemble* e, const ColumnInfo* d_infos, const uint32_t* cnt, size_t nb,
                          const float* const* aD, const fd2_volume_t& vol, float extent, int ss, cudaStream_t st,
                          const ColumnScratch* pre = nullptr) {
    fd2_context* ctx = e->ctx;
    uint32_t* d_nnz = nullptr;
    uint64_t* d_cap_off = nullptr;
    float *d_max = nullptr, *d_iscale = nullptr;
    int rc = [&]() -> int {
        std::vector<uint64_t> cap(nb + 1, 0);
        for (size_t k = 0; k < nb; k++) cap[k + 1] = cap[k] + cnt[k];
        if (pre) {
            // the construction reserved every beamlet's candidates up front
            FD2_REQUIRE(e->nnz_bound + cap[nb] <= e->nnz_cap && e->n_rows + nb + 1 <= e->row_cap, FD2_ERR_CAPACITY,
                        "dose_mat_construct: graph batch beyond the reserved matrix");
        } else {
            if (e->nnz_bound + cap[nb] > e->nnz_cap) {  // the bound may not fit: use the exact count
                FD2_TRY(ensemble_sync_nnz(e));
                FD2_TRY(ensemble_reserve(e, e->n_rows + nb, e->nnz + cap[nb]));
            }
            FD2_TRY(ensemble_reserve(e, e->n_rows + nb, e->nnz_bound + cap[nb]));
        }
        const uint64_t ncap = std::max<uint64_t>(1, cap[nb]);
        void* tmp = nullptr;
        FD2_TRY(ctx_buffer(ctx, kBufColumns, ncap * (sizeof(int32_t) + sizeof(float)), st, &tmp));
        int32_t* d_tcol = (int32_t*)tmp;
        float* d_tval = (float*)(d_tcol + ncap);
        const bool half = e->value_type != FD2_VALUES_F32;
        if (pre) {
            d_cap_off = pre->cap_off;
            d_nnz = pre->nnz;
            d_max = pre->max;
            d_iscale = half ? pre->iscale : nullptr;
        } else {
            FD2_TRY(upload(cap, &d_cap_off, ctx->pool, st));
            FD2_CHECK_CUDA(cudaMallocFromPoolAsync((void**)&d_nnz, nb * sizeof(uint32_t), ctx->pool, st));
            FD2_CHECK_CUDA(cudaMallocFromPoolAsync((void**)&d_max, nb * sizeof(float), ctx->pool, st));
            if (half) FD2_CHECK_CUDA(cudaMallocFromPoolAsync((void**)&d_iscale, nb * sizeof(float), ctx->pool, st));
        }
        FD2_TRY(launch_column_values(d_infos, nb, aD, d_cap_off, d_tcol, d_tval, d_nnz, d_max, vol, extent, ss, st));
        int64_t* d_roff = e->d_row_off + e->n_rows;  // [0] is this batch's first offset
        FD2_TRY(launch_column_rows(nb, d_nnz, d_max, d_roff, half ? e->d_scale + e->n_rows : nullptr, d_iscale, st));
        FD2_TRY(launch_column_gather(nb, d_cap_off, d_roff, d_tcol, d_tval, d_iscale, e->d_col, e->d_val,
                                     e->value_type, st));
        e->n_rows += nb;
        e->nnz_bound += cap[nb];
        ctx->launches += 3;  // values, row offsets, gather
        if (e->verbose)
            std::printf("  columns: %zu beamlets, %llu candidates enqueued\n", nb, (unsigned long long)cap[nb]);
        return FD2_OK;
    }();
    if (!pre)
        for (void* p : {(void*)d_nnz, (void*)d_cap_off, (void*)d_max, (void*)d_iscale})
            if (p) cudaFreeAsync(p, st);
    return rc;
}

static size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// One batch of the construction captured as a CUDA graph and launched with
// one call (fd2_dosemat_params_t.graph).  Everything the batch touches is
// sized before the capture -- the BEV, column, cone and batch buffers of the
// context, and the pinned staging of its small tables -- so the capture holds
// only copies, memsets and kernels.  The context keeps one executable graph
// per batch shape; a later batch of that shape updates it in place
// (cudaGraphExecUpdate: new pointers, sizes and grid extents) and a refused
// update instantiates afresh.  The kernels, their order and their inputs are
// those of the direct path, so the matrix is the same bit for bit.
static int graph_batch(fd2_context* ctx, fd2_csr_ensemble* e, size_t nb, const fd2_beam_t* h_beams,
                       const fd2_beam_t* d_beams, const ColumnInfo* d_infos, const uint32_t* cnt,
                       const float* d_fluence, float* dT, float* dR, float* dD, const size_t* off, size_t P,
                       const fd2_density* density, const fd2_spectrum* spectrum, const fd2_cccs_kernel* kernel,
                       const fd2_dosemat_params_t& params, int schedule, cudaStream_t st) {
    // device layout of the batch buffer: aF, aT, aR, aD (pointers), candidate
    // offsets, the march order (int32) -- uploaded from the staging -- then the
    // column-stage scratch
    const size_t up_bytes = (4 * nb + nb + 1 + (nb + 1) / 2) * sizeof(uint64_t);
    const size_t o_nnz = align256(up_bytes), o_max = o_nnz + align256(nb * 4), o_isc = o_max + align256(nb * 4);
    const size_t dev_bytes = o_isc + align256(nb * 4);
    uint64_t ncap_total = 0;
    for (size_t k = 0; k < nb; k++) ncap_total += cnt[k];
    void *batch = nullptr, *scratch = nullptr, *cols = nullptr;
    FD2_TRY(ctx_buffer(ctx, kBufBatch, dev_bytes, st, &batch));
    FD2_TRY(ctx_scratch(ctx, cccs_scratch_bytes(nb, h_beams, kernel, schedule), st, &scratch));
    FD2_TRY(ctx_buffer(ctx, kBufColumns, std::max<uint64_t>(1, ncap_total) * (sizeof(int32_t) + sizeof(float)), st,
                       &cols));
    // pinned staging: a slot is refilled once the graph that read it has run
    const int slot = ctx->stage_slot;
    ctx->stage_slot ^= 1;
    if (ctx->stage_free[slot]) FD2_CHECK_CUDA(cudaEventSynchronize(ctx->stage_free[slot]));
    else FD2_CHECK_CUDA(cudaEventCreateWithFlags(&ctx->stage_free[slot], cudaEventDisableTiming));
    if (ctx->h_stage_bytes[slot] < up_bytes) {
        // freeing pinned memory waits for the whole device (other workers'
        // streams included), so a slot starts large (1 MiB: 26k beamlets a
        // batch) and grows by doubling
        const size_t want = std::max<size_t>({up_bytes, (size_t)1 << 20, 2 * ctx->h_stage_bytes[slot]});
        if (ctx->h_stage[slot]) FD2_CHECK_CUDA(cudaFreeHost(ctx->h_stage[slot]));
        ctx->h_stage[slot] = nullptr;
        ctx->h_stage_bytes[slot] = 0;
        FD2_CHECK_CUDA(cudaHostAlloc(&ctx->h_stage[slot], want, cudaHostAllocDefault));
        ctx->h_stage_bytes[slot] = want;
    }
    uint64_t* h = (uint64_t*)ctx->h_stage[slot];
    for (size_t k = 0; k < nb; k++) {
        h[k] = (uint64_t)(uintptr_t)d_fluence;
        h[nb + k] = (uint64_t)(uintptr_t)(dT + off[k]);
        h[2 * nb + k] = (uint64_t)(uintptr_t)(dR + off[k]);
        h[3 * nb + k] = (uint64_t)(uintptr_t)(dD + off[k]);
    }
    uint64_t* hc = h + 4 * nb;
    hc[0] = 0;
    for (size_t k = 0; k < nb; k++) hc[k + 1] = hc[k] + cnt[k];
    int* ho = (int*)(hc + nb + 1);
    cccs_longest_first(nb, h_beams, ho);
    char* b = (char*)batch;
    const float** aF = (const float**)b;
    float** aT = (float**)(b + nb * 8);
    float** aR = (float**)(b + 2 * nb * 8);
    float** aD = (float**)(b + 3 * nb * 8);
    const int* d_order = (const int*)(b + (5 * nb + 1) * 8);
    ColumnScratch pre;
    pre.cap_off = (uint64_t*)(b + 4 * nb * 8);
    pre.nnz = (uint32_t*)(b + o_nnz);
    pre.max = (float*)(b + o_max);
    pre.iscale = (float*)(b + o_isc);

    FD2_CHECK_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = [&]() -> int {
        FD2_CHECK_CUDA(cudaMemcpyAsync(batch, h, up_bytes, cudaMemcpyHostToDevice, st));
        FD2_CHECK_CUDA(cudaMemsetAsync(dD, 0, off[nb] * sizeof(float), st));
        FD2_TRY(launch_terma(ctx, P, nb, d_beams, aF, aT, aR, density, spectrum, 1, st));
        FD2_TRY(launch_cccs_host(ctx, nb, h_beams, d_beams, (const float* const*)aT, (const float* const*)aR, aD,
                                 kernel, schedule, st, d_order));
        return append_columns(e, d_infos, cnt, nb, (const float* const*)aD, density->vol, params.extent,
                              params.ss_factor, st, &pre);
    }();
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &g);  // the capture ends on every path
    if (rc || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        if (rc) return rc;
        FD2_CHECK_CUDA(ce);
    }
    const uint64_t key = (uint64_t)h_beams[0].fmap_size[0] | (uint64_t)h_beams[0].fmap_size[1] << 10 |
                         (uint64_t)kernel->n_phi << 20 | (uint64_t)kernel->n_theta << 28 | (uint64_t)schedule << 36 |
                         (uint64_t)params.value_type << 38 | (uint64_t)params.ss_factor << 40;
    cudaGraphExec_t ex = nullptr;
    auto it = ctx->graphs.find(key);
    if (it != ctx->graphs.end()) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(it->second, g, &info) == cudaSuccess) {
            ex = it->second;
            ctx->graph_updates++;
        } else {
            cudaGetLastError();  // a refused update is not an error: instantiate afresh
            cudaGraphExecDestroy(it->second);
            ctx->graphs.erase(it);
        }
    }
    cudaError_t err = cudaSuccess;
    if (!ex) {
        err = cudaGraphInstantiate(&ex, g, 0);
        if (err == cudaSuccess) {
            ctx->graphs[key] = ex;
            ctx->graph_instantiations++;
        }
    }
    cudaGraphDestroy(g);
    FD2_CHECK_CUDA(err);
    FD2_CHECK_CUDA(cudaGraphLaunch(ex, st));
    ctx->graph_launches++;
    FD2_CHECK_CUDA(cudaEventRecord(ctx->stage_free[slot], st));
    return FD2_OK;
}

// The host copy of a matrix under construction (fd2_dosemat_params_t.host_out).
// After the device work of batch k is enqueued, batch k-1's rows are copied
// to the caller's buffers on a copy stream, so the copy runs while the device
// computes batch k; only the last batch's copy follows the construction.  The
// size of a batch's nonzero range is read from its own row offsets, which go
// to the caller's row_off buffer first: the host waits for them (by then the
// device is busy with the next batch) and then issues the column and value
// copies of exactly that range.
struct HostSink {
    struct Batch {
        uint64_t row0 = 0, row1 = 0;
        cudaEvent_t offsets = nullptr;  // on the copy stream: the batch's row offsets are on the host
    };
    fd2_host_csr_t* out = nullptr;
    fd2_csr_ensemble* e = nullptr;
    cudaStream_t cs = nullptr;
    bool have_pending = false;
    Batch pending;

    int init(fd2_host_csr_t* o, fd2_csr_ensemble* ens) {
        FD2_REQUIRE(o->row_off && o->col && o->val, FD2_ERR_INVALID_ARGUMENT,
                    "dose_mat_construct: host_out needs row_off, col and val");
        FD2_REQUIRE(ens->value_type == FD2_VALUES_F32 || o->scale, FD2_ERR_INVALID_ARGUMENT,
                    "dose_mat_construct: host_out of a 16-bit matrix needs scale");
        out = o;
        e = ens;
        out->nnz = 0;
        out->row_off[0] = 0;
        FD2_CHECK_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        return FD2_OK;
    }
    // rows [row0, row1) are enqueued on st
    int batch_done(uint64_t row0, uint64_t row1, cudaStream_t st) {
        if (have_pending) FD2_TRY(flush());
        cudaEvent_t done = nullptr;
        FD2_CHECK_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        cudaError_t err = cudaEventRecord(done, st);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(cs, done, 0);
        cudaEventDestroy(done);  // released once it has completed
        FD2_CHECK_CUDA(err);
        FD2_CHECK_CUDA(cudaMemcpyAsync(out->row_off + row0 + 1, e->d_row_off + row0 + 1,
                                       (row1 - row0) * sizeof(int64_t), cudaMemcpyDeviceToHost, cs));
        pending = Batch{row0, row1, nullptr};
        FD2_CHECK_CUDA(cudaEventCreateWithFlags(&pending.offsets, cudaEventDisableTiming));
        have_pending = true;
        FD2_CHECK_CUDA(cudaEventRecord(pending.offsets, cs));
        return FD2_OK;
    }
    int flush() {
        have_pending = false;
        const Batch b = pending;
        cudaError_t err = cudaEventSynchronize(b.offsets);
        cudaEventDestroy(b.offsets);
        FD2_CHECK_CUDA(err);
        const uint64_t s0 = (uint64_t)out->row_off[b.row0], s1 = (uint64_t)out->row_off[b.row1];
        FD2_REQUIRE(s1 <= out->cap_nnz, FD2_ERR_CAPACITY,
                    "dose_mat_construct: host_out holds %llu nonzeros, the matrix has at least %llu",
                    (unsigned long long)out->cap_nnz, (unsigned long long)s1);
        const size_t vb = value_bytes(e->value_type);
        if (s1 > s0) {
            FD2_CHECK_CUDA(cudaMemcpyAsync(out->col + s0, e->d_col + s0, (s1 - s0) * sizeof(int32_t),
                                           cudaMemcpyDeviceToHost, cs));
            FD2_CHECK_CUDA(cudaMemcpyAsync((char*)out->val + s0 * vb, (const char*)e->d_val + s0 * vb,
                                           (s1 - s0) * vb, cudaMemcpyDeviceToHost, cs));
        }
        if (e->value_type != FD2_VALUES_F32 && b.row1 > b.row0)
            FD2_CHECK_CUDA(cudaMemcpyAsync(out->scale + b.row0, e->d_scale + b.row0, (b.row1 - b.row0) * sizeof(float),
                                           cudaMemcpyDeviceToHost, cs));
        out->nnz = s1;
        return FD2_OK;
    }
    int finish() {
        if (have_pending) FD2_TRY(flush());
        FD2_CHECK_CUDA(cudaStreamSynchronize(cs));
        return FD2_OK;
    }
    void drain() {
        if (cs) cudaStreamSynchronize(cs);
    }
    ~HostSink() {
        if (have_pending) cudaEventDestroy(pending.offsets);
        if (cs) {
            cudaStreamSynchronize(cs);  // no copy may outlive the ensemble's arrays
            cudaStreamDestroy(cs);
        }
    }
};

}  // namespace fd2

using namespace fd2;

extern "C" {

void fd2_dosemat_params_default(fd2_dosemat_params_t* p) {
    if (!p) return;
    p->extent = 2.0f;       // IMRTOpt/src/IMRTArgs.cpp:60
    p->ss_factor = 5;       // IMRTOpt/src/IMRTgeom.cu:352
    p->value_type = FD2_VALUES_F32;
    p->cccs_schedule = -1;
    p->batch_beamlets = 0;
    p->memory_budget = 0;
    p->verbose = 0;
    p->host_out = nullptr;
    p->graph = 0;
    p->overlap = 1;
}

int fd2_bev2pvcs(fd2_context* ctx, const fd2_beam_t* h_beam, const fd2_density* density, const float* d_bev,
                 float* d_out, size_t out_pitch_bytes, void* stream) {
    FD2_REQUIRE(ctx && h_beam && density && d_bev && d_out, FD2_ERR_INVALID_ARGUMENT, "bev2pvcs: null argument");
    FD2_REQUIRE(out_pitch_bytes >= density->vol.dim[0] * sizeof(float) && out_pitch_bytes % sizeof(float) == 0,
                FD2_ERR_INVALID_ARGUMENT, "bev2pvcs: bad pitch");
    ColumnInfo ci;
    make_column_info(*h_beam, nullptr, ci);
    return launch_bev2pvcs(ci, density->vol, d_bev, d_out, out_pitch_bytes / sizeof(float), 0, 0.0f,
                           (cudaStream_t)stream);
}

int fd2_bev2pvcs_supersampling(fd2_context* ctx, const fd2_beam_t* h_beam, const fd2_density* density,
                               const float* d_bev, float* d_out, size_t out_pitch_bytes, int ssfactor, float extent,
                               void* stream) {
    FD2_REQUIRE(ctx && h_beam && density && d_bev && d_out, FD2_ERR_INVALID_ARGUMENT, "bev2pvcs: null argument");
    FD2_REQUIRE(ssfactor > 0 && ssfactor <= 16, FD2_ERR_INVALID_ARGUMENT, "bev2pvcs: ssfactor %d", ssfactor);
    FD2_REQUIRE(out_pitch_bytes >= density->vol.dim[0] * sizeof(float) && out_pitch_bytes % sizeof(float) == 0,
                FD2_ERR_INVALID_ARGUMENT, "bev2pvcs: bad pitch");
    ColumnInfo ci;
    make_column_info(*h_beam, nullptr, ci);
    return launch_bev2pvcs(ci, density->vol, d_bev, d_out, out_pitch_bytes / sizeof(float), ssfactor, extent,
                           (cudaStream_t)stream);
}

int fd2_dose_mat_construct(fd2_context* ctx, size_t n_beams, const uint32_t* n_per_beam, const fd2_beam_t* h_beamlets,
                           const float* h_fluence, const fd2_density* density, const fd2_spectrum* spectrum,
                           const fd2_cccs_kernel* kernel, const fd2_dosemat_params_t* params_in,
                           fd2_csr_ensemble** out, void* stream) {
    FD2_REQUIRE(ctx && n_per_beam && h_beamlets && h_fluence && density && spectrum && kernel && out,
                FD2_ERR_INVALID_ARGUMENT, "dose_mat_construct: null argument");
    *out = nullptr;
    fd2_dosemat_params_t params;
    fd2_dosemat_params_default(&params);
    if (params_in) params = *params_in;
    FD2_REQUIRE(params.ss_factor > 0 && params.ss_factor <= 16, FD2_ERR_INVALID_ARGUMENT, "ss_factor out of range");
    FD2_REQUIRE(params.value_type >= 0 && params.value_type <= 2, FD2_ERR_INVALID_ARGUMENT, "bad value type");
    FD2_REQUIRE(params.cccs_schedule >= -2 && params.cccs_schedule <= 1, FD2_ERR_INVALID_ARGUMENT,
                "cccs_schedule %d (-2..1)", params.cccs_schedule);
    FD2_REQUIRE(params.graph == 0 || params.graph == 1, FD2_ERR_INVALID_ARGUMENT, "graph %d (0 or 1)", params.graph);
    FD2_REQUIRE(params.overlap == 0 || params.overlap == 1, FD2_ERR_INVALID_ARGUMENT, "overlap %d (0 or 1)",
                params.overlap);
    FD2_REQUIRE(!(params.graph && params.host_out), FD2_ERR_NOT_SUPPORTED,
                "dose_mat_construct: graph capture and host_out are exclusive");
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    const fd2_volume_t& vol = density->vol;
    const uint64_t nvox = (uint64_t)vol.dim[0] * vol.dim[1] * vol.dim[2];
    FD2_REQUIRE(nvox < (1ull << 31), FD2_ERR_NOT_SUPPORTED, "volume of %llu voxels exceeds int32 column indices",
                (unsigned long long)nvox);

    size_t total = 0;
    for (size_t i = 0; i < n_beams; i++) total += n_per_beam[i];
    const uint32_t fx = total ? h_beamlets[0].fmap_size[0] : 0, fy = total ? h_beamlets[0].fmap_size[1] : 0;
    const size_t P = (size_t)fx * fy;
    std::vector<fd2_beam_t> beams(h_beamlets, h_beamlets + total);
    for (auto& b : beams) {
        FD2_REQUIRE(b.fmap_size[0] == fx && b.fmap_size[1] == fy, FD2_ERR_INVALID_ARGUMENT,
                    "dose_mat_construct: beamlets must share one fluence-map size");
        FD2_REQUIRE(b.long_dim > 0 && b.sad > 0 && b.long_spacing > 0, FD2_ERR_INVALID_ARGUMENT,
                    "dose_mat_construct: beamlet without a depth range (run calc_range)");
        b.TermaBEV_pitch = b.DensityBEV_pitch = P * sizeof(float);
    }
    FD2_REQUIRE(P > 0 || total == 0, FD2_ERR_INVALID_ARGUMENT, "empty fluence map");
    FD2_REQUIRE(P <= 1024, FD2_ERR_NOT_SUPPORTED, "fluence map of %zu pixels (max 1024)", P);

    auto* e = new fd2_csr_ensemble();
    e->ctx = ctx;
    e->stream = st;
    e->verbose = params.verbose != 0;
    e->n_cols = nvox;
    e->value_type = params.value_type;
    e->mat_rows.assign(1, 0);
    // Column geometry and candidate counts of every beamlet, before the first
    // column stage: their sum bounds the matrix, which is then allocated once.
    // The geometry goes up and the counts run on stream `s`; the reservation
    // is enqueued on st.  With the column stage overlapped this runs after the
    // first batch's Terma and CCCS are enqueued, on the column stream, so the
    // host work and the count kernel hide behind that batch's march.
    std::vector<ColumnInfo> infos;
    ColumnInfo* d_infos = nullptr;
    std::vector<uint32_t> cnt;
    HostSink sink;  // declared before the ensemble is destroyed on any path: its copies finish first
    bool columns_ready = false;
    auto setup_columns = [&](cudaStream_t s) -> int {
        columns_ready = true;
        infos.resize(total);
        for (size_t k = 0; k < total; k++) make_column_info(beams[k], &vol, infos[k]);
        FD2_TRY(upload(infos, &d_infos, ctx->pool, s));
        FD2_TRY(column_counts(ctx, d_infos, total, vol, params.extent, s, cnt));
        uint64_t cap_total = 0;
        for (uint32_t c : cnt) cap_total += c;
        FD2_TRY(ensemble_reserve(e, total, cap_total));
        if (params.host_out) FD2_TRY(sink.init(params.host_out, e));
        return FD2_OK;
    };
    const bool overlap = params.overlap && !params.graph;
    int rc = overlap ? FD2_OK : setup_columns(st);
    if (rc) {
        if (d_infos) cudaFreeAsync(d_infos, st);
        fd2_csr_ensemble_destroy(e);
        return rc;
    }

    // memory budget for the BEV buffers of one batch (a fixed share of the
    // device, so the batches and buffer sizes repeat from plan to plan)
    size_t free_b = 0, tot_b = 0;
    cudaMemGetInfo(&free_b, &tot_b);
    size_t budget = params.memory_budget ? params.memory_budget : std::min<size_t>(tot_b / 10, (size_t)16 << 30);

    float* d_fluence = nullptr;
    fd2_beam_t* d_beams = nullptr;
    rc = upload(std::vector<float>(h_fluence, h_fluence + P), &d_fluence, ctx->pool, st);
    if (!rc) rc = upload(beams, &d_beams, ctx->pool, st);

    // batches of about equal size: as many as the budget needs, whole beams
    // each, so no batch is a small remainder (a launch of a few waves spends
    // proportionally more of its time in its tail)
    {
        size_t all = 0;
        for (const auto& b : beams) all += (size_t)b.long_dim * P * 3 * sizeof(float);
        const size_t n_batches = std::max<size_t>(1, (all + budget - 1) / std::max<size_t>(budget, 1));
        budget = std::min(budget, (all + n_batches - 1) / n_batches + (size_t)1);
    }
    // Column stage beside the next batch (params.overlap, direct launches):
    // batch i fills BEV slot i % 2 on st; its column stage waits for the
    // batch's CCCS and runs on the context's second stream (cs) while st goes
    // on with batch i + 1 in the other slot; before batch i + 2 reuses a slot,
    // st waits for the column stage that read it.
    cudaStream_t cs = st;
    cudaEvent_t ev_ready = nullptr, ev_slot[2] = {nullptr, nullptr};
    bool slot_used[2] = {false, false};
    if (!rc && overlap) {
        if (!ctx->aux_stream && cudaStreamCreateWithFlags(&ctx->aux_stream, cudaStreamNonBlocking) != cudaSuccess) {
            ctx->aux_stream = nullptr;
            set_error("dose_mat_construct: cannot create the column stream");
            rc = FD2_ERR_CUDA;
        }
        for (cudaEvent_t* ev : {&ev_ready, &ev_slot[0], &ev_slot[1]})
            if (!rc && cudaEventCreateWithFlags(ev, cudaEventDisableTiming) != cudaSuccess) {
                set_error("dose_mat_construct: cannot create events");
                rc = FD2_ERR_CUDA;
            }
        if (!rc) cs = ctx->aux_stream;
        // the column stream starts after everything enqueued on st so far
        // (the fluence and beamlet uploads)
        if (!rc && (cudaEventRecord(ev_ready, st) != cudaSuccess || cudaStreamWaitEvent(cs, ev_ready, 0) != cudaSuccess)) {
            set_error("dose_mat_construct: cannot order the column stream");
            rc = FD2_ERR_CUDA;
        }
    }
    size_t n_batch = 0;
    size_t b0 = 0, beam0 = 0;
    const auto t_start = std::chrono::steady_clock::now();
    auto ms_since = [&](std::chrono::steady_clock::time_point t) {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
    };
    while (!rc && beam0 < n_beams) {
        // whole beams into the batch while the scratch fits
        size_t beam1 = beam0, b1 = b0, bytes = 0;
        while (beam1 < n_beams) {
            size_t add = 0;
            for (size_t k = b1; k < b1 + n_per_beam[beam1]; k++) add += (size_t)beams[k].long_dim * P * 3 * sizeof(float);
            size_t cnt = b1 + n_per_beam[beam1] - b0;
            if (beam1 > beam0 && (bytes + add > budget || (params.batch_beamlets && cnt > params.batch_beamlets))) break;
            bytes += add;
            b1 += n_per_beam[beam1];
            beam1++;
        }
        const size_t nb = b1 - b0;
        if (nb == 0) {  // beams without beamlets
            for (size_t i = beam0; i < beam1; i++) e->mat_rows.push_back(e->n_rows);
            beam0 = beam1;
            continue;
        }
        // BEV buffers [beamlet][L][P] for Terma, density, dose
        std::vector<size_t> off(nb + 1, 0);
        for (size_t k = 0; k < nb; k++) off[k + 1] = off[k] + (size_t)beams[b0 + k].long_dim * P;
        const int slot = overlap ? (int)(n_batch & 1) : 0;
        n_batch++;
        if (overlap && slot_used[slot] && cudaStreamWaitEvent(st, ev_slot[slot], 0) != cudaSuccess) {
            set_error("dose_mat_construct: cannot order the BEV buffer reuse");
            rc = FD2_ERR_CUDA;
            break;
        }
        float* d_bev = nullptr;
        rc = ctx_buffer(ctx, slot ? kBufBev2 : kBufBev, off[nb] * 3 * sizeof(float), st, (void**)&d_bev);
        if (rc) break;
        float *dT = d_bev, *dR = d_bev + off[nb], *dD = d_bev + 2 * off[nb];
        if (params.graph) {
            const int sched = params.cccs_schedule >= 0 ? params.cccs_schedule : cccs_auto_schedule(ctx, nb);
            rc = graph_batch(ctx, e, nb, beams.data() + b0, d_beams + b0, d_infos + b0, cnt.data() + b0, d_fluence,
                             dT, dR, dD, off.data(), P, density, spectrum, kernel, params, sched, st);
            if (rc) break;
            size_t row = e->n_rows - nb;
            for (size_t i = beam0; i < beam1; i++) {
                row += n_per_beam[i];
                e->mat_rows.push_back(row);
            }
            b0 = b1;
            beam0 = beam1;
            continue;
        }
        std::vector<const float*> hF(nb, d_fluence);
        std::vector<float*> hT(nb), hR(nb), hD(nb);
        for (size_t k = 0; k < nb; k++) { hT[k] = dT + off[k]; hR[k] = dR + off[k]; hD[k] = dD + off[k]; }
        const float** aF = nullptr;
        float **aT = nullptr, **aR = nullptr, **aD = nullptr;
        int* d_order = nullptr;
        std::vector<int> order(nb);
        cccs_longest_first(nb, beams.data() + b0, order.data());
        rc = [&]() -> int {
            FD2_TRY(upload(order, &d_order, ctx->pool, st));
            FD2_TRY(upload(hF, &aF, ctx->pool, st));
            FD2_TRY(upload(hT, &aT, ctx->pool, st));
            FD2_TRY(upload(hR, &aR, ctx->pool, st));
            FD2_TRY(upload(hD, &aD, ctx->pool, st));
            FD2_CHECK_CUDA(cudaMemsetAsync(dD, 0, off[nb] * sizeof(float), st));
            {
                StageTimer t(ctx, st, FD2_STAGE_TERMA);
                FD2_TRY(launch_terma(ctx, P, nb, d_beams + b0, aF, aT, aR, density, spectrum, 1, st));
                t.stop();
            }
            {
                StageTimer t(ctx, st, FD2_STAGE_CCCS);
                auto run = [&](int sched) {
                    return launch_cccs_host(ctx, nb, beams.data() + b0, d_beams + b0, (const float* const*)aT,
                                            (const float* const*)aR, aD, kernel, sched, st, d_order);
                };
                if (params.cccs_schedule >= 0) {
                    FD2_TRY(run(params.cccs_schedule));
                } else if (params.cccs_schedule == -2) {
                    FD2_TRY(run(cccs_auto_schedule(ctx, nb)));
                } else {
                    FD2_TRY(tuned_cccs(ctx, nb, P, kernel, st, run, dD, off[nb]));
                }
                t.stop();
            }
            if (overlap) {
                if (!columns_ready) FD2_TRY(setup_columns(cs));
                FD2_CHECK_CUDA(cudaEventRecord(ev_ready, st));
                FD2_CHECK_CUDA(cudaStreamWaitEvent(cs, ev_ready, 0));
            }
            StageTimer t(ctx, cs, FD2_STAGE_COLUMNS);
            int r = append_columns(e, d_infos + b0, cnt.data() + b0, nb, (const float* const*)aD, vol,
                                   params.extent, params.ss_factor, cs);
            t.stop();
            return r;
        }();
        // release batch buffers: the dose pointer table after the column stage
        // that reads it (on cs), the others after the CCCS (on st); a failed
        // batch drains both streams first
        if (rc && overlap) {
            cudaStreamSynchronize(st);
            cudaStreamSynchronize(cs);
        }
        for (void* p : {(void*)aF, (void*)aT, (void*)aR, (void*)d_order})  // d_bev is the context's
            if (p) cudaFreeAsync(p, st);
        if (aD) cudaFreeAsync(aD, cs);
        if (rc) break;
        if (overlap) {
            if (cudaEventRecord(ev_slot[slot], cs) != cudaSuccess) {
                set_error("dose_mat_construct: cannot record the column stage");
                rc = FD2_ERR_CUDA;
                break;
            }
            slot_used[slot] = true;
        }
        if (params.host_out) {
            rc = sink.batch_done(e->n_rows - nb, e->n_rows, cs);
            if (rc) break;
        }
        // per-beam row boundaries
        size_t row = e->n_rows - nb;
        for (size_t i = beam0; i < beam1; i++) {
            row += n_per_beam[i];
            e->mat_rows.push_back(row);
        }
        if (params.verbose)
            std::printf("dose matrix batch: beams %zu..%zu, %zu beamlets, nnz bound %llu, host %.1f ms since start\n",
                        beam0, beam1 - 1, nb, (unsigned long long)e->nnz_bound, ms_since(t_start));
        b0 = b1;
        beam0 = beam1;
    }
    // a plan without beamlets still gets its (empty) matrix
    if (!rc && !columns_ready) rc = setup_columns(st);
    if (overlap && cs != st) {
        // st resumes after the last column stage; on an error path the host
        // waits for the column stream instead
        if (cudaEventRecord(ev_ready, cs) != cudaSuccess || cudaStreamWaitEvent(st, ev_ready, 0) != cudaSuccess) {
            cudaStreamSynchronize(cs);
            if (!rc) {
                set_error("dose_mat_construct: cannot join the column stream");
                rc = FD2_ERR_CUDA;
            }
        }
    }
    if (d_fluence) cudaFreeAsync(d_fluence, st);
    if (d_beams) cudaFreeAsync(d_beams, st);
    if (d_infos) cudaFreeAsync(d_infos, st);
    if (!rc) rc = ensemble_sync_nnz(e);  // the one wait of the construction, besides the candidate counts
    cudaStreamSynchronize(st);
    for (cudaEvent_t ev : {ev_ready, ev_slot[0], ev_slot[1]})
        if (ev) cudaEventDestroy(ev);
    if (!rc && params.host_out) rc = sink.finish();
    if (!rc) {
        fd2::DeviceStatus ds;
        if (cudaMemcpy(&ds, ctx->d_status, sizeof(ds), cudaMemcpyDeviceToHost) == cudaSuccess && ds.code != 0) {
            cudaMemset(ctx->d_status, 0, sizeof(ds));
            set_error("dose_mat_construct: a CCCS ray march hit its step cap");
            rc = FD2_ERR_WATCHDOG;
        }
    }
    if (rc) {
        sink.drain();  // copies still reading the ensemble end before its arrays are freed
        fd2_csr_ensemble_destroy(e);
        return rc;
    }
    *out = e;
    return FD2_OK;
}

int fd2_bev2pvcs_interp(fd2_context* ctx, size_t n_beams, const uint32_t* n_per_beam, const fd2_beam_t* h_beamlets,
                        const float* const* d_dose_bev, const fd2_density* density,
                        const fd2_dosemat_params_t* params_in, fd2_csr_ensemble** out, void* stream) {
    FD2_REQUIRE(ctx && n_per_beam && h_beamlets && d_dose_bev && density && out, FD2_ERR_INVALID_ARGUMENT,
                "bev2pvcs_interp: null argument");
    *out = nullptr;
    fd2_dosemat_params_t params;
    fd2_dosemat_params_default(&params);
    if (params_in) params = *params_in;
    FD2_REQUIRE(params.ss_factor > 0 && params.ss_factor <= 16, FD2_ERR_INVALID_ARGUMENT, "ss_factor out of range");
    FD2_REQUIRE(params.value_type >= 0 && params.value_type <= 2, FD2_ERR_INVALID_ARGUMENT, "bad value type");
    const fd2_volume_t& vol = density->vol;
    const uint64_t nvox = (uint64_t)vol.dim[0] * vol.dim[1] * vol.dim[2];
    FD2_REQUIRE(nvox < (1ull << 31), FD2_ERR_NOT_SUPPORTED, "volume exceeds int32 column indices");
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    auto* e = new fd2_csr_ensemble();
    e->ctx = ctx;
    e->stream = st;
    e->verbose = params.verbose != 0;
    e->n_cols = nvox;
    e->value_type = params.value_type;
    e->mat_rows.assign(1, 0);
    int rc = ensemble_reserve(e, 0, 0);
    size_t b0 = 0;
    for (size_t i = 0; !rc && i < n_beams; i++) {
        const size_t nb = n_per_beam[i];
        if (nb) {
            std::vector<ColumnInfo> infos(nb);
            for (size_t k = 0; k < nb; k++) make_column_info(h_beamlets[b0 + k], &vol, infos[k]);
            ColumnInfo* d_infos = nullptr;
            std::vector<uint32_t> cnt;
            rc = upload(infos, &d_infos, ctx->pool, st);
            if (!rc) rc = column_counts(ctx, d_infos, nb, vol, params.extent, st, cnt);
            if (!rc) rc = append_columns(e, d_infos, cnt.data(), nb, d_dose_bev + b0, vol, params.extent,
                                         params.ss_factor, st);
            if (d_infos) cudaFreeAsync(d_infos, st);
        }
        b0 += nb;
        e->mat_rows.push_back(e->n_rows);
    }
    if (!rc) rc = ensemble_sync_nnz(e);
    if (rc) {
        fd2_csr_ensemble_destroy(e);
        return rc;
    }
    *out = e;
    return FD2_OK;
}

int fd2_csr_ensemble_concat(fd2_context* ctx, size_t n, const fd2_csr_ensemble* const* parts,
                            fd2_csr_ensemble** out) {
    FD2_REQUIRE(ctx && parts && out && n > 0, FD2_ERR_INVALID_ARGUMENT, "ensemble_concat: bad argument");
    uint64_t rows = 0, nnz = 0;
    for (size_t i = 0; i < n; i++) {
        FD2_REQUIRE(parts[i], FD2_ERR_INVALID_ARGUMENT, "ensemble_concat: part %zu is null", i);
        FD2_REQUIRE(parts[i]->n_cols == parts[0]->n_cols && parts[i]->value_type == parts[0]->value_type,
                    FD2_ERR_INVALID_ARGUMENT, "ensemble_concat: part %zu has another column count or value type", i);
        rows += parts[i]->n_rows;
        nnz += parts[i]->nnz;
    }
    *out = nullptr;
    auto* e = new fd2_csr_ensemble();
    e->ctx = ctx;
    e->stream = ctx->stream;
    e->n_cols = parts[0]->n_cols;
    e->value_type = parts[0]->value_type;
    e->mat_rows.assign(1, 0);
    int rc = ensemble_reserve(e, rows, nnz);
    cudaStream_t st = e->stream;
    const size_t vb = value_bytes(e->value_type);
    uint64_t r0 = 0, k0 = 0;
    for (size_t i = 0; i < n && !rc; i++) {
        const fd2_csr_ensemble* p = parts[i];
        // the part's own stream has finished writing it
        if (cudaStreamSynchronize(p->stream) != cudaSuccess) rc = FD2_ERR_CUDA;
        if (!rc && p->n_rows) {
            if (launch_offsets_shift(p->d_row_off + 1, p->n_rows, (int64_t)k0, e->d_row_off + r0 + 1, st) != FD2_OK)
                rc = FD2_ERR_CUDA;
            if (!rc && e->d_scale &&
                cudaMemcpyAsync(e->d_scale + r0, p->d_scale, p->n_rows * sizeof(float), cudaMemcpyDeviceToDevice,
                                st) != cudaSuccess)
                rc = FD2_ERR_CUDA;
        }
        if (!rc && p->nnz &&
            (cudaMemcpyAsync(e->d_col + k0, p->d_col, p->nnz * sizeof(int32_t), cudaMemcpyDeviceToDevice, st) !=
                 cudaSuccess ||
             cudaMemcpyAsync((char*)e->d_val + k0 * vb, p->d_val, p->nnz * vb, cudaMemcpyDeviceToDevice, st) !=
                 cudaSuccess))
            rc = FD2_ERR_CUDA;
        for (size_t m = 1; m < p->mat_rows.size() && !rc; m++) e->mat_rows.push_back(r0 + p->mat_rows[m]);
        r0 += p->n_rows;
        k0 += p->nnz;
    }
    if (!rc) {
        e->n_rows = rows;
        e->nnz = e->nnz_bound = nnz;
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = FD2_ERR_CUDA;
    }
    if (rc) {
        if (rc == FD2_ERR_CUDA) set_error("ensemble_concat: %s", cudaGetErrorString(cudaGetLastError()));
        fd2_csr_ensemble_destroy(e);
        return rc;
    }
    *out = e;
    return FD2_OK;
}

int fd2_csr_ensemble_info(const fd2_csr_ensemble* e, fd2_csr_info_t* info) {
    FD2_REQUIRE(e && info, FD2_ERR_INVALID_ARGUMENT, "ensemble_info: null argument");
    info->n_mats = e->mat_rows.size() - 1;
    info->n_rows = e->n_rows;
    info->n_cols = e->n_cols;
    info->nnz = e->nnz;
    info->value_type = e->value_type;
    return FD2_OK;
}

int fd2_csr_ensemble_device(const fd2_csr_ensemble* e, const int64_t** row_offsets, const int32_t** columns,
                            const void** values, const float** row_scale, const uint64_t** mat_rows_host) {
    FD2_REQUIRE(e, FD2_ERR_INVALID_ARGUMENT, "ensemble_device: null ensemble");
    if (row_offsets) *row_offsets = e->d_row_off;
    if (columns) *columns = e->d_col;
    if (values) *values = e->d_val;
    if (row_scale) *row_scale = e->d_scale;
    if (mat_rows_host) *mat_rows_host = e->mat_rows.data();
    return FD2_OK;
}

int fd2_csr_ensemble_to_host(const fd2_csr_ensemble* e, int64_t* row_offsets, int32_t* columns, float* values) {
    FD2_REQUIRE(e, FD2_ERR_INVALID_ARGUMENT, "ensemble_to_host: null ensemble");
    FD2_CHECK_CUDA(cudaStreamSynchronize(e->stream));
    if (row_offsets)
        FD2_CHECK_CUDA(cudaMemcpy(row_offsets, e->d_row_off, (e->n_rows + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost));
    if (columns && e->nnz)
        FD2_CHECK_CUDA(cudaMemcpy(columns, e->d_col, e->nnz * sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (values && e->nnz) {
        if (e->value_type == FD2_VALUES_F32) {
            FD2_CHECK_CUDA(cudaMemcpy(values, e->d_val, e->nnz * sizeof(float), cudaMemcpyDeviceToHost));
        } else {
            std::vector<uint16_t> raw(e->nnz);
            std::vector<float> sc(e->n_rows);
            std::vector<int64_t> ro(e->n_rows + 1);
            FD2_CHECK_CUDA(cudaMemcpy(raw.data(), e->d_val, e->nnz * 2, cudaMemcpyDeviceToHost));
            FD2_CHECK_CUDA(cudaMemcpy(sc.data(), e->d_scale, e->n_rows * sizeof(float), cudaMemcpyDeviceToHost));
            FD2_CHECK_CUDA(cudaMemcpy(ro.data(), e->d_row_off, (e->n_rows + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost));
            for (uint64_t r = 0; r < e->n_rows; r++)
                for (int64_t k = ro[r]; k < ro[r + 1]; k++) {
                    float v;
                    if (e->value_type == FD2_VALUES_F16) {
                        __half h;
                        std::memcpy(&h, &raw[k], 2);
                        v = __half2float(h);
                    } else {
                        uint32_t bits = (uint32_t)raw[k] << 16;
                        std::memcpy(&v, &bits, 4);
                    }
                    values[k] = v * sc[r];
                }
        }
    }
    return FD2_OK;
}

static int write_file(const std::string& path, const void* data, size_t bytes) {
    std::ofstream f(path, std::ios::binary);
    FD2_REQUIRE(f.is_open(), FD2_ERR_IO, "cannot open %s", path.c_str());
    f.write((const char*)data, (std::streamsize)bytes);
    FD2_REQUIRE(f.good(), FD2_ERR_IO, "write failed: %s", path.c_str());
    return FD2_OK;
}

// 16-bit sidecar files beside the reference's layout (valuesBuffer.bin stays
// float32 with the scales applied, for the reference's readers)
static std::string sidecar_values(int vt) { return vt == FD2_VALUES_F16 ? "/valuesBuffer.f16.bin" : "/valuesBuffer.bf16.bin"; }
static std::string sidecar_scales(int vt) { return vt == FD2_VALUES_F16 ? "/rowScales.f16.bin" : "/rowScales.bf16.bin"; }

static int read_file(const std::string& path, std::vector<char>& out) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    FD2_REQUIRE(f.is_open(), FD2_ERR_IO, "cannot open %s", path.c_str());
    std::streamsize n = f.tellg();
    f.seekg(0);
    out.resize((size_t)n);
    f.read(out.data(), n);
    FD2_REQUIRE(f.good() || n == 0, FD2_ERR_IO, "read failed: %s", path.c_str());
    return FD2_OK;
}

// 64-bit voxel indices of a doseMatFolder to the ensemble's int32 columns;
// an index outside the volume sets *bad.
__global__ void columns_from_file_kernel(const uint64_t* __restrict__ in, int32_t* __restrict__ out, size_t n,
                                         uint64_t n_cols, unsigned int* __restrict__ bad) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint64_t c = in[i];
        if (c >= n_cols) {
            atomicOr(bad, 1u);
            out[i] = 0;
        } else {
            out[i] = (int32_t)c;
        }
    }
}

// columnsBuffer.bin and the values file streamed to the device in chunks:
// while the device converts and stores chunk i (from a pinned buffer), the
// host reads chunk i + 1 into the other one.  Host memory stays at two chunks,
// whatever the matrix.
static int stream_columns(fd2_context* ctx, const std::string& col_path, const std::string& val_path, uint64_t nnz,
                          size_t vb, uint64_t n_cols, int32_t* d_col, void* d_val, cudaStream_t st) {
    constexpr size_t kChunk = (size_t)4 << 20;  // nonzeros per chunk: 32 MB of 64-bit columns
    struct Res {
        FILE* fc = nullptr;
        FILE* fv = nullptr;
        void* h[4] = {nullptr, nullptr, nullptr, nullptr};  // columns 0/1, values 0/1 (pinned)
        void* d_c64[2] = {nullptr, nullptr};
        unsigned int* d_bad = nullptr;
        cudaEvent_t ev[2] = {nullptr, nullptr};
        cudaStream_t st = nullptr;
        ~Res() {
            if (st) cudaStreamSynchronize(st);  // no copy still reads the pinned buffers
            if (fc) fclose(fc);
            if (fv) fclose(fv);
            for (void* p : h)
                if (p) cudaFreeHost(p);
            for (void* p : d_c64)
                if (p) cudaFreeAsync(p, st);
            if (d_bad) cudaFreeAsync(d_bad, st);
            for (cudaEvent_t e : ev)
                if (e) cudaEventDestroy(e);
        }
    } res;
    if (nnz == 0) return FD2_OK;
    res.st = st;
    res.fc = fopen(col_path.c_str(), "rb");
    res.fv = fopen(val_path.c_str(), "rb");
    FD2_REQUIRE(res.fc && res.fv, FD2_ERR_IO, "fromfile: cannot open %s or %s", col_path.c_str(), val_path.c_str());
    const size_t chunk = std::min<size_t>(kChunk, nnz);
    for (int b = 0; b < 2; b++) {
        FD2_CHECK_CUDA(cudaHostAlloc(&res.h[b], chunk * 8, cudaHostAllocDefault));
        FD2_CHECK_CUDA(cudaHostAlloc(&res.h[2 + b], chunk * vb, cudaHostAllocDefault));
        FD2_CHECK_CUDA(cudaMallocFromPoolAsync(&res.d_c64[b], chunk * 8, ctx->pool, st));
        FD2_CHECK_CUDA(cudaEventCreateWithFlags(&res.ev[b], cudaEventDisableTiming));
    }
    FD2_CHECK_CUDA(cudaMallocFromPoolAsync((void**)&res.d_bad, sizeof(unsigned int), ctx->pool, st));
    FD2_CHECK_CUDA(cudaMemsetAsync(res.d_bad, 0, sizeof(unsigned int), st));
    for (uint64_t k0 = 0, i = 0; k0 < nnz; k0 += chunk, i++) {
        const int b = (int)(i & 1);
        const size_t n = (size_t)std::min<uint64_t>(chunk, nnz - k0);
        if (i >= 2) FD2_CHECK_CUDA(cudaEventSynchronize(res.ev[b]));  // buffer b's last copies are done
        FD2_REQUIRE(fread(res.h[b], 8, n, res.fc) == n && fread(res.h[2 + b], vb, n, res.fv) == n, FD2_ERR_IO,
                    "fromfile: short read at nonzero %llu", (unsigned long long)k0);
        FD2_CHECK_CUDA(cudaMemcpyAsync(res.d_c64[b], res.h[b], n * 8, cudaMemcpyHostToDevice, st));
        const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->sm_count * 8);
        columns_from_file_kernel<<<blocks, 256, 0, st>>>((const uint64_t*)res.d_c64[b], d_col + k0, n, n_cols,
                                                         res.d_bad);
        FD2_CHECK_CUDA(cudaGetLastError());
        FD2_CHECK_CUDA(cudaMemcpyAsync((char*)d_val + k0 * vb, res.h[2 + b], n * vb, cudaMemcpyHostToDevice, st));
        FD2_CHECK_CUDA(cudaEventRecord(res.ev[b], st));
    }
    unsigned int bad = 0;
    FD2_CHECK_CUDA(cudaMemcpyAsync(&bad, res.d_bad, sizeof(bad), cudaMemcpyDeviceToHost, st));
    FD2_CHECK_CUDA(cudaStreamSynchronize(st));
    FD2_REQUIRE(!bad, FD2_ERR_IO, "fromfile: a column index is outside the %llu-voxel volume",
                (unsigned long long)n_cols);
    return FD2_OK;
}

int fd2_csr_ensemble_tofile(const fd2_csr_ensemble* e, const char* folder) {
    FD2_REQUIRE(e && folder, FD2_ERR_INVALID_ARGUMENT, "tofile: null argument");
    FD2_CHECK_CUDA(cudaStreamSynchronize(e->stream));
    mkdir(folder, 0755);
    const std::string dir(folder);
    const size_t nm = e->mat_rows.size() - 1;
    std::vector<int64_t> ro(e->n_rows + 1);
    FD2_CHECK_CUDA(cudaMemcpy(ro.data(), e->d_row_off, ro.size() * sizeof(int64_t), cudaMemcpyDeviceToHost));
    std::vector<uint64_t> nnz(nm), cnnz(nm), nrows(nm), cnrows(nm), obi(nm);
    std::vector<uint64_t> offsets;
    offsets.reserve(e->n_rows + nm);
    uint64_t obuf = 0;
    for (size_t m = 0; m < nm; m++) {
        uint64_t r0 = e->mat_rows[m], r1 = e->mat_rows[m + 1];
        nnz[m] = (uint64_t)(ro[r1] - ro[r0]);
        cnnz[m] = (m ? cnnz[m - 1] : 0) + nnz[m];
        nrows[m] = r1 - r0;
        cnrows[m] = (m ? cnrows[m - 1] : 0) + nrows[m];
        obi[m] = obuf;
        obuf += nrows[m] + 1;
        for (uint64_t r = r0; r <= r1; r++) offsets.push_back((uint64_t)(ro[r] - ro[r0]));  // local offsets
    }
    FD2_TRY(write_file(dir + "/NonZeroElements.bin", nnz.data(), nm * 8));
    FD2_TRY(write_file(dir + "/CumuNonZeroElements.bin", cnnz.data(), nm * 8));
    FD2_TRY(write_file(dir + "/numRowsPerMat.bin", nrows.data(), nm * 8));
    FD2_TRY(write_file(dir + "/CumuNumRowsPerMat.bin", cnrows.data(), nm * 8));
    FD2_TRY(write_file(dir + "/OffsetBufferIdx.bin", obi.data(), nm * 8));
    FD2_TRY(write_file(dir + "/offsetsBuffer.bin", offsets.data(), offsets.size() * 8));
    std::vector<int32_t> col(e->nnz);
    std::vector<float> val(e->nnz);
    FD2_TRY(fd2_csr_ensemble_to_host(e, nullptr, col.data(), val.data()));
    std::vector<uint64_t> col64(col.begin(), col.end());
    FD2_TRY(write_file(dir + "/columnsBuffer.bin", col64.data(), col64.size() * 8));
    FD2_TRY(write_file(dir + "/valuesBuffer.bin", val.data(), val.size() * 4));
    if (e->value_type != FD2_VALUES_F32) {
        // sidecars of a 16-bit ensemble: its stored values and row scales, so that
        // a 16-bit load reads half the value bytes and reproduces the same bits
        std::vector<uint16_t> raw(e->nnz);
        std::vector<float> scale(e->n_rows);
        if (e->nnz) FD2_CHECK_CUDA(cudaMemcpy(raw.data(), e->d_val, e->nnz * 2, cudaMemcpyDeviceToHost));
        if (e->n_rows) FD2_CHECK_CUDA(cudaMemcpy(scale.data(), e->d_scale, e->n_rows * 4, cudaMemcpyDeviceToHost));
        FD2_TRY(write_file(dir + sidecar_values(e->value_type), raw.data(), raw.size() * 2));
        FD2_TRY(write_file(dir + sidecar_scales(e->value_type), scale.data(), scale.size() * 4));
    }
    return FD2_OK;
}

int fd2_csr_ensemble_fromfile(fd2_context* ctx, const char* folder, uint64_t n_cols, int value_type,
                              fd2_csr_ensemble** out) {
    FD2_REQUIRE(ctx && folder && out, FD2_ERR_INVALID_ARGUMENT, "fromfile: null argument");
    FD2_REQUIRE(value_type >= FD2_VALUES_F32 && value_type <= FD2_VALUES_BF16, FD2_ERR_INVALID_ARGUMENT,
                "fromfile: value type %d", value_type);
    // columns are held as int32 on the device: a volume of 2^31 voxels or more
    // would let an index pass the range check and wrap negative
    FD2_REQUIRE(n_cols <= (uint64_t)INT32_MAX, FD2_ERR_INVALID_ARGUMENT,
                "fromfile: a %llu-voxel volume exceeds the int32 column range", (unsigned long long)n_cols);
    *out = nullptr;
    const std::string dir(folder);
    const bool half = value_type != FD2_VALUES_F32;
    const size_t vb = half ? 2 : 4;
    // the per-matrix tables and the row offsets are small: read whole
    std::vector<char> b_nrows, b_off, b_nnz, b_scale;
    FD2_TRY(read_file(dir + "/numRowsPerMat.bin", b_nrows));
    FD2_TRY(read_file(dir + "/NonZeroElements.bin", b_nnz));
    FD2_TRY(read_file(dir + "/offsetsBuffer.bin", b_off));
    std::string val_path = dir + "/valuesBuffer.bin";
    if (half) {
        // a 16-bit ensemble loads from the sidecars its tofile wrote; folders from
        // the reference (float32 only) load as F32 and are rounded by the VOI step
        FD2_REQUIRE(std::ifstream(dir + sidecar_values(value_type)).good(), FD2_ERR_NOT_SUPPORTED,
                    "fromfile: %s has no %s sidecar; load F32 and restrict with a 16-bit value type", folder,
                    sidecar_values(value_type).c_str() + 1);
        val_path = dir + sidecar_values(value_type);
        FD2_TRY(read_file(dir + sidecar_scales(value_type), b_scale));
    }
    const size_t nm = b_nrows.size() / 8;
    FD2_REQUIRE(b_nnz.size() / 8 == nm, FD2_ERR_IO, "fromfile: NonZeroElements.bin has %zu entries, expected %zu",
                b_nnz.size() / 8, nm);
    const uint64_t* nrows = (const uint64_t*)b_nrows.data();
    const uint64_t* off = (const uint64_t*)b_off.data();
    const uint64_t* mnnz = (const uint64_t*)b_nnz.data();
    uint64_t total_rows = 0, nnz = 0;
    for (size_t m = 0; m < nm; m++) { total_rows += nrows[m]; nnz += mnnz[m]; }
    struct stat sc{}, sv{};
    const std::string col_path = dir + "/columnsBuffer.bin";
    FD2_REQUIRE(stat(col_path.c_str(), &sc) == 0 && stat(val_path.c_str(), &sv) == 0, FD2_ERR_IO,
                "fromfile: cannot stat the columns or values of %s", folder);
    FD2_REQUIRE((uint64_t)sc.st_size == nnz * 8, FD2_ERR_IO, "fromfile: nnz mismatch");
    FD2_REQUIRE((uint64_t)sv.st_size == nnz * vb, FD2_ERR_IO, "fromfile: values/columns size mismatch");
    FD2_REQUIRE(b_off.size() / 8 == total_rows + nm, FD2_ERR_IO, "fromfile: offsetsBuffer size mismatch");
    FD2_REQUIRE(!half || b_scale.size() / 4 == total_rows, FD2_ERR_IO, "fromfile: row scales size mismatch");
    std::vector<int64_t> ro(total_rows + 1, 0);
    std::vector<uint64_t> mat_rows(1, 0);
    size_t ob = 0, r = 0;
    int64_t base = 0;
    for (size_t m = 0; m < nm; m++) {
        FD2_REQUIRE(off[ob] == 0 && off[ob + nrows[m]] == mnnz[m], FD2_ERR_IO, "fromfile: bad offsets of matrix %zu", m);
        for (uint64_t k = 1; k <= nrows[m]; k++) {
            FD2_REQUIRE(off[ob + k] >= off[ob + k - 1], FD2_ERR_IO, "fromfile: offsets not monotone");
            ro[++r] = base + (int64_t)off[ob + k];
        }
        base += (int64_t)mnnz[m];
        ob += nrows[m] + 1;
        mat_rows.push_back(r);
    }
    auto* e = new fd2_csr_ensemble();
    e->ctx = ctx;
    e->stream = ctx->stream;
    e->n_cols = n_cols;
    e->value_type = value_type;
    e->mat_rows = mat_rows;
    int rc = ensemble_reserve(e, total_rows, nnz);
    if (!rc) rc = stream_columns(ctx, col_path, val_path, nnz, vb, n_cols, e->d_col, e->d_val, e->stream);
    if (!rc && cudaMemcpyAsync(e->d_row_off, ro.data(), ro.size() * 8, cudaMemcpyHostToDevice, e->stream) != cudaSuccess)
        rc = FD2_ERR_CUDA;
    if (!rc && half && total_rows &&
        cudaMemcpyAsync(e->d_scale, b_scale.data(), total_rows * 4, cudaMemcpyHostToDevice, e->stream) != cudaSuccess)
        rc = FD2_ERR_CUDA;
    if (!rc && cudaStreamSynchronize(e->stream) != cudaSuccess) rc = FD2_ERR_CUDA;
    if (!rc) {
        e->n_rows = total_rows;
        e->nnz = e->nnz_bound = nnz;
    }
    if (rc) {
        fd2_csr_ensemble_destroy(e);
        return rc;
    }
    *out = e;
    return FD2_OK;
}

int fd2_csr_ensemble_destroy(fd2_csr_ensemble* e) {
    if (!e) return FD2_OK;
    for (void* p : {(void*)e->d_row_off, (void*)e->d_col, e->d_val, (void*)e->d_scale})
        if (p) cudaFreeAsync(p, e->stream);  // back to the context's pool, after the stream's pending work
    delete e;
    return FD2_OK;
}

int fd2_beamlet_flags_save(const uint8_t* flags, size_t n, const char* path) {
    FD2_REQUIRE(flags && path, FD2_ERR_INVALID_ARGUMENT, "flags_save: null argument");
    return write_file(path, flags, n);
}

}  // extern "C"

namespace fd2 {
fd2_context* ensemble_context(const fd2_csr_ensemble* e) { return e->ctx; }
cudaStream_t ensemble_stream(const fd2_csr_ensemble* e) { return e->stream; }
}  // namespace fd2
