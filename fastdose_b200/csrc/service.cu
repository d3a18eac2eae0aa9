// service.cu -- served dose calculation (fd2_service.h).
//
// A FIFO of plan requests feeds `workers` host threads, each owning an
// fd2_context (its own stream, stream-ordered pool and grow-only buffers) on
// the service's device.  The head of the queue is admitted when the sum of the
// admitted requests' device-memory estimates plus its own stays within the HBM
// budget (or when nothing else is running), so a large plan waits for memory
// instead of failing, and admission never reorders requests.  A worker copies
// the request's phantom and tables to its context, runs
// fd2_dose_mat_construct on its stream and hands the matrix to the waiter.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/fd2_service.h"
#include "fd2_internal.cuh"

namespace {

struct Request {
    uint64_t id = 0;
    std::vector<float> density;
    fd2_volume_t vol{};
    std::vector<uint32_t> per_beam;
    std::vector<fd2_beam_t> beamlets;
    std::vector<float> fluence;
    std::vector<float> energy, sfl, mu, mu_en;
    std::vector<float> theta, A, a, B, b, phi;
    fd2_dosemat_params_t params{};
    fd2_request_stats_t stats{};
    fd2_csr_ensemble* result = nullptr;
    std::string error;  // the worker's message when the construction failed
    bool done = false;
};

// Device bytes a request holds while it runs: its density, one batch of BEV
// volumes, the column scratch and the finished matrix.  The matrix is bounded
// by the candidate voxels of each beamlet: a cylinder of radius extent + half a
// voxel diagonal around its axis over its depth range.
uint64_t estimate_bytes(const Request& r, uint64_t bev_budget) {
    const double nvox = (double)r.vol.dim[0] * r.vol.dim[1] * r.vol.dim[2];
    const double vx = r.vol.voxel_size[0], vy = r.vol.voxel_size[1], vz = r.vol.voxel_size[2];
    const double hdiag = 0.5 * std::sqrt(vx * vx + vy * vy + vz * vz);
    const double rr = r.params.extent + hdiag;
    double bev = 0, nnz = 0;
    for (const auto& bl : r.beamlets) {
        bev += (double)bl.long_dim * bl.fmap_size[0] * bl.fmap_size[1] * 3 * sizeof(float);
        nnz += M_PI * rr * rr * bl.long_dim * bl.long_spacing / (vx * vy * vz);
    }
    const double vb = r.params.value_type == FD2_VALUES_F32 ? 4 : 2;
    const double bev_batch = std::min(bev, (double)bev_budget);
    const double batch_share = bev > 0 ? bev_batch / bev : 1.0;
    const double bytes = nvox * 4 + bev_batch + nnz * (4 + vb) + nnz * batch_share * 8 +
                         (double)r.beamlets.size() * 64 + (64ull << 20);
    return (uint64_t)bytes;
}

double now_ms(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct fd2_service {
    int device = 0;
    uint64_t budget = 0, bev_budget = 0, in_use = 0;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::deque<Request*> queue;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> all;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::vector<std::thread> workers;
    std::vector<fd2_context*> contexts;  // one per worker; destroyed after the uncollected results
    bool stop = false;
    uint64_t next_id = 1;
    int running = 0;
};

namespace {

int run_request(fd2_context* ctx, Request& r) {
    fd2_density* d = nullptr;
    fd2_spectrum* sp = nullptr;
    fd2_cccs_kernel* k = nullptr;
    // every allocation of a request is stream-ordered on the worker's stream:
    // a free that waited for the whole device would wait for the other
    // workers' requests too
    int rc = fd2::density_create_pooled(ctx, r.density.data(), &r.vol, &d);
    if (!rc)
        rc = fd2_spectrum_create(ctx, (int)r.energy.size(), r.energy.data(), r.sfl.data(), r.mu.data(),
                                 r.mu_en.data(), &sp);
    if (!rc)
        rc = fd2_kernel_create(ctx, (int)r.theta.size(), r.theta.data(), r.A.data(), r.a.data(), r.B.data(),
                               r.b.data(), (int)r.phi.size(), r.phi.data(), &k);
    if (!rc)
        rc = fd2_dose_mat_construct(ctx, r.per_beam.size(), r.per_beam.data(), r.beamlets.data(), r.fluence.data(),
                                    d, sp, k, &r.params, &r.result, ctx->stream);
    if (!rc) {
        fd2_csr_info_t info;
        if (fd2_csr_ensemble_info(r.result, &info) == FD2_OK) r.stats.nnz = info.nnz;
    }
    cudaStreamSynchronize(ctx->stream);
    if (k) fd2_kernel_destroy(k);
    if (sp) fd2_spectrum_destroy(sp);
    if (d) fd2_density_destroy(d);
    return rc;
}

void worker_main(fd2_service* s, int index) {
    fd2_context* ctx = nullptr;
    const int crc = fd2_context_create(s->device, &ctx);
    if (!crc) {
        // Grow the worker's pool once, up front, by a request's usual working
        // set (one batch of BEV volumes and as much again for the matrix and
        // the column scratch): mapping new device memory while the other
        // workers' kernels run stalls them, so requests should find it mapped.
        void* p = nullptr;
        if (cudaMallocFromPoolAsync(&p, 2 * s->bev_budget, ctx->pool, ctx->stream) == cudaSuccess)
            cudaFreeAsync(p, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
        cudaGetLastError();  // an oversized reserve is not an error of the service
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->contexts[index] = ctx;
    }
    for (;;) {
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] {
                if (s->stop) return true;
                if (s->queue.empty()) return false;
                const uint64_t need = s->queue.front()->stats.est_bytes;
                return s->running == 0 || s->in_use + need <= s->budget;
            });
            if (s->stop) break;
            r = s->queue.front();
            s->queue.pop_front();
            s->in_use += r->stats.est_bytes;
            s->running++;
            r->stats.start_ms = now_ms(s->t0);
            r->stats.worker = index;
        }
        const int rc = crc ? crc : run_request(ctx, *r);
        const std::string msg = rc ? std::string(fd2_last_error()) : std::string();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r->stats.status = rc;
            r->error = msg;
            r->stats.end_ms = now_ms(s->t0);
            s->in_use -= r->stats.est_bytes;
            s->running--;
            r->done = true;
            // the request's inputs are no longer needed
            std::vector<float>().swap(r->density);
            std::vector<fd2_beam_t>().swap(r->beamlets);
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

}  // namespace

extern "C" {

int fd2_service_create(const fd2_service_params_t* p, fd2_service** out) {
    FD2_REQUIRE(p && out, FD2_ERR_INVALID_ARGUMENT, "service_create: null argument");
    FD2_REQUIRE(p->workers >= 1 && p->workers <= 8, FD2_ERR_INVALID_ARGUMENT, "service_create: %d workers (1..8)",
                p->workers);
    int n = 0;
    FD2_CHECK_CUDA(cudaGetDeviceCount(&n));
    FD2_REQUIRE(p->device >= 0 && p->device < n, FD2_ERR_INVALID_ARGUMENT, "service_create: no device %d",
                p->device);
    FD2_CHECK_CUDA(cudaSetDevice(p->device));
    size_t free_b = 0, tot_b = 0;
    FD2_CHECK_CUDA(cudaMemGetInfo(&free_b, &tot_b));
    auto* s = new fd2_service();
    s->device = p->device;
    s->budget = p->hbm_budget ? p->hbm_budget : free_b / 4 * 3;
    s->bev_budget = p->bev_budget ? p->bev_budget : (4ull << 30);
    s->contexts.assign(p->workers, nullptr);
    for (int i = 0; i < p->workers; i++) s->workers.emplace_back(worker_main, s, i);
    *out = s;
    return FD2_OK;
}

int fd2_service_destroy(fd2_service* s) {
    if (!s) return FD2_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        for (Request* r : s->queue) {
            r->stats.status = FD2_ERR_ADMISSION;
            r->done = true;
        }
        s->queue.clear();
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    for (auto& t : s->workers) t.join();
    for (auto& kv : s->all)
        if (kv.second->result) fd2_csr_ensemble_destroy(kv.second->result);  // results nobody collected
    for (fd2_context* c : s->contexts)
        if (c) fd2_context_destroy(c);
    delete s;
    return FD2_OK;
}

int fd2_service_submit(fd2_service* s, const fd2_plan_request_t* q, uint64_t* ticket) {
    FD2_REQUIRE(s && q && ticket && q->density && q->n_beamlets_per_beam && q->beamlets && q->fluence && q->energy &&
                    q->spectrum_fluence && q->mu && q->mu_en && q->theta && q->A && q->a && q->B && q->b && q->phi,
                FD2_ERR_INVALID_ARGUMENT, "service_submit: null argument");
    auto r = std::make_unique<Request>();
    const size_t nvox = (size_t)q->volume.dim[0] * q->volume.dim[1] * q->volume.dim[2];
    r->density.assign(q->density, q->density + nvox);
    r->vol = q->volume;
    r->per_beam.assign(q->n_beamlets_per_beam, q->n_beamlets_per_beam + q->n_beams);
    size_t total = 0;
    for (uint32_t c : r->per_beam) total += c;
    r->beamlets.assign(q->beamlets, q->beamlets + total);
    const size_t P = total ? (size_t)q->beamlets[0].fmap_size[0] * q->beamlets[0].fmap_size[1] : 0;
    r->fluence.assign(q->fluence, q->fluence + P);
    r->energy.assign(q->energy, q->energy + q->n_spectrum);
    r->sfl.assign(q->spectrum_fluence, q->spectrum_fluence + q->n_spectrum);
    r->mu.assign(q->mu, q->mu + q->n_spectrum);
    r->mu_en.assign(q->mu_en, q->mu_en + q->n_spectrum);
    for (auto pr : {std::make_pair(&r->theta, q->theta), std::make_pair(&r->A, q->A), std::make_pair(&r->a, q->a),
                    std::make_pair(&r->B, q->B), std::make_pair(&r->b, q->b)})
        pr.first->assign(pr.second, pr.second + q->n_theta);
    r->phi.assign(q->phi, q->phi + q->n_phi);
    r->params = q->params;
    r->params.memory_budget = s->bev_budget;
    r->params.host_out = nullptr;  // a served request's result stays on the device
    // the admission estimate counts one BEV batch per request, so a worker
    // builds with one BEV buffer: no column-stage overlap
    r->params.overlap = 0;
    // a request's latency must not carry a timing run of both CCCS schedules
    // (each new batch shape would add one): served requests take the rule
    if (r->params.cccs_schedule == -1) r->params.cccs_schedule = -2;
    r->stats.beamlets = total;
    r->stats.est_bytes = estimate_bytes(*r, s->bev_budget);
    FD2_REQUIRE(r->stats.est_bytes <= s->budget, FD2_ERR_ADMISSION,
                "service_submit: request needs ~%llu bytes, the budget is %llu",
                (unsigned long long)r->stats.est_bytes, (unsigned long long)s->budget);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        FD2_REQUIRE(!s->stop, FD2_ERR_ADMISSION, "service_submit: the service is stopping");
        r->id = s->next_id++;
        r->stats.submit_ms = now_ms(s->t0);
        s->queue.push_back(r.get());
        *ticket = r->id;
        s->all.emplace(r->id, std::move(r));
    }
    s->cv_work.notify_all();
    return FD2_OK;
}

int fd2_service_wait(fd2_service* s, uint64_t ticket, fd2_csr_ensemble** out, fd2_request_stats_t* stats) {
    FD2_REQUIRE(s && out, FD2_ERR_INVALID_ARGUMENT, "service_wait: null argument");
    std::unique_ptr<Request> r;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->all.find(ticket);
        FD2_REQUIRE(it != s->all.end(), FD2_ERR_INVALID_ARGUMENT, "service_wait: unknown ticket %llu",
                    (unsigned long long)ticket);
        Request* rp = it->second.get();
        s->cv_done.wait(lk, [&] { return rp->done; });
        r = std::move(it->second);
        s->all.erase(it);
    }
    *out = r->result;
    if (stats) *stats = r->stats;
    if (r->stats.status) {
        fd2::set_error("service request %llu: %s", (unsigned long long)ticket,
                       r->error.empty() ? "not run" : r->error.c_str());
        return r->stats.status;
    }
    return FD2_OK;
}

double fd2_service_clock_ms(const fd2_service* s) { return s ? now_ms(s->t0) : 0.0; }

}  // extern "C"
