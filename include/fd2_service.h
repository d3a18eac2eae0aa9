/*
 * fd2_service.h -- served dose calculation.
 *
 * No counterpart in the reference, which computes one plan per process
 * (IMRTOpt/main.cu, IMRT::DoseMatConstruction over the beams of one patient).
 * A service takes plan requests (phantom, beamlets, spectrum, kernel) from any
 * host thread, admits them in arrival order while the sum of their device
 * memory estimates stays under an HBM budget, and runs each on one of its
 * worker contexts.  Workers keep their device buffers (BEV volumes, column
 * scratch, the stream-ordered pool) from request to request, so a steady
 * stream of requests allocates nothing after warm-up.  Every request records
 * its submit, start and end times on the service's clock, from which a client
 * reports queueing and end-to-end latency.
 */
#ifndef FD2_SERVICE_H
#define FD2_SERVICE_H

#include <stddef.h>
#include <stdint.h>

#include "fd2.h"
#include "fd2_imrt.h"

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef struct fd2_service fd2_service;

typedef struct fd2_service_params {
    int device;
    int workers;           /* worker contexts (1..8); each has its own stream */
    int32_t reserved;
    uint64_t hbm_budget;   /* bytes admitted requests may hold on the device at once (0: 3/4 of free memory) */
    uint64_t bev_budget;   /* BEV bytes per construction batch (fd2_dosemat_params_t::memory_budget; 0: 4 GiB) */
} fd2_service_params_t;

/* One plan.  All host arrays are copied by fd2_service_submit. */
typedef struct fd2_plan_request {
    const float* density;              /* [z][y][x] */
    fd2_volume_t volume;
    size_t n_beams;
    const uint32_t* n_beamlets_per_beam;
    const fd2_beam_t* beamlets;        /* sum(n_beamlets_per_beam), after fd2_beam_calc_range */
    const float* fluence;              /* one beamlet's fluence map, fmap_size[0] * fmap_size[1] */
    int n_spectrum;
    const float* energy;
    const float* spectrum_fluence;
    const float* mu;
    const float* mu_en;
    int n_theta;
    const float* theta;
    const float* A;
    const float* a;
    const float* B;
    const float* b;
    int n_phi;
    const float* phi;
    fd2_dosemat_params_t params;       /* memory_budget is replaced by the service's bev_budget */
} fd2_plan_request_t;

typedef struct fd2_request_stats {
    double submit_ms;   /* service clock */
    double start_ms;
    double end_ms;
    uint64_t beamlets;
    uint64_t nnz;
    uint64_t est_bytes; /* admission estimate */
    int32_t status;     /* fd2_status of the construction */
    int32_t worker;
} fd2_request_stats_t;

int fd2_service_create(const fd2_service_params_t* params, fd2_service** out);
/*
 * Stops taking requests, finishes the running ones, fails the queued ones
 * (FD2_ERR_ADMISSION) and frees the workers.  Destroy every result first:
 * a result's memory belongs to its worker's context.
 */
int fd2_service_destroy(fd2_service* s);
/* Queues a request; FD2_ERR_ADMISSION when it could never fit the budget. */
int fd2_service_submit(fd2_service* s, const fd2_plan_request_t* request, uint64_t* ticket);
/*
 * Waits for a request and hands over its dose-loading matrix (the caller
 * destroys it; NULL when the construction failed -- see stats.status).
 * Each ticket can be waited for once.
 */
int fd2_service_wait(fd2_service* s, uint64_t ticket, fd2_csr_ensemble** out, fd2_request_stats_t* stats);
/* Milliseconds on the service clock (the clock of the request stats). */
double fd2_service_clock_ms(const fd2_service* s);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
