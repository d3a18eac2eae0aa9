/*
 * fd2_imrt.h -- C ABI of the IMRT planning layer: beamlet flagging, the
 * dose-loading-matrix construction and its on-disk layout.  Replaces the
 * IMRTOpt entry points named beside each declaration.  Conventions as in fd2.h.
 */
#ifndef FD2_IMRT_H
#define FD2_IMRT_H

#include "fd2.h"

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* Value storage of a dose-loading matrix. 16-bit formats carry one float scale
 * per row (beamlet), value = scale * stored. */
typedef enum fd2_value_type {
    FD2_VALUES_F32 = 0,
    FD2_VALUES_F16 = 1,
    FD2_VALUES_BF16 = 2
} fd2_value_type;

/*
 * IMRT::beamletFlagInit (IMRTOpt/src/IMRTBeamBundle.cu:130-316): a fluence
 * pixel of a bundle is on when any of super_sampling^2 sub-rays, at any slice
 * of the bundle's range, samples the (linear-filtered) PTV mask above zero.
 * h_ptv_mask is uint8[z][y][x]; h_flags_out is uint8[n_bundles][fy][fx].
 * Sampling uses the GPU texture unit, like the reference.
 */
int fd2_beamlet_flags(fd2_context* ctx, size_t n_bundles, const fd2_bundle_t* h_bundles,
                      const uint8_t* h_ptv_mask, const fd2_volume_t* volume, int super_sampling,
                      uint8_t* h_flags_out);

/*
 * Host copy of a dose matrix, filled while the matrix is built (see
 * fd2_dosemat_params_t.host_out).  The buffers are the caller's; pinned ones
 * (cudaHostAlloc, cudaHostRegister) let each batch's copy run on a copy stream
 * while the device computes the next batch, pageable ones give the same
 * contents without the overlap.  On return row_off[0..n_rows] holds the
 * matrix's row offsets (row_off[0] = 0), col/val its first nnz nonzeros, and
 * for 16-bit values scale[0..n_rows) the row scales -- the arrays
 * fd2_csr_ensemble_device exposes, in the ensemble's value type.
 */
typedef struct fd2_host_csr {
    int64_t* row_off;   /* [n_rows + 1] */
    int32_t* col;       /* [cap_nnz] voxel indices */
    void* val;          /* [cap_nnz] values: float, or 16-bit words for FD2_VALUES_F16/BF16 */
    float* scale;       /* [n_rows] row scales of 16-bit values; not used (may be NULL) for F32 */
    uint64_t cap_nnz;   /* capacity of col and val in nonzeros; too small -> FD2_ERR_CAPACITY */
    uint64_t nnz;       /* out: nonzeros written */
} fd2_host_csr_t;

/* Dose-matrix construction parameters (the getarg reads of
 * IMRT::DoseMatConstruction, IMRTOpt/src/IMRTDoseMat.cu:32,58,80-81). */
typedef struct fd2_dosemat_params {
    float extent;               /* cm; voxels farther from a beamlet axis are 0 (default 2.0) */
    int ss_factor;              /* supersampling per axis of the column stage (default 5) */
    int value_type;             /* fd2_value_type (default F32) */
    int cccs_schedule;          /* -1 auto (both timed on the first batch of a shape, the faster kept),
                                   -2 rule (zenith split below 4 blocks per SM; no timing run),
                                   0 zenith loop per block, 1 zenith split */
    uint64_t batch_beamlets;    /* 0 = auto (memory budget) */
    uint64_t memory_budget;     /* bytes of BEV scratch per batch; 0 = auto */
    int verbose;                /* print per-batch timings to stdout */
    fd2_host_csr_t* host_out;   /* NULL (default), or host buffers the matrix is copied into
                                   batch by batch as it is built (fd2_dose_mat_construct only) */
    int graph;                  /* 0 (default): each batch's work is launched call by call.
                                   1: each batch's device work -- uploads of its descriptor tables,
                                   Terma, cone directions, CCCS, column values, row offsets, gather
                                   -- is captured as one CUDA graph and launched with one call; the
                                   context keeps one executable graph per batch shape (map size,
                                   cones, schedule, value type, supersampling) and updates it in
                                   place with the next batch's parameters.  The CCCS schedule is
                                   then fixed per batch (-1 acts as -2), and the matrix is bit for
                                   bit the one direct launches give.  fd2_dose_mat_construct only. */
    int overlap;                /* 1 (default): the column stage of each batch runs on a second stream
                                   of the context beside the next batch's Terma and CCCS, which then
                                   fill a second BEV buffer (a plan of several batches holds up to
                                   twice memory_budget of BEV scratch); 0: one stream, one buffer.
                                   The matrix is the same bit for bit.  Ignored with graph = 1.
                                   fd2_dose_mat_construct only. */
} fd2_dosemat_params_t;

void fd2_dosemat_params_default(fd2_dosemat_params_t* p);

/*
 * IMRT::DoseMatConstruction (IMRTOpt/src/IMRTDoseMat.cu:14-301): Terma, CCCS
 * and BEV->PVCS column emission for every beamlet of every beam, producing one
 * CSR matrix per beam (rows = beamlets in the order given, columns = voxel
 * index x + X*(y + Y*z), ascending, exact zeros dropped -- the layout
 * cusparseDenseToSparse gives the reference).
 *   n_beamlets_per_beam[n_beams]; h_beamlets: all beamlets, beam after beam;
 *   h_fluence: the sub-beam fluence map (fmap_x*fmap_y floats) shared by all.
 * The beamlets' BEV dose buffers are zeroed before each beam; the reference
 * reuses them without clearing (its beams accumulate), which is not reproduced.
 */
int fd2_dose_mat_construct(fd2_context* ctx, size_t n_beams, const uint32_t* n_beamlets_per_beam,
                           const fd2_beam_t* h_beamlets, const float* h_fluence,
                           const fd2_density* density, const fd2_spectrum* spectrum,
                           const fd2_cccs_kernel* kernel, const fd2_dosemat_params_t* params,
                           fd2_csr_ensemble** out, void* stream);

/*
 * IMRT::BEV2PVCSInterp (batched, IMRTOpt/src/IMRTgeom.cu:221-367) followed by
 * MatCSREnsemble::addMat (IMRTSparseMatEns.cu:66-165): the dose columns of
 * beamlets whose BEV dose is already on the device.  d_dose_bev is a device
 * array of device pointers, one [long_dim][fmap_y][fmap_x] array per beamlet.
 * One CSR matrix per beam, as fd2_dose_mat_construct.
 */
int fd2_bev2pvcs_interp(fd2_context* ctx, size_t n_beams, const uint32_t* n_beamlets_per_beam,
                        const fd2_beam_t* h_beamlets, const float* const* d_dose_bev,
                        const fd2_density* density, const fd2_dosemat_params_t* params,
                        fd2_csr_ensemble** out, void* stream);

typedef struct fd2_csr_info {
    uint64_t n_mats;      /* beams */
    uint64_t n_rows;      /* beamlets in total */
    uint64_t n_cols;      /* voxels */
    uint64_t nnz;
    int value_type;
} fd2_csr_info_t;

int fd2_csr_ensemble_info(const fd2_csr_ensemble* e, fd2_csr_info_t* info);

/* Device views: row_offsets int64[n_rows+1] (global), columns int32[nnz],
 * values (f32/f16/bf16)[nnz], row_scale float[n_rows] (NULL for F32),
 * mat_rows uint64[n_mats+1] (first row of each beam).
 * An ensemble's arrays come from the context's stream-ordered memory pool and
 * are ordered on the stream it was built on (the construction call's stream,
 * or the context's for fromfile): work on another stream must wait for that
 * stream first, and the ensemble must be destroyed before that stream is. */
int fd2_csr_ensemble_device(const fd2_csr_ensemble* e, const int64_t** row_offsets,
                            const int32_t** columns, const void** values, const float** row_scale,
                            const uint64_t** mat_rows_host);

/* Copies the ensemble to host buffers, values decoded to float. */
int fd2_csr_ensemble_to_host(const fd2_csr_ensemble* e, int64_t* row_offsets, int32_t* columns,
                             float* values);

/*
 * MatCSREnsemble::tofile (IMRTOpt/src/IMRTSparseMatEns.cu:168-239): writes
 * NonZeroElements.bin, CumuNonZeroElements.bin, numRowsPerMat.bin,
 * CumuNumRowsPerMat.bin, OffsetBufferIdx.bin (uint64[n_mats] each),
 * offsetsBuffer.bin (uint64, per matrix n_rows+1 local offsets), columnsBuffer.bin
 * (uint64[nnz]) and valuesBuffer.bin (float32[nnz]) into `folder` (created).
 * A 16-bit ensemble also writes its stored values and row scales as sidecars
 * (valuesBuffer.f16.bin or .bf16.bin: uint16[nnz]; rowScales.f16.bin or
 * .bf16.bin: float32[n_rows]); the reference's files are unchanged by them.
 */
int fd2_csr_ensemble_tofile(const fd2_csr_ensemble* e, const char* folder);

/*
 * MatCSREnsemble::fromfile (IMRTSparseMatEns.cu:242-337) into a device ensemble.
 * value_type F32 reads valuesBuffer.bin; F16/BF16 read that type's sidecars
 * (the exact stored values and scales) and refuse a folder without them.
 * Columns and values stream to the device in chunks of 4M nonzeros through
 * two pinned host buffers (host memory stays at two chunks); a column index
 * >= n_cols is refused with FD2_ERR_IO.
 */
int fd2_csr_ensemble_fromfile(fd2_context* ctx, const char* folder, uint64_t n_cols,
                              int value_type, fd2_csr_ensemble** out);

int fd2_csr_ensemble_destroy(fd2_csr_ensemble* e);

/*
 * The matrices of several ensembles (same voxel count and value type) as one
 * ensemble, in order, on ctx's stream -- e.g. the per-isocentre dose-loading
 * matrices of a multi-isocentre plan for a joint optimization.  No reference
 * counterpart (its joint problems concatenate the Eigen matrices on the host).
 */
int fd2_csr_ensemble_concat(fd2_context* ctx, size_t n, const fd2_csr_ensemble* const* parts,
                            fd2_csr_ensemble** out);

/* IMRT::beamletFlagSave (IMRTBeamBundle.cu:572-601): uint8 flags to a file. */
int fd2_beamlet_flags_save(const uint8_t* flags, size_t n, const char* path);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* FD2_IMRT_H */
