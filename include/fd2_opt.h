/*
 * fd2_opt.h -- C ABI of the fluence optimizer: device CSR matrices and their
 * SpMV, the VOI restriction of a dose-loading matrix, the objective and
 * gradient of the IMRT problem, the group-sparsity proximal operator and the
 * two accelerated proximal-gradient solvers.
 *
 * Replaces (IMRTOpt, reference layout):
 *   IMRT::MatCSR64 + Eigen2Cusparse        IMRTOpt/include/IMRTDoseMat.cuh:29-69,
 *                                          IMRTOpt/src/IMRTEigenLoad.cu:390-435
 *   getStructFilter + parallelSpGEMM       IMRTOpt/src/IMRTEigenLoad.cu:101-273,
 *                                          IMRTOpt/src/IMRTEigenLoad.cpp:10-149
 *   parallelMatCoalesce / transposes       IMRTOpt/src/IMRTEigenLoad.cpp:190-304
 *   beamWeightsInit_func                   IMRTOpt/src/IMRTOptimize_var1.cu:125-161
 *   eval_g::evaluate                       IMRTOpt/src/IMRTOptUtils.cu:74-156
 *   eval_grad::evaluate                    IMRTOpt/src/IMRTOptUtils.cu:512-631
 *   proxL2Onehalf_QL_gpu::evaluate         IMRTOpt/src/IMRTOptimize_var1.cu:502-570
 *   BOO_IMRT_L2OneHalf_gpu_QL              IMRTOpt/src/IMRTOptimize.cu:16-194
 *   polish_BOO_IMRT_gpu                    IMRTOpt/src/IMRTOptimize.cu:391-476
 *   BeamOrientationOptimization            IMRTOpt/src/IMRTOptimize.cu:197-388
 *   DimReduction                           IMRTOpt/src/IMRTOptUtils.cu:726-793
 *   DVH curves of doseAnalyze              IMRTOpt/src/doseAnalyze.py:53-62
 *
 * Matrices hold int64 row offsets, int32 column indices and FP32, FP16 or BF16
 * values; 16-bit values carry one FP32 scale per column (a matrix of VOI rows x
 * beamlet columns) or per row (its transpose), so a matrix and its transpose
 * hold the same rounded values and the gradient stays the exact adjoint of
 * the objective's product.  Every product accumulates in FP32; the objective
 * terms, the group norms and the line-search test accumulate in FP64.  All
 * device pointers are caller-owned unless a handle owns them.
 */
#ifndef FD2_OPT_H
#define FD2_OPT_H

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

typedef struct fd2_matrix fd2_matrix;
typedef struct fd2_opt_problem fd2_opt_problem;

typedef enum fd2_scale_axis {
    FD2_SCALE_NONE = 0,
    FD2_SCALE_ROWS = 1,
    FD2_SCALE_COLS = 2
} fd2_scale_axis;

/*
 * Column index storage.  I32: one int32 per nonzero.  PACKED16: the nonzeros
 * are cut into chunks of 256; each chunk stores one int32 base column and a
 * 16-bit offset per nonzero, and a chunk whose columns span 65536 or more
 * keeps int32 columns in a side array -- 2 bytes per nonzero plus 4 per chunk
 * for matrices whose rows have local column ranges (VOI matrices, and any
 * matrix with at most 65536 columns).
 */
typedef enum fd2_index_format {
    FD2_INDEX_I32 = 0,
    FD2_INDEX_PACKED16 = 1
} fd2_index_format;

typedef struct fd2_matrix_info {
    int64_t rows, cols, nnz;
    int32_t value_type;   /* fd2_value_type */
    int32_t scale_axis;   /* fd2_scale_axis */
    int64_t device_bytes; /* bytes one SpMV pass streams: offsets/plan, columns, values, scales */
    int32_t index_format; /* fd2_index_format */
    int32_t x_in_shared; /* SpMV instance: 1 = x staged in shared memory (cols x 4 bytes <= 200 KiB) */
    int64_t exception_chunks; /* PACKED16 chunks stored with int32 columns */
} fd2_matrix_info_t;

/*
 * Upload a host CSR (Eigen2Cusparse): int64 offsets [rows+1], int64 columns
 * [nnz] (the reference's MatCSR64 index type), FP32 values [nnz].  16-bit
 * value types are scaled per column (column max -> 1) before rounding.
 */
int fd2_matrix_create(fd2_context* ctx, int64_t rows, int64_t cols, int64_t nnz, const int64_t* h_offsets,
                      const int64_t* h_columns, const float* h_values, int value_type, int index_format,
                      fd2_matrix** out);
int fd2_matrix_destroy(fd2_matrix* m);
int fd2_matrix_info(const fd2_matrix* m, fd2_matrix_info_t* info);
/* Copy to host as FP32 (scales applied): offsets [rows+1], columns [nnz], values [nnz]. */
int fd2_matrix_to_host(const fd2_matrix* m, int64_t* h_offsets, int32_t* h_columns, float* h_values);
/*
 * Transpose on the device: rows become columns, each new row lists its
 * columns in ascending order, values move unchanged (a column scale becomes a
 * row scale and vice versa).
 */
int fd2_matrix_transpose(const fd2_matrix* m, fd2_matrix** out);
/* d_y[rows] = M d_x[cols] (cusparseSpMV with alpha 1, beta 0), FP32 accumulation. */
int fd2_matrix_spmv(const fd2_matrix* m, const float* d_x, float* d_y, void* stream);

/*
 * VOI restriction of a dose-loading matrix (getStructFilter + parallelSpGEMM):
 * h_voxel_row[v] is the VOI row of PVCS voxel v (PTV rows first, then OAR
 * rows, each structure in voxel order) or -1.  Returns A = [n_voi x beamlets]
 * and AT = its transpose, in value_type (an FP32 source rounded to 16 bits
 * with a per-beamlet scale; a 16-bit source keeps its values and scales).
 * n_voxels must equal the dose matrix's column count.
 */
int fd2_voi_matrices(const fd2_csr_ensemble* dose, const int32_t* h_voxel_row, int64_t n_voxels, int64_t n_voi,
                     int value_type, int index_format, fd2_matrix** A, fd2_matrix** AT);

/*
 * Seeded synthetic VOI matrix pair for optimizer benchmarks: rows x cols with
 * each column j covering a window of `window` consecutive rows centred at
 * (j + 1/2) rows / cols, each (row, column) of the window kept with
 * probability `density` (a hash of seed, row and column), the value falling
 * off with the distance to the window centre.  A and its transpose are
 * generated independently from the same formula, so they hold identical
 * values.
 */
int fd2_matrix_synthetic(fd2_context* ctx, int64_t rows, int64_t cols, int64_t window, float density, uint64_t seed,
                         int value_type, int index_format, fd2_matrix** A, fd2_matrix** AT);

/*
 * fluenceGradInit for one beam (IMRTOpt/src/IMRTOptimize_var.cpp:59-180 with
 * DxyInit / KroneckerProduct, IMRTOpt/src/IMRTEigenLoad.cpp:307-407): the CSR
 * of D_b over the beam's active beamlets (active[fluence_dim^2], row-major
 * fluence map; beamlet columns numbered in map order), one row (-1, +1) per
 * pair of horizontally, then vertically, adjacent active pixels.  Caller
 * capacities: offsets 2 n^2 + 1, columns and values 4 n^2.  Host only.
 */
int fd2_fluence_grad(int fluence_dim, const uint8_t* active, int64_t* rows, int64_t* nnz, int64_t* offsets,
                     int64_t* columns, float* values);

/*
 * The IMRT problem (eval_g / eval_grad state).  A: [n_ptv + n_oar] x n
 * (PTV rows first), AT its transpose, D the fluence-gradient rows [m x n],
 * DT its transpose.  Weight vectors are host arrays: max_dose and
 * max_weights [n_ptv + n_oar], min_dose and min_weights [n_ptv], oar_weights
 * [n_oar].  The handle keeps pointers to the four matrices (they must
 * outlive it) and owns its work vectors.
 */
int fd2_opt_problem_create(fd2_context* ctx, const fd2_matrix* A, const fd2_matrix* AT, const fd2_matrix* D,
                           const fd2_matrix* DT, int64_t n_ptv, int64_t n_oar, const float* h_max_dose,
                           const float* h_max_weights, const float* h_min_dose, const float* h_min_weights,
                           const float* h_oar_weights, float gamma, float eta, fd2_opt_problem** out);
int fd2_opt_problem_destroy(fd2_opt_problem* p);
/*
 * Line-search trials as one CUDA graph (default on): the trial's kernels and
 * copies are captured once per solver call (per state vectors and group
 * count) and replayed with the trial's scalars read from pinned memory.  Off:
 * the same launches one by one.  Results are identical either way.
 */
int fd2_opt_problem_set_graph(fd2_opt_problem* p, int on);

/*
 * Row-sharded problems (one process per GPU, each holding a contiguous block
 * of A's VOI rows, PTV rows first, with x, D and the weights of its rows): fn
 * must replace d_buf[0..n) by its sum over the ranks before returning (e.g. an
 * all-reduce over NCCL), on or after the given stream's work -- the solver has
 * synchronised that stream before the call.  The solver calls it once per
 * objective evaluation with the three VOI-row objective terms and, for a
 * gradient, the partial A^T g (FP64), and once in fd2_beam_weights_init; every
 * rank then takes the same steps.  A reducer turns graph capture off.  NULL
 * restores the single-GPU problem.
 */
typedef int (*fd2_reduce_fn)(void* user, double* d_buf, int64_t n, void* stream);
int fd2_opt_problem_set_reducer(fd2_opt_problem* p, fd2_reduce_fn fn, void* user);

/* eval_g::evaluate: *h_value = g(d_x) (synchronises the context's stream). */
int fd2_eval_g(fd2_opt_problem* p, const float* d_x, double* h_value);
/* eval_grad::evaluate: d_grad[n] = grad g(d_x), *h_value = g(d_x). */
int fd2_eval_grad(fd2_opt_problem* p, const float* d_x, float* d_grad, double* h_value);

/*
 * proxL2Onehalf_QL_gpu::evaluate on groups of consecutive entries
 * (group r = [d_group_offsets[r], d_group_offsets[r+1])): prox of
 * tau_r * ||x_r||_2^(1/2) at g0, and the new group norms.
 */
int fd2_prox_l2onehalf(fd2_context* ctx, int64_t n_groups, const int64_t* d_group_offsets, const float* d_g0,
                       const float* d_tau, float* d_prox, float* d_nrm, void* stream);

/* beamWeightsInit_func: w_b from the PTV rows of A over each beam's columns. */
int fd2_beam_weights_init(fd2_opt_problem* p, int64_t n_groups, const int64_t* h_group_offsets, float* h_weights);

/* Solver state carried between calls (the reference's by-reference arguments). */
typedef struct fd2_opt_state {
    int32_t k_global;
    float theta_km1, tkm1;
    int32_t trials;     /* out: line-search trials in this call */
    float* d_xkm1;      /* [n] device, in/out */
    float* d_vkm1;      /* [n] device, in/out */
    float* h_loss;      /* [iters_global] host, out (may be NULL) */
    float* h_nrm;       /* [n_groups] host, out (BOO only, may be NULL) */
    float num_active;   /* out (BOO only) */
    int32_t stop;       /* out (BOO only) */
} fd2_opt_state_t;

/* BOO_IMRT_L2OneHalf_gpu_QL (h_beam_weights in/out, h_prune_trigger ascending). */
int fd2_boo_l2onehalf(fd2_opt_problem* p, int64_t n_groups, const int64_t* h_group_offsets, float* h_beam_weights,
                      int show_trigger, int change_weights_trigger, int iters_global, const int32_t* h_prune_trigger,
                      int n_prune, int num_beams_we_want, fd2_opt_state_t* st);
/* polish_BOO_IMRT_gpu */
int fd2_polish(fd2_opt_problem* p, int iters_global, int iters_local, fd2_opt_state_t* st);

/*
 * Row-block selection (replaces parallelMatCoalesce over the active beams'
 * VOIMatricesT and diagBlock over their SpFluenceGrad, IMRTOptimize.cu:278-300,
 * IMRTEigenLoad.cpp:190-304, done on the host there at every prune phase):
 * block b = rows [h_block_rows[b], h_block_rows[b+1]) of m; the blocks
 * h_order[0..n_keep) are copied, in that order, into a new matrix of the same
 * value type, index format and scale axis.  With h_block_cols (m block-
 * diagonal: block b's rows use only columns [h_block_cols[b], h_block_cols[b+1]))
 * the columns are renumbered block by block in the kept order; with NULL they
 * are unchanged.  Values are copied, not re-rounded.
 */
int fd2_matrix_select_blocks(const fd2_matrix* m, int64_t n_blocks, const int64_t* h_block_rows,
                             const int64_t* h_block_cols, int64_t n_keep, const int64_t* h_order, fd2_matrix** out);

/*
 * Cumulative dose-volume histograms (the curve doseAnalyze.py:53-62 draws from
 * sorted structure doses, binned): structure s owns the voxel indices
 * d_voxels[h_struct_offsets[s] .. h_struct_offsets[s+1]) (host offsets;
 * structures may overlap); voxel v falls in bin floor(d_dose[v] / bin_width)
 * clamped to [0, n_bins); d_cumulative[s * n_bins + k] = voxels of s in bins
 * >= k, i.e. receiving at least k * bin_width.  Voxel indices outside
 * [0, n_voxels) are an error.  Synchronises the stream.
 */
int fd2_dvh(fd2_context* ctx, const float* d_dose, int64_t n_voxels, int64_t n_structs,
            const int64_t* h_struct_offsets, const int32_t* d_voxels, int n_bins, float bin_width,
            unsigned long long* d_cumulative, void* stream);

/* Parameters of the beam-orientation loop (the reference's Params). */
typedef struct fd2_boo_params {
    float beam_weight;             /* beamWeight: factor on the initial beam weights */
    float step_size;               /* stepSize: initial step t */
    float gamma, eta;              /* Huber threshold and TV weight */
    int32_t max_iter;              /* maxIter: global iteration budget */
    int32_t change_weights_trigger;
    int32_t show_trigger;          /* the reference's progress print period (no output here) */
    int32_t n_beams_want;          /* numBeamsWeWant */
    const int32_t* prune_trigger;  /* pruneTrigger: ascending global iterations that end a phase */
    int32_t n_prune;
    int32_t reserved;
} fd2_boo_params_t;

typedef struct fd2_boo_result {
    int32_t iterations;  /* k_global at the end */
    int32_t n_active;    /* beams kept */
    int32_t phases;      /* solver phases (matrix selections) run */
    int32_t trials;      /* line-search trials over all phases */
} fd2_boo_result_t;

/*
 * BeamOrientationOptimization (IMRTOptimize.cu:197-388) with DimReduction
 * (IMRTOptUtils.cu:726-793), the matrices never leaving the device.
 *   AT     beamlets x VOI rows of all candidate beams; beam b owns rows
 *          [h_beam_rows[b], h_beam_rows[b+1]) (its active beamlets)
 *   D      block-diagonal fluence-gradient operator; beam b owns rows
 *          [h_d_rows[b], h_d_rows[b+1]) and columns [h_beam_rows[b], h_beam_rows[b+1])
 *   VOI weights as fd2_opt_problem_create
 *   d_x0   initial fluence of all beamlets (the reference draws rand()/RAND_MAX
 *          after srand(10086), IMRTOptimize.cu:240-243); v starts equal to it
 * Each phase runs the accelerated proximal-gradient loop until a prune trigger,
 * the beam target or max_iter; then the beams are ranked by group norm
 * (descending, ties by position) and those with norm > 1e-4 are kept, with
 * their weights and their x, v segments, in that order.
 * Out: h_costs[k] for every iteration k run ([max_iter]); h_active[0..n_active)
 * the kept beams in their final order and h_norms their norms (the reference
 * leaves its norms in the order before the last ranking); d_x[0..) the kept
 * beams' fluence in that order (capacity: all beamlets).
 */
int fd2_beam_orientation_optimization(fd2_context* ctx, const fd2_matrix* AT, const fd2_matrix* D, int64_t n_beams,
                                      const int64_t* h_beam_rows, const int64_t* h_d_rows, int64_t n_ptv,
                                      int64_t n_oar, const float* h_max_dose, const float* h_max_weights,
                                      const float* h_min_dose, const float* h_min_weights,
                                      const float* h_oar_weights, const fd2_boo_params_t* params, const float* d_x0,
                                      float* h_costs, int32_t* h_active, float* h_norms, float* d_x,
                                      fd2_boo_result_t* result);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
