// opt_internal.cuh -- device CSR matrix of the optimizer, shared by the SpMV,
// VOI-restriction and solver translation units.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "../../include/fd2_opt.h"
#include "fd2_internal.cuh"

struct fd2_matrix {
    fd2_context* ctx = nullptr;
    int64_t rows = 0, cols = 0, nnz = 0;
    int value_type = FD2_VALUES_F32;
    int scale_axis = FD2_SCALE_NONE;
    int64_t* d_off = nullptr;    // [rows + 1]
    int32_t* d_col = nullptr;    // [nnz]
    void* d_val = nullptr;       // [nnz] float / __half / __nv_bfloat16
    float* d_scale = nullptr;    // [rows] or [cols] when scale_axis != NONE
    // merge-path SpMV plan (rows + nnz items cut into equal tiles)
    int64_t n_tiles = 0;
    int64_t* d_tile_row = nullptr;   // [n_tiles + 1] path coordinate (rows consumed)
    int64_t* d_tile_nz = nullptr;    // [n_tiles + 1] path coordinate (nonzeros consumed)
    int64_t* d_carry_row = nullptr;  // [n_tiles] row in progress at each tile's end
    float* d_carry_val = nullptr;    // [n_tiles] its partial sum within the tile
    float* d_xs = nullptr;           // [cols] x times the column scale
};

namespace fd2 {

constexpr int kSpmvThreads = 256;
constexpr int kSpmvItems = 8;  // merge items (row ends + nonzeros) per thread
constexpr int kSpmvTile = kSpmvThreads * kSpmvItems;

inline size_t value_size(int vt) { return vt == FD2_VALUES_F32 ? 4 : 2; }

// Allocates the plan buffers and computes the tile coordinates (after d_off is set).
int matrix_plan(fd2_matrix* m, cudaStream_t stream);
// Allocates d_off/d_col/d_val (and d_scale when scale_axis != NONE) for the sizes in m.
int matrix_alloc(fd2_matrix* m);
void matrix_free(fd2_matrix* m);
// y = M x on `stream`.  Not re-entrant per matrix: a column-scaled matrix
// stages the scaled x in its own buffer.
int matrix_spmv(const fd2_matrix* m, const float* d_x, float* d_y, cudaStream_t stream);
// The context a dose-loading matrix was built on.
fd2_context* ensemble_context(const fd2_csr_ensemble* e);

}  // namespace fd2
