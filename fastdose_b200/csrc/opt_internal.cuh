// opt_internal.cuh -- device CSR matrix of the optimizer, shared by the SpMV,
// VOI-restriction and solver translation units.
#pragma once
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "../../include/fd2_opt.h"
#include "fd2_internal.cuh"

namespace fd2 {

constexpr int kChunk = 256;           // nonzeros per SpMV chunk (32 lanes x 8)
constexpr int kChunkWords = kChunk / 32;

// Storage position of logical nonzero k.  Inside a chunk, logical element
// 32 i + l is stored at 8 l + i, so that lane l's two 16-byte loads bring it
// elements l, l + 32, ..., l + 224: each of the warp's x-gathers then covers 32
// consecutive nonzeros of the row instead of 32 elements 8 apart.
__host__ __device__ __forceinline__ int64_t slot(int64_t k) {
    const int64_t c = k / kChunk;
    const int e = (int)(k % kChunk);
    return c * kChunk + (e % 32) * 8 + e / 32;
}

// Column index of logical nonzero k in either index format (after finalize).
struct ColView {
    const int32_t* col;     // I32: [nnz_pad], storage order
    const uint16_t* col16;  // PACKED16: [nnz_pad] offset from the chunk base, storage order
    const int32_t* cbase;   // PACKED16: per chunk base, or -(1 + exception slot)
    const int32_t* exc;     // PACKED16: [slots * kChunk] columns of exception chunks, storage order
    __device__ __forceinline__ int at(int64_t k) const {
        const int64_t q = slot(k);
        if (col) return col[q];
        const int32_t b = cbase[k / kChunk];
        return b >= 0 ? b + (int)col16[q] : exc[(int64_t)(-1 - b) * kChunk + (q % kChunk)];
    }
};

inline size_t value_size(int vt) { return vt == FD2_VALUES_F32 ? 4 : 2; }
inline int64_t round_chunk(int64_t n) { return (n + kChunk - 1) / kChunk * kChunk; }

}  // namespace fd2

struct fd2_matrix {
    fd2_context* ctx = nullptr;
    int64_t rows = 0, cols = 0, nnz = 0;
    int value_type = FD2_VALUES_F32;
    int scale_axis = FD2_SCALE_NONE;
    int index_format = FD2_INDEX_I32;
    int64_t* d_off = nullptr;      // [rows + 1]
    // Builders write d_col / d_val in logical order; matrix_finalize moves them
    // to storage order (slot()), after which readers index through slot().
    int32_t* d_col = nullptr;      // I32: [nnz_pad]; PACKED16: released after packing
    uint16_t* d_col16 = nullptr;   // PACKED16: [nnz_pad]
    int32_t* d_cbase = nullptr;    // PACKED16: [n_chunks]
    int32_t* d_exc = nullptr;      // PACKED16: [n_exc * kChunk]
    int64_t n_exc = 0;
    void* d_val = nullptr;         // [nnz_pad] float / __half / __nv_bfloat16, zero past nnz
    float* d_scale = nullptr;      // [rows] or [cols] when scale_axis != NONE
    // stream SpMV plan
    int64_t n_chunks = 0;          // nnz_pad / kChunk
    uint32_t* d_head = nullptr;    // [n_chunks * kChunkWords] row starts: per chunk 32 bytes, one per
                                   // lane; bit i of byte l: element 32 i + l starts its row
    int32_t* d_chunk_h = nullptr;  // [n_chunks] row starts before the chunk
    int32_t* d_chunk_row0 = nullptr;  // [n_chunks] first row starting in the chunk if its starts are
                                      // consecutive rows, else -1 - d_chunk_h[c]
    int32_t* d_nzrow = nullptr;    // [n_nzrows] rows with nonzeros, in order
    int64_t n_nzrows = 0;
    int n_warps = 0;               // SpMV warps (contiguous chunk ranges)
    bool x_in_smem = false;        // SpMV instance: x staged in shared memory (cols small enough)
    int64_t* d_carry_row = nullptr;  // [n_warps] row open at each warp's range end
    float* d_carry_val = nullptr;    // [n_warps] its partial sum
    float* d_xs = nullptr;           // [cols] x times the column scale

    fd2::ColView cols_view() const { return fd2::ColView{d_col, d_col16, d_cbase, d_exc}; }
};

namespace fd2 {

// Allocates d_off (rows + 1), d_col (int32, nnz padded to kChunk), d_val
// (padded, zeroed past nnz) and d_scale for the sizes in m.
int matrix_alloc(fd2_matrix* m, cudaStream_t stream);
// The same without d_off (for builders that write the offsets first).
int matrix_alloc_entries(fd2_matrix* m, cudaStream_t stream);
// Builds the SpMV plan (row-start bitmap, chunk row counts, non-empty rows,
// warp partition) from d_off, and packs the columns when m->index_format is
// PACKED16.  Call once the offsets, columns and values are written.
int matrix_finalize(fd2_matrix* m, cudaStream_t stream);
void matrix_free(fd2_matrix* m);
// Transpose into a matrix of the given index format.
int matrix_transpose_fmt(const fd2_matrix* m, int index_format, fd2_matrix** out);
// Row blocks of m in a given order (fd2_matrix_select_blocks).
int matrix_select_blocks(const fd2_matrix* m, int64_t n_blocks, const int64_t* h_rows, const int64_t* h_cols,
                         int64_t n_keep, const int64_t* h_order, fd2_matrix** out);
// y = M x on `stream`.  Not re-entrant per matrix: a column-scaled matrix
// stages the scaled x, and every product its carries, in the matrix's buffers.
int matrix_spmv(const fd2_matrix* m, const float* d_x, float* d_y, cudaStream_t stream);
// The context a dose-loading matrix was built on.
fd2_context* ensemble_context(const fd2_csr_ensemble* e);
// The stream a dose-loading matrix's arrays are ordered on.
cudaStream_t ensemble_stream(const fd2_csr_ensemble* e);

}  // namespace fd2
