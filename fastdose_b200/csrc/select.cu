// select.cu -- beam selection on device matrices.
//
// The reference's beam-orientation loop rebuilds the active beams' matrices
// on the host at every prune phase: parallelMatCoalesce stacks the active
// beams' VOIMatricesT rows and transposes, diagBlock stacks their fluence
// gradients (IMRTOptimize.cu:278-300, IMRTEigenLoad.cpp:190-304), and
// Eigen2Cusparse uploads the result.  Here the full matrices stay on the device
// and a selection copies the kept row blocks, in the kept order, into a new
// matrix: for Aᵀ the blocks are beams (their beamlet rows); for the
// block-diagonal D the columns are renumbered block by block as well.  Values
// move unchanged (no re-rounding of 16-bit values); the plan of the new matrix
// is built by matrix_finalize.
#include <algorithm>
#include <vector>

#include "opt_internal.cuh"

namespace fd2 {

namespace {

// One warp per kept row: its entries in logical order, the column moved by the
// row's block shift.  A column outside [lo, hi) of its block (a matrix that is
// not block-diagonal as declared) is counted in *bad.
template <typename T>
__global__ void select_rows_kernel(const int64_t* __restrict__ src_off, ColView cv, const T* __restrict__ src_val,
                                   const int64_t* __restrict__ map_row, const int32_t* __restrict__ shift,
                                   const int32_t* __restrict__ lo, const int32_t* __restrict__ hi,
                                   const int64_t* __restrict__ dst_off, int64_t new_rows,
                                   int32_t* __restrict__ dst_col, T* __restrict__ dst_val, int* __restrict__ bad) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < new_rows; r += warps) {
        const int64_t s = map_row[r];
        const int64_t a = src_off[s], n = src_off[s + 1] - a, d = dst_off[r];
        const int sh = shift[r], l = lo[r], h = hi[r];
        for (int64_t i = lane; i < n; i += 32) {
            const int c = cv.at(a + i);
            if (c < l || c >= h) atomicAdd(bad, 1);
            dst_col[d + i] = c + sh;
            dst_val[d + i] = src_val[slot(a + i)];
        }
    }
}

__global__ void gather_scale(const float* __restrict__ src, const int64_t* __restrict__ map, int64_t n,
                             float* __restrict__ dst) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[map[i]];
}

unsigned blocks_for(int64_t n, int threads = 256) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 16));
}

}  // namespace

int matrix_select_blocks(const fd2_matrix* m, int64_t n_blocks, const int64_t* h_rows, const int64_t* h_cols,
                         int64_t n_keep, const int64_t* h_order, fd2_matrix** out) {
    FD2_REQUIRE(m && h_rows && out && n_blocks >= 0 && n_keep >= 0 && (n_keep == 0 || h_order),
                FD2_ERR_INVALID_ARGUMENT, "matrix_select_blocks: bad argument");
    FD2_REQUIRE(h_rows[0] == 0 && h_rows[n_blocks] == m->rows, FD2_ERR_INVALID_ARGUMENT,
                "matrix_select_blocks: row blocks must cover the %lld rows", (long long)m->rows);
    if (h_cols)
        FD2_REQUIRE(h_cols[0] == 0 && h_cols[n_blocks] == m->cols, FD2_ERR_INVALID_ARGUMENT,
                    "matrix_select_blocks: column blocks must cover the %lld columns", (long long)m->cols);
    for (int64_t b = 0; b < n_blocks; b++) {
        FD2_REQUIRE(h_rows[b + 1] >= h_rows[b] && (!h_cols || h_cols[b + 1] >= h_cols[b]), FD2_ERR_INVALID_ARGUMENT,
                    "matrix_select_blocks: block %lld has negative size", (long long)b);
    }
    std::vector<char> seen(n_blocks, 0);
    for (int64_t j = 0; j < n_keep; j++) {
        const int64_t b = h_order[j];
        FD2_REQUIRE(b >= 0 && b < n_blocks && !seen[b], FD2_ERR_INVALID_ARGUMENT,
                    "matrix_select_blocks: order[%lld] = %lld is out of range or repeated", (long long)j,
                    (long long)b);
        seen[b] = 1;
    }
    cudaStream_t st = m->ctx->stream;
    // source row offsets on the host; the new rows, offsets, shifts and bounds
    std::vector<int64_t> src_off(m->rows + 1);
    FD2_CHECK_CUDA(cudaMemcpyAsync(src_off.data(), m->d_off, (m->rows + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost,
                                   st));
    FD2_CHECK_CUDA(cudaStreamSynchronize(st));
    int64_t new_rows = 0, new_cols = 0;
    for (int64_t j = 0; j < n_keep; j++) {
        const int64_t b = h_order[j];
        new_rows += h_rows[b + 1] - h_rows[b];
        if (h_cols) new_cols += h_cols[b + 1] - h_cols[b];
    }
    if (!h_cols) new_cols = m->cols;
    std::vector<int64_t> map_row(new_rows), dst_off(new_rows + 1, 0), map_col;
    std::vector<int32_t> shift(new_rows), lo(new_rows), hi(new_rows);
    if (h_cols && m->scale_axis == FD2_SCALE_COLS) map_col.resize(new_cols);
    int64_t r = 0, c0 = 0;
    for (int64_t j = 0; j < n_keep; j++) {
        const int64_t b = h_order[j];
        const int32_t l = h_cols ? (int32_t)h_cols[b] : 0, h = h_cols ? (int32_t)h_cols[b + 1] : (int32_t)m->cols;
        for (int64_t s = h_rows[b]; s < h_rows[b + 1]; s++, r++) {
            map_row[r] = s;
            dst_off[r + 1] = dst_off[r] + (src_off[s + 1] - src_off[s]);
            shift[r] = h_cols ? (int32_t)(c0 - l) : 0;
            lo[r] = l;
            hi[r] = h;
        }
        if (h_cols) {
            if (!map_col.empty())
                for (int64_t c = l; c < h; c++) map_col[c0 + c - l] = c;
            c0 += h - l;
        }
    }
    auto* t = new fd2_matrix();
    t->ctx = m->ctx;
    t->rows = new_rows;
    t->cols = new_cols;
    t->nnz = dst_off[new_rows];
    t->value_type = m->value_type;
    t->index_format = m->index_format;
    t->scale_axis = m->scale_axis;
    int rc = matrix_alloc(t, st);
    int64_t* d_map = nullptr;
    int64_t* d_mapc = nullptr;
    int32_t *d_shift = nullptr, *d_lo = nullptr, *d_hi = nullptr;
    int* d_bad = nullptr;
    auto dev = [&](void** p, const void* h, size_t bytes) {
        if (rc) return;
        if (cudaMalloc(p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
            rc = FD2_ERR_OUT_OF_MEMORY;
            return;
        }
        if (bytes && cudaMemcpyAsync(*p, h, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) rc = FD2_ERR_CUDA;
    };
    dev((void**)&d_map, map_row.data(), new_rows * sizeof(int64_t));
    dev((void**)&d_shift, shift.data(), new_rows * sizeof(int32_t));
    dev((void**)&d_lo, lo.data(), new_rows * sizeof(int32_t));
    dev((void**)&d_hi, hi.data(), new_rows * sizeof(int32_t));
    const int zero = 0;
    dev((void**)&d_bad, &zero, sizeof(int));
    if (!rc && cudaMemcpyAsync(t->d_off, dst_off.data(), (new_rows + 1) * sizeof(int64_t), cudaMemcpyHostToDevice,
                               st) != cudaSuccess)
        rc = FD2_ERR_CUDA;
    if (!rc && new_rows) {
        const ColView cv = m->cols_view();
        const unsigned grid = blocks_for(new_rows * 32);
        switch (m->value_type) {
            case FD2_VALUES_F16:
                select_rows_kernel<__half><<<grid, 256, 0, st>>>(m->d_off, cv, (const __half*)m->d_val, d_map, d_shift,
                                                                 d_lo, d_hi, t->d_off, new_rows, t->d_col,
                                                                 (__half*)t->d_val, d_bad);
                break;
            case FD2_VALUES_BF16:
                select_rows_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(
                    m->d_off, cv, (const __nv_bfloat16*)m->d_val, d_map, d_shift, d_lo, d_hi, t->d_off, new_rows,
                    t->d_col, (__nv_bfloat16*)t->d_val, d_bad);
                break;
            default:
                select_rows_kernel<float><<<grid, 256, 0, st>>>(m->d_off, cv, (const float*)m->d_val, d_map, d_shift,
                                                                d_lo, d_hi, t->d_off, new_rows, t->d_col,
                                                                (float*)t->d_val, d_bad);
        }
        if (cudaGetLastError() != cudaSuccess) rc = FD2_ERR_CUDA;
        m->ctx->launches += 1;
    }
    // scales follow their rows, or their columns' blocks
    if (!rc && t->d_scale) {
        if (m->scale_axis == FD2_SCALE_ROWS && new_rows) {
            gather_scale<<<blocks_for(new_rows), 256, 0, st>>>(m->d_scale, d_map, new_rows, t->d_scale);
        } else if (m->scale_axis == FD2_SCALE_COLS && new_cols) {
            if (map_col.empty()) {
                if (cudaMemcpyAsync(t->d_scale, m->d_scale, new_cols * sizeof(float), cudaMemcpyDeviceToDevice, st) !=
                    cudaSuccess)
                    rc = FD2_ERR_CUDA;
            } else {
                dev((void**)&d_mapc, map_col.data(), new_cols * sizeof(int64_t));
                if (!rc) gather_scale<<<blocks_for(new_cols), 256, 0, st>>>(m->d_scale, d_mapc, new_cols, t->d_scale);
            }
        }
        if (cudaGetLastError() != cudaSuccess) rc = FD2_ERR_CUDA;
    }
    int bad = 0;
    if (!rc && (cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess))
        rc = FD2_ERR_CUDA;
    for (void* p : {(void*)d_map, (void*)d_mapc, (void*)d_shift, (void*)d_lo, (void*)d_hi, (void*)d_bad})
        if (p) cudaFree(p);
    if (!rc && bad) {
        set_error("matrix_select_blocks: %d entries lie outside their column block (not block-diagonal)", bad);
        rc = FD2_ERR_INVALID_ARGUMENT;
    }
    if (!rc) rc = matrix_finalize(t, st);
    if (rc) {
        if (rc == FD2_ERR_CUDA) set_error("matrix_select_blocks: %s", cudaGetErrorString(cudaGetLastError()));
        matrix_free(t);
        delete t;
        return rc;
    }
    *out = t;
    return FD2_OK;
}

}  // namespace fd2

extern "C" int fd2_matrix_select_blocks(const fd2_matrix* m, int64_t n_blocks, const int64_t* h_block_rows,
                                        const int64_t* h_block_cols, int64_t n_keep, const int64_t* h_order,
                                        fd2_matrix** out) {
    return fd2::matrix_select_blocks(m, n_blocks, h_block_rows, h_block_cols, n_keep, h_order, out);
}
