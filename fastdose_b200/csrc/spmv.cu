// spmv.cu -- device CSR matrices of the optimizer and their products.
//
// The reference multiplies with cusparseSpMV on 64-bit-index FP32 CSR
// (IMRT::MatCSR64, IMRTOpt/include/IMRTDoseMat.cuh:29-69).  Here a matrix
// holds int64 row offsets, int32 columns and FP32/FP16/BF16 values, and the
// product is a merge-path SpMV: the sequence of row ends + nonzeros is cut
// into equal tiles of kSpmvTile items, so every block streams the same number
// of matrix bytes whatever the row lengths (VOI rows of a few hundred
// nonzeros, beamlet rows of tens of thousands, empty rows).  A tile stages its
// products val * x[col] in shared memory with independent, coalesced
// streaming loads, each thread walks kSpmvItems items of the tile's merge
// path, a block reduce-by-key scan joins the partial sums of rows that span
// threads, and a second kernel adds the carries of rows that span tiles, in
// tile order.  Summation order depends only on the matrix, so products are
// reproducible run to run.  The product is HBM-bound: a pass reads
// nnz * (value + 4-byte column) bytes plus the offsets, while x (a few hundred
// KB to a few tens of MB) stays in L2.
#include <algorithm>
#include <cmath>
#include <vector>

#include <cub/block/block_scan.cuh>
#include <cub/device/device_radix_sort.cuh>

#include "opt_internal.cuh"

namespace fd2 {

namespace {

__device__ __forceinline__ float load_value(const float* v, int64_t k) { return __ldcs(v + k); }
__device__ __forceinline__ float load_value(const __half* v, int64_t k) {
    return __half2float(__ushort_as_half(__ldcs(reinterpret_cast<const unsigned short*>(v) + k)));
}
__device__ __forceinline__ float load_value(const __nv_bfloat16* v, int64_t k) {
    return __bfloat162float(__ushort_as_bfloat16(__ldcs(reinterpret_cast<const unsigned short*>(v) + k)));
}

// Merge-path coordinate of a diagonal: rows consumed = the number of row ends
// (offsets[1..rows]) that come before nonzero (diag - rows consumed).  A row
// end is consumed before the nonzero with the same index.
__global__ void spmv_plan_kernel(const int64_t* __restrict__ off, int64_t rows, int64_t nnz, int64_t n_tiles,
                                 int64_t* __restrict__ tile_row, int64_t* __restrict__ tile_nz) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t > n_tiles) return;
    const int64_t diag = min(t * (int64_t)kSpmvTile, rows + nnz);
    int64_t lo = max(diag - nnz, (int64_t)0), hi = min(diag, rows);
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (off[mid + 1] <= diag - 1 - mid)
            lo = mid + 1;
        else
            hi = mid;
    }
    tile_row[t] = lo;
    tile_nz[t] = diag - lo;
}

struct RowCarry {
    int key;  // tile-relative row
    float value;
};

struct CarryJoin {  // reduce-by-key: sums runs of equal keys
    __device__ __forceinline__ RowCarry operator()(const RowCarry& a, const RowCarry& b) const {
        return b.key == a.key ? RowCarry{b.key, a.value + b.value} : b;
    }
};

template <typename T>
__global__ void __launch_bounds__(kSpmvThreads) spmv_tile_kernel(
    const int64_t* __restrict__ off, const int32_t* __restrict__ col, const T* __restrict__ val,
    const float* __restrict__ x, const float* __restrict__ row_scale, const int64_t* __restrict__ tile_row,
    const int64_t* __restrict__ tile_nz, float* __restrict__ y, int64_t* __restrict__ carry_row,
    float* __restrict__ carry_val) {
    __shared__ float s_prod[kSpmvTile];
    __shared__ int s_rowend[kSpmvTile + 1];
    typedef cub::BlockScan<RowCarry, kSpmvThreads> Scan;
    __shared__ typename Scan::TempStorage scan_tmp;

    const int64_t t = blockIdx.x;
    const int64_t r0 = tile_row[t], z0 = tile_nz[t];
    const int nr = (int)(tile_row[t + 1] - r0), nz = (int)(tile_nz[t + 1] - z0);

    // stage the tile's row ends (relative to z0) and products
    for (int i = threadIdx.x; i < nr; i += kSpmvThreads) s_rowend[i] = (int)(off[r0 + i + 1] - z0);
    if (threadIdx.x == 0) s_rowend[nr] = nz + 1;  // the row in progress at the tile end does not end here
    {
        int c[kSpmvItems];
        float v[kSpmvItems];
#pragma unroll
        for (int u = 0; u < kSpmvItems; u++) {
            const int j = u * kSpmvThreads + threadIdx.x;
            c[u] = 0;
            v[u] = 0.0f;
            if (j < nz) {
                c[u] = __ldcs(col + z0 + j);
                v[u] = load_value(val, z0 + j);
            }
        }
#pragma unroll
        for (int u = 0; u < kSpmvItems; u++) {
            const int j = u * kSpmvThreads + threadIdx.x;
            if (j < nz) s_prod[j] = v[u] * __ldg(x + c[u]);
        }
    }
    __syncthreads();

    // this thread's stretch of the tile's merge path
    const int total = nr + nz;
    const int diag = min((int)threadIdx.x * kSpmvItems, total);
    const int dend = min(diag + kSpmvItems, total);
    int lo = max(diag - nz, 0), hi = min(diag, nr);
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (s_rowend[mid] <= diag - 1 - mid)
            lo = mid + 1;
        else
            hi = mid;
    }
    int i = lo, j = diag - lo;
    float run = 0.0f, first_val = 0.0f;
    int first_row = -1;
    for (int it = diag; it < dend; it++) {
        if (j < s_rowend[i]) {
            run += s_prod[j];
            j++;
        } else {
            if (first_row < 0) {
                first_row = i;
                first_val = run;
            } else {
                const int64_t r = r0 + i;
                y[r] = row_scale ? row_scale[r] * run : run;
            }
            run = 0.0f;
            i++;
        }
    }
    // the first row this thread ends also holds the trailing partial sums of
    // the threads before it that carried the same row
    RowCarry mine{i, run}, prefix, total_carry;
    Scan(scan_tmp).ExclusiveScan(mine, prefix, RowCarry{-1, 0.0f}, CarryJoin(), total_carry);
    if (first_row >= 0) {
        const float v = first_val + (prefix.key == first_row ? prefix.value : 0.0f);
        const int64_t r = r0 + first_row;
        y[r] = row_scale ? row_scale[r] * v : v;
    }
    if (threadIdx.x == 0) {
        carry_row[t] = r0 + total_carry.key;
        carry_val[t] = total_carry.value;
    }
}

// Adds the carries of rows that span tiles: the first tile of each run of
// equal carry rows sums the run in tile order.
__global__ void spmv_fixup_kernel(int64_t n_tiles, const int64_t* __restrict__ carry_row,
                                  const float* __restrict__ carry_val, const float* __restrict__ row_scale,
                                  int64_t rows, float* __restrict__ y) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n_tiles) return;
    const int64_t r = carry_row[t];
    if (r >= rows || (t > 0 && carry_row[t - 1] == r)) return;
    float s = 0.0f;
    for (int64_t u = t; u < n_tiles && carry_row[u] == r; u++) s += carry_val[u];
    y[r] += row_scale ? row_scale[r] * s : s;
}

__global__ void scale_vector_kernel(const float* __restrict__ s, const float* __restrict__ x, float* __restrict__ out,
                                    int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = s[i] * x[i];
}

// ---------------------------------------------------------------- creation
__global__ void abs_max_by_column(const int32_t* __restrict__ col, const float* __restrict__ v, int64_t nnz,
                                  unsigned* __restrict__ mx) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
        atomicMax(mx + col[k], __float_as_uint(fabsf(v[k])));  // order-free on non-negative floats
}

__global__ void finish_scale(const unsigned* __restrict__ mx, float* __restrict__ s, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float m = __uint_as_float(mx[i]);
        s[i] = m > 0.0f ? m : 1.0f;
    }
}

template <typename T>
__device__ __forceinline__ T from_float(float v);
template <>
__device__ __forceinline__ __half from_float<__half>(float v) {
    return __float2half_rn(v);
}
template <>
__device__ __forceinline__ __nv_bfloat16 from_float<__nv_bfloat16>(float v) {
    return __float2bfloat16_rn(v);
}

template <typename T>
__global__ void quantize_by_column(const int32_t* __restrict__ col, const float* __restrict__ v,
                                   const float* __restrict__ s, int64_t nnz, T* __restrict__ out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
        out[k] = from_float<T>(__fdiv_rn(v[k], s[col[k]]));
}

// row holding nonzero k: the last row whose offset is <= k
__device__ __forceinline__ int64_t row_of(const int64_t* __restrict__ off, int64_t rows, int64_t k) {
    int64_t lo = 0, hi = rows;
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (off[mid] <= k) lo = mid; else hi = mid;
    }
    return lo;
}

// to FP32 with the scale applied
template <typename T>
__global__ void dequantize(const int64_t* __restrict__ off, int64_t rows, const int32_t* __restrict__ col,
                           const T* __restrict__ val, const float* __restrict__ s, int axis, int64_t nnz,
                           float* __restrict__ out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
        float v = load_value(val, k);
        if (axis == FD2_SCALE_COLS)
            v *= s[col[k]];
        else if (axis == FD2_SCALE_ROWS)
            v *= s[row_of(off, rows, k)];
        out[k] = v;
    }
}

// ---------------------------------------------------------------- transpose
__global__ void iota64(int64_t* __restrict__ p, int64_t n) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        p[k] = k;
}

// new offsets: first sorted position whose key is >= c
__global__ void offsets_from_sorted(const int32_t* __restrict__ keys, int64_t nnz, int64_t n_rows_new,
                                    int64_t* __restrict__ off) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c <= n_rows_new;
         c += (int64_t)gridDim.x * blockDim.x) {
        int64_t lo = 0, hi = nnz;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (keys[mid] < c) lo = mid + 1; else hi = mid;
        }
        off[c] = lo;
    }
}

template <typename T>
__global__ void gather_transposed(const int64_t* __restrict__ off, int64_t rows, const int64_t* __restrict__ perm,
                                  const T* __restrict__ val, int64_t nnz, int32_t* __restrict__ col_out,
                                  T* __restrict__ val_out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t src = perm[k];
        col_out[k] = (int32_t)row_of(off, rows, src);
        val_out[k] = val[src];
    }
}

unsigned grid_for(int64_t n, int threads = 256) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 16));
}

template <typename T>
int launch_spmv(const fd2_matrix* m, const float* x, float* y, cudaStream_t st) {
    const float* rs = m->scale_axis == FD2_SCALE_ROWS ? m->d_scale : nullptr;
    spmv_tile_kernel<T><<<(unsigned)m->n_tiles, kSpmvThreads, 0, st>>>(
        m->d_off, m->d_col, (const T*)m->d_val, x, rs, m->d_tile_row, m->d_tile_nz, y, m->d_carry_row,
        m->d_carry_val);
    FD2_CHECK_CUDA(cudaGetLastError());
    spmv_fixup_kernel<<<grid_for(m->n_tiles), 256, 0, st>>>(m->n_tiles, m->d_carry_row, m->d_carry_val, rs, m->rows,
                                                             y);
    FD2_CHECK_CUDA(cudaGetLastError());
    return FD2_OK;
}

template <typename T>
int transpose_typed(const fd2_matrix* m, fd2_matrix* t, cudaStream_t st) {
    const int64_t nnz = m->nnz;
    int32_t* keys_out = nullptr;
    int64_t *perm_in = nullptr, *perm_out = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    int end_bit = 1;
    while (end_bit < 31 && ((int64_t)1 << end_bit) < m->cols) end_bit++;
    int rc = FD2_OK;
    cudaError_t e = cudaMalloc(&keys_out, nnz * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&perm_in, nnz * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMalloc(&perm_out, nnz * sizeof(int64_t));
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, m->d_col, keys_out, perm_in, perm_out, nnz, 0, end_bit,
                                            st);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tmp_bytes);
    if (e == cudaSuccess) {
        // stable sort by column: within a new row, entries keep ascending old-row order
        iota64<<<grid_for(nnz), 256, 0, st>>>(perm_in, nnz);
        e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, m->d_col, keys_out, perm_in, perm_out, nnz, 0, end_bit,
                                            st);
    }
    if (e == cudaSuccess) {
        offsets_from_sorted<<<grid_for(t->rows + 1), 256, 0, st>>>(keys_out, nnz, t->rows, t->d_off);
        gather_transposed<T><<<grid_for(nnz), 256, 0, st>>>(m->d_off, m->rows, perm_out, (const T*)m->d_val, nnz,
                                                            t->d_col, (T*)t->d_val);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error("matrix_transpose: %s", cudaGetErrorString(e));
        rc = e == cudaErrorMemoryAllocation ? FD2_ERR_OUT_OF_MEMORY : FD2_ERR_CUDA;
    }
    for (void* p : {(void*)keys_out, (void*)perm_in, (void*)perm_out, tmp})
        if (p) cudaFree(p);
    return rc;
}

}  // namespace

int matrix_alloc(fd2_matrix* m) {
    FD2_CHECK_CUDA(cudaMalloc(&m->d_off, (m->rows + 1) * sizeof(int64_t)));
    FD2_CHECK_CUDA(cudaMalloc(&m->d_col, std::max<int64_t>(m->nnz, 1) * sizeof(int32_t)));
    FD2_CHECK_CUDA(cudaMalloc(&m->d_val, std::max<int64_t>(m->nnz, 1) * value_size(m->value_type)));
    if (m->scale_axis != FD2_SCALE_NONE) {
        const int64_t n = m->scale_axis == FD2_SCALE_ROWS ? m->rows : m->cols;
        FD2_CHECK_CUDA(cudaMalloc(&m->d_scale, std::max<int64_t>(n, 1) * sizeof(float)));
    }
    return FD2_OK;
}

void matrix_free(fd2_matrix* m) {
    for (void* p : {(void*)m->d_off, (void*)m->d_col, m->d_val, (void*)m->d_scale, (void*)m->d_tile_row,
                    (void*)m->d_tile_nz, (void*)m->d_carry_row, (void*)m->d_carry_val, (void*)m->d_xs})
        if (p) cudaFree(p);
    m->d_off = nullptr;
    m->d_col = nullptr;
    m->d_val = nullptr;
    m->d_scale = nullptr;
    m->d_tile_row = m->d_tile_nz = m->d_carry_row = nullptr;
    m->d_carry_val = m->d_xs = nullptr;
}

int matrix_plan(fd2_matrix* m, cudaStream_t st) {
    const int64_t items = m->rows + m->nnz;
    m->n_tiles = (items + kSpmvTile - 1) / kSpmvTile;
    FD2_CHECK_CUDA(cudaMalloc(&m->d_tile_row, (m->n_tiles + 1) * sizeof(int64_t)));
    FD2_CHECK_CUDA(cudaMalloc(&m->d_tile_nz, (m->n_tiles + 1) * sizeof(int64_t)));
    FD2_CHECK_CUDA(cudaMalloc(&m->d_carry_row, std::max<int64_t>(m->n_tiles, 1) * sizeof(int64_t)));
    FD2_CHECK_CUDA(cudaMalloc(&m->d_carry_val, std::max<int64_t>(m->n_tiles, 1) * sizeof(float)));
    if (m->scale_axis == FD2_SCALE_COLS)
        FD2_CHECK_CUDA(cudaMalloc(&m->d_xs, std::max<int64_t>(m->cols, 1) * sizeof(float)));
    spmv_plan_kernel<<<(unsigned)((m->n_tiles + 1 + 255) / 256), 256, 0, st>>>(m->d_off, m->rows, m->nnz, m->n_tiles,
                                                                              m->d_tile_row, m->d_tile_nz);
    FD2_CHECK_CUDA(cudaGetLastError());
    return FD2_OK;
}

int matrix_spmv(const fd2_matrix* m, const float* x, float* y, cudaStream_t st) {
    if (m->rows == 0) return FD2_OK;
    if (m->scale_axis == FD2_SCALE_COLS) {
        scale_vector_kernel<<<grid_for(m->cols), 256, 0, st>>>(m->d_scale, x, m->d_xs, m->cols);
        FD2_CHECK_CUDA(cudaGetLastError());
        x = m->d_xs;
        m->ctx->launches += 1;
    }
    m->ctx->launches += 2;
    switch (m->value_type) {
        case FD2_VALUES_F16: return launch_spmv<__half>(m, x, y, st);
        case FD2_VALUES_BF16: return launch_spmv<__nv_bfloat16>(m, x, y, st);
        default: return launch_spmv<float>(m, x, y, st);
    }
}

}  // namespace fd2

using namespace fd2;

extern "C" {

int fd2_matrix_create(fd2_context* ctx, int64_t rows, int64_t cols, int64_t nnz, const int64_t* h_off,
                      const int64_t* h_col, const float* h_val, int value_type, fd2_matrix** out) {
    FD2_REQUIRE(ctx && h_off && out && (nnz == 0 || (h_col && h_val)), FD2_ERR_INVALID_ARGUMENT,
                "matrix_create: null argument");
    FD2_REQUIRE(rows >= 0 && cols >= 0 && nnz >= 0 && cols < ((int64_t)1 << 31), FD2_ERR_INVALID_ARGUMENT,
                "matrix_create: sizes rows=%lld cols=%lld nnz=%lld", (long long)rows, (long long)cols,
                (long long)nnz);
    FD2_REQUIRE(value_type >= FD2_VALUES_F32 && value_type <= FD2_VALUES_BF16, FD2_ERR_INVALID_ARGUMENT,
                "matrix_create: value type %d", value_type);
    FD2_REQUIRE(h_off[0] == 0 && h_off[rows] == nnz, FD2_ERR_INVALID_ARGUMENT,
                "matrix_create: offsets must run from 0 to nnz");
    for (int64_t r = 0; r < rows; r++)
        FD2_REQUIRE(h_off[r + 1] >= h_off[r], FD2_ERR_INVALID_ARGUMENT, "matrix_create: offsets decrease at row %lld",
                    (long long)r);
    std::vector<int32_t> col32(nnz);
    for (int64_t k = 0; k < nnz; k++) {
        FD2_REQUIRE(h_col[k] >= 0 && h_col[k] < cols, FD2_ERR_INVALID_ARGUMENT,
                    "matrix_create: column %lld out of range at %lld", (long long)h_col[k], (long long)k);
        col32[k] = (int32_t)h_col[k];
    }
    auto* m = new fd2_matrix();
    m->ctx = ctx;
    m->rows = rows;
    m->cols = cols;
    m->nnz = nnz;
    m->value_type = value_type;
    m->scale_axis = value_type == FD2_VALUES_F32 ? FD2_SCALE_NONE : FD2_SCALE_COLS;
    cudaStream_t st = ctx->stream;
    float* d_f = nullptr;
    unsigned* d_mx = nullptr;
    auto fail = [&](int rc) {
        if (d_f) cudaFree(d_f);
        if (d_mx) cudaFree(d_mx);
        matrix_free(m);
        delete m;
        return rc;
    };
    int rc = matrix_alloc(m);
    if (rc) return fail(rc);
    cudaError_t e = cudaMemcpyAsync(m->d_off, h_off, (rows + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nnz)
        e = cudaMemcpyAsync(m->d_col, col32.data(), nnz * sizeof(int32_t), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && value_type == FD2_VALUES_F32) {
        if (nnz) e = cudaMemcpyAsync(m->d_val, h_val, nnz * sizeof(float), cudaMemcpyHostToDevice, st);
    } else if (e == cudaSuccess) {
        const int64_t nc = std::max<int64_t>(cols, 1);
        e = cudaMalloc(&d_mx, nc * sizeof(unsigned));
        if (e == cudaSuccess) e = cudaMemsetAsync(d_mx, 0, nc * sizeof(unsigned), st);
        if (e == cudaSuccess && nnz) {
            e = cudaMalloc(&d_f, nnz * sizeof(float));
            if (e == cudaSuccess) e = cudaMemcpyAsync(d_f, h_val, nnz * sizeof(float), cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) abs_max_by_column<<<grid_for(nnz), 256, 0, st>>>(m->d_col, d_f, nnz, d_mx);
        }
        if (e == cudaSuccess) finish_scale<<<grid_for(cols), 256, 0, st>>>(d_mx, m->d_scale, cols);
        if (e == cudaSuccess && nnz) {
            if (value_type == FD2_VALUES_F16)
                quantize_by_column<__half>
                    <<<grid_for(nnz), 256, 0, st>>>(m->d_col, d_f, m->d_scale, nnz, (__half*)m->d_val);
            else
                quantize_by_column<__nv_bfloat16>
                    <<<grid_for(nnz), 256, 0, st>>>(m->d_col, d_f, m->d_scale, nnz, (__nv_bfloat16*)m->d_val);
        }
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_error("matrix_create: %s", cudaGetErrorString(e));
        return fail(e == cudaErrorMemoryAllocation ? FD2_ERR_OUT_OF_MEMORY : FD2_ERR_CUDA);
    }
    rc = matrix_plan(m, st);
    if (rc) return fail(rc);
    e = cudaStreamSynchronize(st);  // the host staging buffers must outlive the copies
    if (e != cudaSuccess) {
        set_error("matrix_create: %s", cudaGetErrorString(e));
        return fail(FD2_ERR_CUDA);
    }
    if (d_f) cudaFree(d_f);
    if (d_mx) cudaFree(d_mx);
    *out = m;
    return FD2_OK;
}

int fd2_matrix_destroy(fd2_matrix* m) {
    if (!m) return FD2_OK;
    matrix_free(m);
    delete m;
    return FD2_OK;
}

int fd2_matrix_info(const fd2_matrix* m, fd2_matrix_info_t* info) {
    FD2_REQUIRE(m && info, FD2_ERR_INVALID_ARGUMENT, "matrix_info: null argument");
    info->rows = m->rows;
    info->cols = m->cols;
    info->nnz = m->nnz;
    info->value_type = m->value_type;
    info->scale_axis = m->scale_axis;
    const int64_t ns = m->scale_axis == FD2_SCALE_ROWS ? m->rows : m->scale_axis == FD2_SCALE_COLS ? m->cols : 0;
    info->device_bytes =
        (m->rows + 1) * 8 + m->nnz * (4 + (int64_t)value_size(m->value_type)) + ns * (int64_t)sizeof(float);
    return FD2_OK;
}

int fd2_matrix_to_host(const fd2_matrix* m, int64_t* h_off, int32_t* h_col, float* h_val) {
    FD2_REQUIRE(m && h_off && (m->nnz == 0 || (h_col && h_val)), FD2_ERR_INVALID_ARGUMENT,
                "matrix_to_host: null argument");
    cudaStream_t st = m->ctx->stream;
    FD2_CHECK_CUDA(cudaMemcpyAsync(h_off, m->d_off, (m->rows + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    if (m->nnz) {
        FD2_CHECK_CUDA(cudaMemcpyAsync(h_col, m->d_col, m->nnz * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        float* d_f = nullptr;
        FD2_CHECK_CUDA(cudaMalloc(&d_f, m->nnz * sizeof(float)));
        switch (m->value_type) {
            case FD2_VALUES_F16:
                dequantize<__half><<<grid_for(m->nnz), 256, 0, st>>>(m->d_off, m->rows, m->d_col,
                                                                     (const __half*)m->d_val, m->d_scale,
                                                                     m->scale_axis, m->nnz, d_f);
                break;
            case FD2_VALUES_BF16:
                dequantize<__nv_bfloat16><<<grid_for(m->nnz), 256, 0, st>>>(
                    m->d_off, m->rows, m->d_col, (const __nv_bfloat16*)m->d_val, m->d_scale, m->scale_axis, m->nnz,
                    d_f);
                break;
            default:
                dequantize<float><<<grid_for(m->nnz), 256, 0, st>>>(m->d_off, m->rows, m->d_col,
                                                                    (const float*)m->d_val, m->d_scale,
                                                                    m->scale_axis, m->nnz, d_f);
        }
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_val, d_f, m->nnz * sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(d_f);
        FD2_CHECK_CUDA(e);
    }
    FD2_CHECK_CUDA(cudaStreamSynchronize(st));
    return FD2_OK;
}

int fd2_matrix_transpose(const fd2_matrix* m, fd2_matrix** out) {
    FD2_REQUIRE(m && out, FD2_ERR_INVALID_ARGUMENT, "matrix_transpose: null argument");
    FD2_REQUIRE(m->rows < ((int64_t)1 << 31), FD2_ERR_INVALID_ARGUMENT,
                "matrix_transpose: %lld rows do not fit int32 columns", (long long)m->rows);
    auto* t = new fd2_matrix();
    t->ctx = m->ctx;
    t->rows = m->cols;
    t->cols = m->rows;
    t->nnz = m->nnz;
    t->value_type = m->value_type;
    t->scale_axis = m->scale_axis == FD2_SCALE_ROWS   ? FD2_SCALE_COLS
                    : m->scale_axis == FD2_SCALE_COLS ? FD2_SCALE_ROWS
                                                      : FD2_SCALE_NONE;
    cudaStream_t st = m->ctx->stream;
    int rc = matrix_alloc(t);
    if (rc == FD2_OK && t->d_scale) {
        const int64_t ns = t->scale_axis == FD2_SCALE_ROWS ? t->rows : t->cols;
        if (ns && cudaMemcpyAsync(t->d_scale, m->d_scale, ns * sizeof(float), cudaMemcpyDeviceToDevice, st) !=
                      cudaSuccess)
            rc = FD2_ERR_CUDA;
    }
    if (rc == FD2_OK) {
        if (m->nnz == 0) {
            rc = cudaMemsetAsync(t->d_off, 0, (t->rows + 1) * sizeof(int64_t), st) == cudaSuccess ? FD2_OK
                                                                                                  : FD2_ERR_CUDA;
        } else {
            switch (m->value_type) {
                case FD2_VALUES_F16: rc = transpose_typed<__half>(m, t, st); break;
                case FD2_VALUES_BF16: rc = transpose_typed<__nv_bfloat16>(m, t, st); break;
                default: rc = transpose_typed<float>(m, t, st);
            }
        }
    }
    if (rc == FD2_OK) rc = matrix_plan(t, st);
    if (rc == FD2_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = FD2_ERR_CUDA;
    if (rc) {
        matrix_free(t);
        delete t;
        return rc;
    }
    *out = t;
    return FD2_OK;
}

int fd2_matrix_spmv(const fd2_matrix* m, const float* d_x, float* d_y, void* stream) {
    FD2_REQUIRE(m && d_y && (m->cols == 0 || d_x), FD2_ERR_INVALID_ARGUMENT, "matrix_spmv: null argument");
    return matrix_spmv(m, d_x, d_y, (cudaStream_t)stream);
}

}  // extern "C"
