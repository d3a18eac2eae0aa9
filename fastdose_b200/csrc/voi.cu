// voi.cu -- optimizer matrices built on the device: the VOI restriction of a
// dose-loading matrix, and a seeded synthetic VOI matrix pair.
//
// VOI restriction replaces getStructFilter + parallelSpGEMM
// (IMRTOpt/src/IMRTEigenLoad.cu:101-273, IMRTOpt/src/IMRTEigenLoad.cpp:10-149),
// which form A_b = (MatT_b F)^T on the host with Eigen for every beam: F is
// the 0/1 filter that keeps VOI voxels (PTV rows first, then OAR rows) and
// MatT_b the beam's [beamlets x voxels] CSR.  Here one kernel pass keeps and
// renumbers the columns of every beamlet row in order, and two device
// transposes give A (VOI rows, beamlet columns ascending) and its transpose
// with ascending VOI columns -- the layouts parallelMatCoalesce assembles.
#include <algorithm>
#include <type_traits>
#include <vector>

#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>
#include <cub/device/device_scan.cuh>

#include "opt_internal.cuh"

namespace fd2 {

namespace {

constexpr int kThreads = 256;

template <typename T>
__device__ __forceinline__ float to_f(T v);
template <>
__device__ __forceinline__ float to_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }
template <>
__device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename T>
__device__ __forceinline__ T of_f(float v);
template <>
__device__ __forceinline__ float of_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ __half of_f<__half>(float v) { return __float2half_rn(v); }
template <>
__device__ __forceinline__ __nv_bfloat16 of_f<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// per beamlet row: kept entries and the largest kept |value| (source scale applied)
template <typename S>
__global__ void __launch_bounds__(kThreads) voi_count(const int64_t* __restrict__ off, const int32_t* __restrict__ col,
                                                      const S* __restrict__ val, const float* __restrict__ src_scale,
                                                      const int32_t* __restrict__ map, int64_t* __restrict__ count,
                                                      float* __restrict__ vmax) {
    typedef cub::BlockReduce<int64_t, kThreads> RC;
    typedef cub::BlockReduce<float, kThreads> RM;
    __shared__ typename RC::TempStorage tc;
    __shared__ typename RM::TempStorage tm;
    const int64_t r = blockIdx.x;
    const float s = src_scale ? src_scale[r] : 1.0f;
    int64_t c = 0;
    float m = 0.0f;
    for (int64_t k = off[r] + threadIdx.x; k < off[r + 1]; k += kThreads)
        if (map[col[k]] >= 0) {
            c++;
            m = fmaxf(m, fabsf(to_f(val[k]) * s));
        }
    c = RC(tc).Sum(c);
    m = RM(tm).Reduce(m, cub::Max());
    if (threadIdx.x == 0) {
        count[r] = c;
        vmax[r] = m;
    }
}

// Ordered compaction of the kept entries of each beamlet row.  Same value
// type in and out: the stored value (and the row scale, copied by the host)
// moves unchanged.  Otherwise the value is rescaled: source value times
// source scale, divided by the destination scale (16-bit output).
template <typename S, typename T>
__global__ void __launch_bounds__(kThreads) voi_fill(const int64_t* __restrict__ off, const int32_t* __restrict__ col,
                                                     const S* __restrict__ val, const float* __restrict__ src_scale,
                                                     const int32_t* __restrict__ map,
                                                     const float* __restrict__ dst_scale,
                                                     const int64_t* __restrict__ out_off, int32_t* __restrict__ out_col,
                                                     T* __restrict__ out_val) {
    typedef cub::BlockScan<int, kThreads> Scan;
    __shared__ typename Scan::TempStorage ts;
    const int64_t r = blockIdx.x;
    const float s = src_scale ? src_scale[r] : 1.0f;
    const float ds = dst_scale ? dst_scale[r] : 1.0f;
    int64_t w = out_off[r];
    for (int64_t k0 = off[r]; k0 < off[r + 1]; k0 += kThreads) {
        const int64_t k = k0 + threadIdx.x;
        int m = -1;
        if (k < off[r + 1]) m = map[col[k]];
        int pos, total;
        Scan(ts).ExclusiveSum(m >= 0 ? 1 : 0, pos, total);
        if (m >= 0) {
            out_col[w + pos] = m;
            if constexpr (std::is_same<S, T>::value) {
                out_val[w + pos] = val[k];
            } else {
                float v = to_f(val[k]) * s;
                if (dst_scale) v = __fdiv_rn(v, ds);
                out_val[w + pos] = of_f<T>(v);
            }
        }
        w += total;
        __syncthreads();
    }
}

__global__ void unit_or_max(const float* __restrict__ mx, float* __restrict__ s, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s[i] = mx[i] > 0.0f ? mx[i] : 1.0f;
}

// ------------------------------------------------------------ synthetic pair
struct SynthSpec {
    int64_t rows, cols, window;
    uint32_t keep_below;  // 24-bit threshold
    uint64_t seed;
};

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ int64_t synth_centre(const SynthSpec& sp, int64_t j) {
    return (int64_t)(((double)j + 0.5) * (double)sp.rows / (double)sp.cols);
}
__device__ __forceinline__ int64_t synth_start(const SynthSpec& sp, int64_t j) {
    return synth_centre(sp, j) - sp.window / 2;
}
__device__ __forceinline__ bool synth_keep(const SynthSpec& sp, int64_t r, int64_t j, uint64_t& h) {
    h = mix64(sp.seed ^ mix64((uint64_t)r * 0x9e3779b97f4a7c15ull + (uint64_t)j));
    return (uint32_t)(h >> 40) < sp.keep_below;
}
// Value of a kept entry: a Lorentzian fall-off with the distance from the
// window centre times a hashed factor in [0.25, 1); IEEE operations only, so
// every kernel that evaluates it gets the same bits.
__device__ __forceinline__ float synth_value(const SynthSpec& sp, int64_t r, int64_t j, uint64_t h) {
    const float d = (float)(r - synth_centre(sp, j));
    const float q = __fdiv_rn(d, (float)sp.window * 0.25f);
    const float f = __fdiv_rn(1.0f, __fadd_rn(1.0f, __fmul_rn(q, q)));
    const float u = (float)(uint32_t)(h & 0xffffffu) * (1.0f / 16777216.0f);
    return __fmul_rn(f, __fadd_rn(0.25f, __fmul_rn(0.75f, u)));
}

// transpose side: one block per column j, over the rows of its window
__global__ void __launch_bounds__(kThreads) synth_t_count(SynthSpec sp, int64_t* __restrict__ count,
                                                          float* __restrict__ vmax) {
    typedef cub::BlockReduce<int64_t, kThreads> RC;
    typedef cub::BlockReduce<float, kThreads> RM;
    __shared__ typename RC::TempStorage tc;
    __shared__ typename RM::TempStorage tm;
    const int64_t j = blockIdx.x;
    const int64_t a = max(synth_start(sp, j), (int64_t)0), b = min(synth_start(sp, j) + sp.window, sp.rows);
    int64_t c = 0;
    float m = 0.0f;
    for (int64_t r = a + threadIdx.x; r < b; r += kThreads) {
        uint64_t h;
        if (synth_keep(sp, r, j, h)) {
            c++;
            m = fmaxf(m, synth_value(sp, r, j, h));
        }
    }
    c = RC(tc).Sum(c);
    m = RM(tm).Reduce(m, cub::Max());
    if (threadIdx.x == 0) {
        count[j] = c;
        vmax[j] = m;
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) synth_t_fill(SynthSpec sp, const float* __restrict__ scale,
                                                         const int64_t* __restrict__ off, int32_t* __restrict__ col,
                                                         T* __restrict__ val) {
    typedef cub::BlockScan<int, kThreads> Scan;
    __shared__ typename Scan::TempStorage ts;
    const int64_t j = blockIdx.x;
    const int64_t a = max(synth_start(sp, j), (int64_t)0), b = min(synth_start(sp, j) + sp.window, sp.rows);
    const float s = scale ? scale[j] : 1.0f;
    int64_t w = off[j];
    for (int64_t r0 = a; r0 < b; r0 += kThreads) {
        const int64_t r = r0 + threadIdx.x;
        uint64_t h = 0;
        const bool kept = r < b && synth_keep(sp, r, j, h);
        int pos, total;
        Scan(ts).ExclusiveSum(kept ? 1 : 0, pos, total);
        if (kept) {
            const float v = synth_value(sp, r, j, h);
            col[w + pos] = (int32_t)r;
            val[w + pos] = of_f<T>(scale ? __fdiv_rn(v, s) : v);
        }
        w += total;
        __syncthreads();
    }
}

// columns whose window holds row r: [j0, j1)
__device__ __forceinline__ void synth_cols_of_row(const SynthSpec& sp, int64_t r, int64_t& j0, int64_t& j1) {
    int64_t lo = 0, hi = sp.cols;  // first j whose window ends after r
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (synth_start(sp, mid) + sp.window > r) hi = mid; else lo = mid + 1;
    }
    j0 = lo;
    hi = sp.cols;  // first j whose window starts after r
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (synth_start(sp, mid) > r) hi = mid; else lo = mid + 1;
    }
    j1 = lo;
}

// row side: one warp per row
__global__ void synth_count(SynthSpec sp, int64_t* __restrict__ count) {
    const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= sp.rows) return;
    int64_t j0, j1;
    synth_cols_of_row(sp, r, j0, j1);
    int64_t c = 0;
    for (int64_t j = j0 + lane; j < j1; j += 32) {
        uint64_t h;
        c += synth_keep(sp, r, j, h);
    }
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) count[r] = c;
}

template <typename T>
__global__ void synth_fill(SynthSpec sp, const float* __restrict__ scale, const int64_t* __restrict__ off,
                           int32_t* __restrict__ col, T* __restrict__ val) {
    const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= sp.rows) return;
    int64_t j0, j1;
    synth_cols_of_row(sp, r, j0, j1);
    int64_t w = off[r];
    for (int64_t jb = j0; jb < j1; jb += 32) {
        const int64_t j = jb + lane;
        uint64_t h = 0;
        const bool kept = j < j1 && synth_keep(sp, r, j, h);
        const unsigned bal = __ballot_sync(0xffffffffu, kept);
        if (kept) {
            const int pos = __popc(bal & ((1u << lane) - 1u));
            const float v = synth_value(sp, r, j, h);
            col[w + pos] = (int32_t)j;
            val[w + pos] = of_f<T>(scale ? __fdiv_rn(v, scale[j]) : v);
        }
        w += __popc(bal);
    }
}

unsigned blocks_for(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

// offsets [n+1] from counts [n] (device), and the total
int offsets_from_counts(const int64_t* d_count, int64_t n, int64_t* d_off, int64_t* total, cudaStream_t st) {
    FD2_CHECK_CUDA(cudaMemsetAsync(d_off, 0, sizeof(int64_t), st));
    if (n) {
        size_t tb = 0;
        FD2_CHECK_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, d_count, d_off + 1, n, st));
        void* tmp = nullptr;
        FD2_CHECK_CUDA(cudaMalloc(&tmp, std::max<size_t>(tb, 16)));
        cudaError_t e = cub::DeviceScan::InclusiveSum(tmp, tb, d_count, d_off + 1, n, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(tmp);
        FD2_CHECK_CUDA(e);
    }
    FD2_CHECK_CUDA(cudaMemcpyAsync(total, d_off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    FD2_CHECK_CUDA(cudaStreamSynchronize(st));
    return FD2_OK;
}

template <typename S>
void voi_fill_dispatch(int dst_type, int64_t rows, const int64_t* off, const int32_t* col, const void* val,
                       const float* src_scale, const int32_t* map, const float* dst_scale, const int64_t* out_off,
                       int32_t* out_col, void* out_val, cudaStream_t st) {
    const unsigned g = (unsigned)rows;
    switch (dst_type) {
        case FD2_VALUES_F16:
            voi_fill<S, __half><<<g, kThreads, 0, st>>>(off, col, (const S*)val, src_scale, map, dst_scale, out_off,
                                                        out_col, (__half*)out_val);
            break;
        case FD2_VALUES_BF16:
            voi_fill<S, __nv_bfloat16><<<g, kThreads, 0, st>>>(off, col, (const S*)val, src_scale, map, dst_scale,
                                                               out_off, out_col, (__nv_bfloat16*)out_val);
            break;
        default:
            voi_fill<S, float><<<g, kThreads, 0, st>>>(off, col, (const S*)val, src_scale, map, dst_scale, out_off,
                                                       out_col, (float*)out_val);
    }
}

struct Guard {  // frees device buffers on scope exit
    std::vector<void*> p;
    ~Guard() {
        for (void* q : p)
            if (q) cudaFree(q);
    }
    template <typename T>
    cudaError_t alloc(T** ptr, size_t bytes) {
        cudaError_t e = cudaMalloc((void**)ptr, std::max<size_t>(bytes, 16));
        if (e == cudaSuccess) p.push_back((void*)*ptr);
        return e;
    }
};

}  // namespace

}  // namespace fd2

using namespace fd2;

extern "C" {

int fd2_voi_matrices(const fd2_csr_ensemble* dose, const int32_t* h_voxel_row, int64_t n_voxels, int64_t n_voi,
                     int value_type, int index_format, fd2_matrix** A, fd2_matrix** AT) {
    FD2_REQUIRE(dose && h_voxel_row && A && AT, FD2_ERR_INVALID_ARGUMENT, "voi_matrices: null argument");
    FD2_REQUIRE(value_type >= FD2_VALUES_F32 && value_type <= FD2_VALUES_BF16, FD2_ERR_INVALID_ARGUMENT,
                "voi_matrices: value type %d", value_type);
    FD2_REQUIRE(index_format == FD2_INDEX_I32 || index_format == FD2_INDEX_PACKED16, FD2_ERR_INVALID_ARGUMENT,
                "voi_matrices: index format %d", index_format);
    fd2_csr_info_t info;
    FD2_TRY(fd2_csr_ensemble_info(dose, &info));
    FD2_REQUIRE((int64_t)info.n_cols == n_voxels, FD2_ERR_INVALID_ARGUMENT,
                "voi_matrices: %lld voxels given, the dose matrix has %llu columns", (long long)n_voxels,
                (unsigned long long)info.n_cols);
    FD2_REQUIRE(n_voi >= 0 && n_voi < ((int64_t)1 << 31), FD2_ERR_INVALID_ARGUMENT, "voi_matrices: n_voi %lld",
                (long long)n_voi);
    for (int64_t v = 0; v < n_voxels; v++)
        FD2_REQUIRE(h_voxel_row[v] < n_voi, FD2_ERR_INVALID_ARGUMENT,
                    "voi_matrices: voxel %lld maps to row %d >= %lld", (long long)v, h_voxel_row[v], (long long)n_voi);
    const int64_t* d_off = nullptr;
    const int32_t* d_col = nullptr;
    const void* d_val = nullptr;
    const float* d_src_scale = nullptr;
    FD2_TRY(fd2_csr_ensemble_device(dose, &d_off, &d_col, &d_val, &d_src_scale, nullptr));
    fd2_context* ctx = ensemble_context(dose);
    cudaStream_t st = ctx->stream;
    FD2_CHECK_CUDA(cudaStreamSynchronize(ensemble_stream(dose)));  // the dose matrix is complete
    const int64_t rows = (int64_t)info.n_rows;
    const int src_type = info.value_type;
    if (src_type == FD2_VALUES_F32) d_src_scale = nullptr;

    Guard g;
    int32_t* d_map = nullptr;
    int64_t* d_count = nullptr;
    float* d_max = nullptr;
    FD2_CHECK_CUDA(g.alloc(&d_map, n_voxels * sizeof(int32_t)));
    FD2_CHECK_CUDA(g.alloc(&d_count, rows * sizeof(int64_t)));
    FD2_CHECK_CUDA(g.alloc(&d_max, rows * sizeof(float)));
    FD2_CHECK_CUDA(cudaMemcpyAsync(d_map, h_voxel_row, n_voxels * sizeof(int32_t), cudaMemcpyHostToDevice, st));

    auto* t = new fd2_matrix();  // beamlet rows, VOI columns in the dose matrix's voxel order
    t->ctx = ctx;
    t->rows = rows;
    t->cols = n_voi;
    t->value_type = value_type;
    t->scale_axis = value_type == FD2_VALUES_F32 ? FD2_SCALE_NONE : FD2_SCALE_ROWS;
    auto drop = [&]() {
        matrix_free(t);
        delete t;
        t = nullptr;
    };
    auto fail = [&](int rc) {
        drop();
        return rc;
    };
    if (rows) {
        switch (src_type) {
            case FD2_VALUES_F16:
                voi_count<__half><<<(unsigned)rows, kThreads, 0, st>>>(d_off, d_col, (const __half*)d_val,
                                                                       d_src_scale, d_map, d_count, d_max);
                break;
            case FD2_VALUES_BF16:
                voi_count<__nv_bfloat16><<<(unsigned)rows, kThreads, 0, st>>>(
                    d_off, d_col, (const __nv_bfloat16*)d_val, d_src_scale, d_map, d_count, d_max);
                break;
            default:
                voi_count<float><<<(unsigned)rows, kThreads, 0, st>>>(d_off, d_col, (const float*)d_val, nullptr,
                                                                      d_map, d_count, d_max);
        }
        if (cudaGetLastError() != cudaSuccess) return fail(FD2_ERR_CUDA);
    }
    if (cudaMalloc(&t->d_off, (rows + 1) * sizeof(int64_t)) != cudaSuccess) return fail(FD2_ERR_OUT_OF_MEMORY);
    int64_t nnz = 0;
    int rc = offsets_from_counts(d_count, rows, t->d_off, &nnz, st);
    if (rc) return fail(rc);
    t->nnz = nnz;
    rc = matrix_alloc_entries(t, st);
    if (rc) return fail(rc);
    const float* dst_scale = nullptr;
    if (t->scale_axis == FD2_SCALE_ROWS) {
        if (d_src_scale && rows)  // a 16-bit source keeps its per-beamlet scale
            cudaMemcpyAsync(t->d_scale, d_src_scale, rows * sizeof(float), cudaMemcpyDeviceToDevice, st);
        else
            unit_or_max<<<blocks_for(rows), 256, 0, st>>>(d_max, t->d_scale, rows);
        dst_scale = t->d_scale;
    }
    if (rows) {
        switch (src_type) {
            case FD2_VALUES_F16:
                voi_fill_dispatch<__half>(value_type, rows, d_off, d_col, d_val, d_src_scale, d_map, dst_scale,
                                          t->d_off, t->d_col, t->d_val, st);
                break;
            case FD2_VALUES_BF16:
                voi_fill_dispatch<__nv_bfloat16>(value_type, rows, d_off, d_col, d_val, d_src_scale, d_map, dst_scale,
                                                 t->d_off, t->d_col, t->d_val, st);
                break;
            default:
                voi_fill_dispatch<float>(value_type, rows, d_off, d_col, d_val, nullptr, d_map, dst_scale, t->d_off,
                                         t->d_col, t->d_val, st);
        }
        if (cudaGetLastError() != cudaSuccess) return fail(FD2_ERR_CUDA);
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(FD2_ERR_CUDA);
    rc = matrix_finalize(t, st);  // storage order, which the transpose reads
    if (rc) return fail(rc);
    fd2_matrix *a = nullptr, *at = nullptr;
    rc = matrix_transpose_fmt(t, index_format, &a);  // VOI rows, beamlet columns ascending
    drop();
    if (rc) return rc;
    rc = matrix_transpose_fmt(a, index_format, &at);  // beamlet rows, VOI columns ascending
    if (rc) {
        fd2_matrix_destroy(a);
        return rc;
    }
    *A = a;
    *AT = at;
    return FD2_OK;
}

int fd2_matrix_synthetic(fd2_context* ctx, int64_t rows, int64_t cols, int64_t window, float density, uint64_t seed,
                         int value_type, int index_format, fd2_matrix** A, fd2_matrix** AT) {
    FD2_REQUIRE(ctx && A && AT, FD2_ERR_INVALID_ARGUMENT, "matrix_synthetic: null argument");
    FD2_REQUIRE(index_format == FD2_INDEX_I32 || index_format == FD2_INDEX_PACKED16, FD2_ERR_INVALID_ARGUMENT,
                "matrix_synthetic: index format %d", index_format);
    FD2_REQUIRE(rows > 0 && cols > 0 && rows < ((int64_t)1 << 31) && cols < ((int64_t)1 << 31) && window > 0 &&
                    density > 0.0f && density <= 1.0f,
                FD2_ERR_INVALID_ARGUMENT, "matrix_synthetic: rows %lld cols %lld window %lld density %g",
                (long long)rows, (long long)cols, (long long)window, (double)density);
    FD2_REQUIRE(value_type >= FD2_VALUES_F32 && value_type <= FD2_VALUES_BF16, FD2_ERR_INVALID_ARGUMENT,
                "matrix_synthetic: value type %d", value_type);
    SynthSpec sp{rows, cols, window, (uint32_t)std::min(16777216.0, (double)density * 16777216.0), seed};
    cudaStream_t st = ctx->stream;
    const bool half = value_type != FD2_VALUES_F32;
    fd2_matrix* m[2] = {new fd2_matrix(), new fd2_matrix()};  // A, AT
    auto fail = [&](int rc) {
        for (auto* q : m) {
            matrix_free(q);
            delete q;
        }
        return rc;
    };
    for (int i = 0; i < 2; i++) {
        m[i]->ctx = ctx;
        m[i]->value_type = value_type;
        m[i]->rows = i == 0 ? rows : cols;
        m[i]->cols = i == 0 ? cols : rows;
        m[i]->scale_axis = !half ? FD2_SCALE_NONE : i == 0 ? FD2_SCALE_COLS : FD2_SCALE_ROWS;
        m[i]->index_format = index_format;
    }
    Guard g;
    int64_t* d_count = nullptr;
    float* d_max = nullptr;
    if (g.alloc(&d_count, std::max(rows, cols) * sizeof(int64_t)) != cudaSuccess ||
        g.alloc(&d_max, cols * sizeof(float)) != cudaSuccess)
        return fail(FD2_ERR_OUT_OF_MEMORY);
    // transpose side first: counts and per-column maxima (the scales)
    synth_t_count<<<(unsigned)cols, kThreads, 0, st>>>(sp, d_count, d_max);
    if (cudaGetLastError() != cudaSuccess) return fail(FD2_ERR_CUDA);
    fd2_matrix* t = m[1];
    if (cudaMalloc(&t->d_off, (cols + 1) * sizeof(int64_t)) != cudaSuccess) return fail(FD2_ERR_OUT_OF_MEMORY);
    int64_t nnz = 0;
    int rc = offsets_from_counts(d_count, cols, t->d_off, &nnz, st);
    if (rc) return fail(rc);
    t->nnz = nnz;
    rc = matrix_alloc_entries(t, st);
    if (rc) return fail(rc);
    if (half) unit_or_max<<<blocks_for(cols), 256, 0, st>>>(d_max, t->d_scale, cols);
    switch (value_type) {
        case FD2_VALUES_F16:
            synth_t_fill<__half><<<(unsigned)cols, kThreads, 0, st>>>(sp, t->d_scale, t->d_off, t->d_col,
                                                                     (__half*)t->d_val);
            break;
        case FD2_VALUES_BF16:
            synth_t_fill<__nv_bfloat16><<<(unsigned)cols, kThreads, 0, st>>>(sp, t->d_scale, t->d_off, t->d_col,
                                                                             (__nv_bfloat16*)t->d_val);
            break;
        default:
            synth_t_fill<float><<<(unsigned)cols, kThreads, 0, st>>>(sp, nullptr, t->d_off, t->d_col,
                                                                    (float*)t->d_val);
    }
    if (cudaGetLastError() != cudaSuccess) return fail(FD2_ERR_CUDA);
    // row side
    fd2_matrix* a = m[0];
    const unsigned wblocks = (unsigned)((rows * 32 + 255) / 256);
    synth_count<<<wblocks, 256, 0, st>>>(sp, d_count);
    if (cudaGetLastError() != cudaSuccess) return fail(FD2_ERR_CUDA);
    if (cudaMalloc(&a->d_off, (rows + 1) * sizeof(int64_t)) != cudaSuccess) return fail(FD2_ERR_OUT_OF_MEMORY);
    int64_t nnz_a = 0;
    rc = offsets_from_counts(d_count, rows, a->d_off, &nnz_a, st);
    if (rc) return fail(rc);
    if (nnz_a != nnz) {
        set_error("matrix_synthetic: %lld vs %lld nonzeros", (long long)nnz_a, (long long)nnz);
        return fail(FD2_ERR_CUDA);
    }
    a->nnz = nnz;
    rc = matrix_alloc_entries(a, st);
    if (rc) return fail(rc);
    if (half) cudaMemcpyAsync(a->d_scale, t->d_scale, cols * sizeof(float), cudaMemcpyDeviceToDevice, st);
    switch (value_type) {
        case FD2_VALUES_F16:
            synth_fill<__half><<<wblocks, 256, 0, st>>>(sp, a->d_scale, a->d_off, a->d_col, (__half*)a->d_val);
            break;
        case FD2_VALUES_BF16:
            synth_fill<__nv_bfloat16><<<wblocks, 256, 0, st>>>(sp, a->d_scale, a->d_off, a->d_col,
                                                              (__nv_bfloat16*)a->d_val);
            break;
        default:
            synth_fill<float><<<wblocks, 256, 0, st>>>(sp, nullptr, a->d_off, a->d_col, (float*)a->d_val);
    }
    if (cudaGetLastError() != cudaSuccess) return fail(FD2_ERR_CUDA);
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(FD2_ERR_CUDA);
    for (auto* q : m) {
        rc = matrix_finalize(q, st);
        if (rc) return fail(rc);
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(FD2_ERR_CUDA);
    *A = m[0];
    *AT = m[1];
    return FD2_OK;
}

}  // extern "C"
