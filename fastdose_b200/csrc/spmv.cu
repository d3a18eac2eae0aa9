// spmv.cu -- device CSR matrices of the optimizer and their products.
//
// The reference multiplies with cusparseSpMV on 64-bit-index FP32 CSR
// (IMRT::MatCSR64, IMRTOpt/include/IMRTDoseMat.cuh:29-69).  Here a matrix
// holds int64 row offsets, int32 or packed 16-bit column indices and
// FP32/FP16/BF16 values, and the product is a stream SpMV:
//
//  * the nonzeros are cut into chunks of 256 (32 lanes x 8); every warp owns
//    a contiguous range of chunks, so every warp streams the same number of
//    matrix bytes whatever the row lengths (VOI rows of a few hundred
//    nonzeros, beamlet rows of tens of thousands, empty rows);
//  * inside a chunk the nonzeros are stored lane-major (slot()), so a lane's
//    two 16-byte streaming loads (`ld.global.cs`: the matrix is read once, x
//    stays in the 126 MB L2) bring its 8 elements l, l+32, ..., l+224, and each
//    x-gather of the warp covers 32 consecutive nonzeros;
//  * rows are found from a row-start bitmap (1 bit per nonzero) and a per-chunk
//    count of row starts: a 32-element slice without a row start is one FMA
//    per lane into the open row; a slice with row starts closes the open row
//    with a warp sum and sums the rows inside it with a segmented warp-shuffle
//    scan -- no shared memory, no block barrier;
//  * the row open at the end of a warp's range is carried; a second kernel
//    adds carries in warp order.
//
// Summation order depends only on the matrix and the launch shape, so products
// are reproducible run to run.  A pass is HBM-bound: it reads nnz x (value +
// column) bytes, the bitmap (nnz/8 bytes) and x, and writes y.
#include <algorithm>
#include <cmath>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "opt_internal.cuh"

namespace fd2 {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kStreamThreads = 256;
constexpr int kMaxStreamWarps = 148 * 64;  // one full wave of 64 warps per SM
constexpr int kSmemThreads = 1024;          // x-in-shared-memory variant: one block per SM
constexpr int64_t kSmemXMaxBytes = 200 * 1024;

struct StreamArgs {
    const void* val;
    ColView cols;
    const uint32_t* head;
    const int32_t* chunk_h;
    const int32_t* chunk_row0;
    const int32_t* nzrow;
    const float* row_scale;
    int64_t n_chunks;
    int n_warps;
    int64_t rows;
    int64_t* carry_row;
    float* carry_val;
    int x_len;  // kSmemX: floats of x staged in shared memory
};

// A lane's share of one chunk as loaded, values and columns still packed, so
// that two chunks can be in flight per warp without holding 2 x 16 unpacked
// registers.
template <typename T, bool kPacked>
struct RawChunk {
    uint4 v[sizeof(T) == 4 ? 2 : 1];  // 8 values
    uint4 c[kPacked ? 1 : 2];         // 8 int32 columns, or 8 16-bit offsets from base
    int base;                         // kPacked: the chunk's column base; < 0: exception chunk
    int row0;                         // first row starting in the chunk, or -1 - (row starts before it)
    uint32_t h;                       // this lane's row-start bits (bit i: slice i)
};

template <typename T, bool kPacked>
__device__ __forceinline__ void load_raw(const StreamArgs& a, int64_t c, int lane, RawChunk<T, kPacked>& r) {
    const int64_t k = c * kChunk + 8 * lane;  // 16-byte aligned: k is a multiple of 8
    const uint4* vp = reinterpret_cast<const uint4*>(static_cast<const T*>(a.val) + k);
    r.v[0] = __ldcs(vp);
    if constexpr (sizeof(T) == 4) r.v[1] = __ldcs(vp + 1);
    if constexpr (kPacked) {
        r.base = __ldg(a.cols.cbase + c);  // one address for the warp
        r.c[0] = __ldcs(reinterpret_cast<const uint4*>(a.cols.col16 + k));
    } else {
        const uint4* cp = reinterpret_cast<const uint4*>(a.cols.col + k);
        r.c[0] = __ldcs(cp);
        r.c[1] = __ldcs(cp + 1);
        r.base = 0;
    }
    r.row0 = __ldg(a.chunk_row0 + c);
    r.h = __ldg(reinterpret_cast<const uint8_t*>(a.head) + c * (kChunk / 8) + lane);
}

__device__ __forceinline__ void unpack_vals(const uint4 (&u)[2], float (&o)[8]) {
    const uint32_t w[8] = {u[0].x, u[0].y, u[0].z, u[0].w, u[1].x, u[1].y, u[1].z, u[1].w};
#pragma unroll
    for (int i = 0; i < 8; i++) o[i] = __uint_as_float(w[i]);
}
template <typename H>
__device__ __forceinline__ void unpack_vals(const uint4 (&u)[1], float (&o)[8]) {
    const uint32_t w[4] = {u[0].x, u[0].y, u[0].z, u[0].w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
        float2 f;
        if constexpr (std::is_same<H, __half>::value)
            f = __half22float2(*reinterpret_cast<const __half2*>(&w[i]));
        else
            f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w[i]));
        o[2 * i] = f.x;
        o[2 * i + 1] = f.y;
    }
}

__device__ __forceinline__ void load_i32x8(const int32_t* c, int64_t k, int (&o)[8]) {
    const int4* p = reinterpret_cast<const int4*>(c + k);
    const int4 a = __ldcs(p), b = __ldcs(p + 1);
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
    o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
}

template <typename T, bool kPacked>
__device__ __forceinline__ void unpack_cols(const RawChunk<T, kPacked>& r, const ColView& cv, int64_t chunk, int lane,
                                            int (&o)[8]) {
    if constexpr (!kPacked) {
        const uint32_t w[8] = {r.c[0].x, r.c[0].y, r.c[0].z, r.c[0].w, r.c[1].x, r.c[1].y, r.c[1].z, r.c[1].w};
#pragma unroll
        for (int i = 0; i < 8; i++) o[i] = (int)w[i];
    } else if (r.base >= 0) {
        const uint32_t w[4] = {r.c[0].x, r.c[0].y, r.c[0].z, r.c[0].w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
            o[2 * i] = r.base + (int)(w[i] & 0xffffu);
            o[2 * i + 1] = r.base + (int)(w[i] >> 16);
        }
    } else {  // a chunk whose columns span 65536 or more: int32 columns in the side array
        load_i32x8(cv.exc, (int64_t)(-1 - r.base) * kChunk + 8 * lane, o);
    }
}

__device__ __forceinline__ void put(float* y, const float* rs, int r, float v) { y[r] = rs ? rs[r] * v : v; }

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// One warp per contiguous range of chunks.  In a chunk, slice i holds logical
// elements 32 i .. 32 i + 31 (one per lane); bit i of lane l's row-start byte
// flags element 32 i + l.  A slice without row starts only adds to the open
// row (one FMA per lane); a slice with row starts closes the open row (warp
// sum), sums the rows that start and end inside it with a segmented warp scan,
// and leaves its last row open.
//
// kSmemX: x is copied to shared memory first (one block of kSmemThreads per
// SM) and the gathers read it there: 32 lanes reading 32 scattered columns
// cost a few bank cycles instead of up to 32 L1 tag lookups.  With 16-bit
// values a warp loads ahead: the next chunk while it sums the current one (x
// in shared memory), or two chunks at a time (x in global memory).
template <typename T, bool kPacked, bool kSmemX>
__global__ void __launch_bounds__(kSmemX ? kSmemThreads : kStreamThreads, kSmemX ? 1 : 4)
    spmv_stream_kernel(StreamArgs a, const float* __restrict__ x, float* __restrict__ y) {
    extern __shared__ float xs[];
    if constexpr (kSmemX) {
        for (int i = threadIdx.x; i < a.x_len; i += blockDim.x) xs[i] = __ldg(x + i);
        __syncthreads();
    }
    const int lane = threadIdx.x & 31;
    const int w = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    if (w >= a.n_warps) return;  // uniform per warp
    const int64_t c0 = (int64_t)w * a.n_chunks / a.n_warps, c1 = (int64_t)(w + 1) * a.n_chunks / a.n_warps;
    float oacc = 0.0f;        // this lane's share of the open row (the row in progress), this warp's part
    bool open_valid = false;  // the warp has met an element of the open row
    int open_row = 0;
    if (c0 < c1) {
        const int hb0 = __ldg(a.chunk_h + c0);
        if (hb0 > 0 && !(__ldg(a.head + c0 * kChunkWords) & 1u)) open_row = __ldg(a.nzrow + hb0 - 1);
    }
    auto xv = [&](int col) -> float {
        if constexpr (kSmemX)
            return xs[col];
        else
            return __ldg(x + col);
    };
    // row of the chunk's j-th row start: consecutive rows need no lookup
    auto row_at = [&](const RawChunk<T, kPacked>& r, int j) -> int {
        return r.row0 >= 0 ? r.row0 + j : __ldg(a.nzrow + (-1 - r.row0) + j);
    };
    auto body = [&](const RawChunk<T, kPacked>& r, int64_t c) {
        float v[8];
        int col[8];
        if constexpr (sizeof(T) == 4)
            unpack_vals(r.v, v);
        else
            unpack_vals<T>(r.v, v);
        unpack_cols<T, kPacked>(r, a.cols, c, lane, col);
        if (!__any_sync(kFull, r.h != 0u)) {  // no row starts: all of it is the open row
#pragma unroll
            for (int i = 0; i < 8; i++) oacc = fmaf(v[i], xv(col[i]), oacc);
            open_valid = true;
            return;
        }
        int hcnt = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const float p = v[i] * xv(col[i]);
            const uint32_t m = __ballot_sync(kFull, (r.h >> i) & 1u);
            if (m == 0) {
                oacc += p;
                open_valid = true;
                continue;
            }
            // close the open row: its lanes' shares plus the lanes before the first start
            const int fh = __ffs(m) - 1;
            const float closing = warp_sum(oacc + (lane < fh ? p : 0.0f));
            if ((open_valid || fh > 0) && lane == 0) put(y, a.row_scale, open_row, closing);
            if ((m & (m - 1u)) == 0u) {  // one row start: no row begins and ends in the slice
                oacc = lane >= fh ? p : 0.0f;
                hcnt += 1;
                open_row = row_at(r, hcnt - 1);
                open_valid = true;
                continue;
            }
            // rows inside the slice: segmented inclusive scan from the first start
            float s = lane >= fh ? p : 0.0f;
            int f = (m >> lane) & 1u;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const float ts = __shfl_up_sync(kFull, s, o);
                const int tf = __shfl_up_sync(kFull, f, o);
                if (lane >= o) {
                    if (!f) s += ts;
                    f |= tf;
                }
            }
            if (lane < 31 && lane >= fh && ((m >> (lane + 1)) & 1u))
                put(y, a.row_scale, row_at(r, hcnt + __popc(m & ((2u << lane) - 1u)) - 1), s);
            // the slice's last row stays open
            const int lh = 31 - __clz(m);
            oacc = lane >= lh ? p : 0.0f;
            hcnt += __popc(m);
            open_row = row_at(r, hcnt - 1);
            open_valid = true;
        }
    };
    if constexpr (sizeof(T) == 2 && kSmemX) {
        // 16-bit values, x in shared memory: the next chunk's loads are issued
        // before this chunk is summed, so a warp keeps a chunk in flight while
        // it computes
        RawChunk<T, kPacked> r;
        if (c0 < c1) load_raw(a, c0, lane, r);
        for (int64_t c = c0; c < c1; c++) {
            RawChunk<T, kPacked> rn;
            const bool more = c + 1 < c1;  // uniform per warp
            if (more) load_raw(a, c + 1, lane, rn);
            body(r, c);
            if (more) r = rn;
        }
    } else if constexpr (sizeof(T) == 2) {
        // 16-bit values, x gathered from global memory: two chunks' loads are
        // issued together (fewer registers held than the rolling form)
        for (int64_t c = c0; c < c1; c += 2) {
            RawChunk<T, kPacked> r0, r1;
            load_raw(a, c, lane, r0);
            const bool two = c + 1 < c1;  // uniform per warp
            if (two) load_raw(a, c + 1, lane, r1);
            body(r0, c);
            if (two) body(r1, c + 1);
        }
    } else {
        for (int64_t c = c0; c < c1; c++) {
            RawChunk<T, kPacked> r;
            load_raw(a, c, lane, r);
            body(r, c);
        }
    }
    const float part = warp_sum(oacc);
    if (lane == 0) {
        a.carry_row[w] = open_valid ? (int64_t)open_row : a.rows;
        a.carry_val[w] = part;
    }
}

// Adds the carries of rows that cross warp ranges: the first warp of each run
// of equal carry rows sums the run in warp order.
__global__ void spmv_fixup_kernel(int n_warps, const int64_t* __restrict__ carry_row,
                                  const float* __restrict__ carry_val, const float* __restrict__ row_scale,
                                  int64_t rows, float* __restrict__ y) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_warps) return;
    const int64_t r = carry_row[t];
    if (r >= rows || (t > 0 && carry_row[t - 1] == r)) return;
    float s = 0.0f;
    for (int u = t; u < n_warps && carry_row[u] == r; u++) s += carry_val[u];
    y[r] += row_scale ? row_scale[r] * s : s;
}

__global__ void scale_vector_kernel(const float* __restrict__ s, const float* __restrict__ x, float* __restrict__ out,
                                    int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = s[i] * x[i];
}

// ---------------------------------------------------------------- plan
unsigned grid_for(int64_t n, int threads = 256) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 16));
}

// the row-start bit of off[r] for every row with nonzeros (rows own distinct
// bits; atomicOr makes the word updates safe).  Layout: a chunk has 32 bytes,
// one per lane; bit i of byte l flags logical element 32 i + l.
__global__ void mark_row_starts(const int64_t* __restrict__ off, int64_t rows, uint32_t* __restrict__ head,
                                int32_t* __restrict__ nonempty) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
        const bool ne = off[r + 1] > off[r];
        nonempty[r] = ne;
        if (ne) {  // element e of chunk c: lane e % 32's byte, bit e / 32
            const int64_t c = off[r] / kChunk;
            const int e = (int)(off[r] % kChunk), l = e & 31;
            atomicOr(head + c * kChunkWords + (l >> 2), 1u << ((l & 3) * 8 + (e >> 5)));
        }
    }
}

// Per chunk: the row of its first row start when all its row starts belong to
// consecutive rows (no empty row between them), so the j-th is row0 + j;
// otherwise -1 - (row starts before the chunk), and the rows come from nzrow.
__global__ void chunk_first_rows(const int32_t* __restrict__ cnt, const int32_t* __restrict__ chunk_h,
                                 const int32_t* __restrict__ nzrow, int64_t n_chunks, int32_t* __restrict__ row0) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n_chunks;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int n = cnt[c], hb = chunk_h[c];
        if (n == 0) {
            row0[c] = 0;  // no row starts: never read
            continue;
        }
        const int r0 = nzrow[hb];
        row0[c] = nzrow[hb + n - 1] - r0 == n - 1 ? r0 : -1 - hb;
    }
}

__global__ void scatter_rows(const int32_t* __restrict__ nonempty, const int32_t* __restrict__ pos, int64_t rows,
                             int32_t* __restrict__ nzrow) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x)
        if (nonempty[r]) nzrow[pos[r]] = (int32_t)r;
}

__global__ void chunk_head_counts(const uint32_t* __restrict__ head, int64_t n_chunks, int32_t* __restrict__ cnt) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n_chunks;
         c += (int64_t)gridDim.x * blockDim.x) {
        int s = 0;
#pragma unroll
        for (int i = 0; i < kChunkWords; i++) s += __popc(head[c * kChunkWords + i]);
        cnt[c] = s;
    }
}

// PACKED16, pass 1: one warp per chunk; is the chunk's column span < 65536?
__global__ void chunk_span(const int32_t* __restrict__ col, int64_t nnz, int64_t n_chunks, int32_t* __restrict__ base,
                           int32_t* __restrict__ wide) {
    const int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c >= n_chunks) return;
    int lo = 0x7fffffff, hi = -1;
    for (int i = lane; i < kChunk; i += 32) {
        const int64_t k = c * kChunk + i;
        if (k < nnz) {
            lo = min(lo, col[k]);
            hi = max(hi, col[k]);
        }
    }
    for (int o = 16; o; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(kFull, lo, o));
        hi = max(hi, __shfl_xor_sync(kFull, hi, o));
    }
    if (lane == 0) {
        if (hi < 0) lo = hi = 0;  // chunk of padding only
        base[c] = lo;
        wide[c] = hi - lo > 0xffff;
    }
}

// PACKED16, pass 2: offsets for narrow chunks, int32 copies for wide ones,
// from logical-order columns into storage order
__global__ void pack_columns(const int32_t* __restrict__ col, int64_t nnz, int64_t n_chunks,
                             const int32_t* __restrict__ wide, const int32_t* __restrict__ exc_slot,
                             int32_t* __restrict__ base, uint16_t* __restrict__ col16, int32_t* __restrict__ exc) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n_chunks * kChunk;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = k / kChunk, q = slot(k);
        const int cv = k < nnz ? col[k] : 0;
        if (wide[c]) {
            exc[(int64_t)exc_slot[c] * kChunk + q % kChunk] = cv;
            col16[q] = 0;
        } else {
            col16[q] = (uint16_t)(k < nnz ? cv - base[c] : 0);
        }
    }
}

// logical order -> storage order
template <typename E>
__global__ void to_storage_order(const E* __restrict__ src, E* __restrict__ dst, int64_t n) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        dst[slot(k)] = src[k];
}

__global__ void mark_wide_bases(const int32_t* __restrict__ wide, const int32_t* __restrict__ slot, int64_t n_chunks,
                                int32_t* __restrict__ base) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n_chunks;
         c += (int64_t)gridDim.x * blockDim.x)
        if (wide[c]) base[c] = -1 - slot[c];
}

template <typename T>
int exclusive_scan(const T* in, T* out, int64_t n, cudaStream_t st) {
    if (n <= 0) return FD2_OK;
    size_t tb = 0;
    FD2_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, n, st));
    void* tmp = nullptr;
    FD2_CHECK_CUDA(cudaMalloc(&tmp, std::max<size_t>(tb, 16)));
    cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, tb, in, out, n, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(tmp);
    FD2_CHECK_CUDA(e);
    return FD2_OK;
}

// ---------------------------------------------------------------- set-up kernels
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
__device__ __forceinline__ float to_float(float v) { return v; }
__device__ __forceinline__ float to_float(__half v) { return __half2float(v); }
__device__ __forceinline__ float to_float(__nv_bfloat16 v) { return __bfloat162float(v); }

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

// columns (decoded) and values as FP32 with the scale applied
template <typename T>
__global__ void unpack_entries(const int64_t* __restrict__ off, int64_t rows, ColView cv, const T* __restrict__ val,
                               const float* __restrict__ s, int axis, int64_t nnz, int32_t* __restrict__ col_out,
                               float* __restrict__ val_out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
        const int c = cv.at(k);
        float v = to_float(val[slot(k)]);
        if (axis == FD2_SCALE_COLS)
            v *= s[c];
        else if (axis == FD2_SCALE_ROWS)
            v *= s[row_of(off, rows, k)];
        if (col_out) col_out[k] = c;
        if (val_out) val_out[k] = v;
    }
}

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
        val_out[k] = val[slot(src)];
    }
}

// The x-in-shared-memory instance of the stream kernel, allowed the largest x.
template <typename T, bool kPacked>
cudaError_t allow_smem_x() {
    return cudaFuncSetAttribute(spmv_stream_kernel<T, kPacked, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kSmemXMaxBytes);
}

template <typename T, bool kPacked>
int launch_stream_fmt(const fd2_matrix* m, const StreamArgs& a, const float* x, float* y, cudaStream_t st) {
    if (m->x_in_smem) {  // the shared-memory limit was raised when the matrix was finalized
        const unsigned blocks = (unsigned)(((int64_t)m->n_warps * 32 + kSmemThreads - 1) / kSmemThreads);
        spmv_stream_kernel<T, kPacked, true><<<blocks, kSmemThreads, (size_t)m->cols * sizeof(float), st>>>(a, x, y);
    } else {
        const unsigned blocks = (unsigned)(((int64_t)m->n_warps * 32 + kStreamThreads - 1) / kStreamThreads);
        spmv_stream_kernel<T, kPacked, false><<<blocks, kStreamThreads, 0, st>>>(a, x, y);
    }
    FD2_CHECK_CUDA(cudaGetLastError());
    return FD2_OK;
}

template <typename T>
int launch_stream(const fd2_matrix* m, const float* x, float* y, cudaStream_t st) {
    StreamArgs a{m->d_val, m->cols_view(), m->d_head, m->d_chunk_h, m->d_chunk_row0, m->d_nzrow,
                 m->scale_axis == FD2_SCALE_ROWS ? m->d_scale : nullptr, m->n_chunks, m->n_warps, m->rows,
                 m->d_carry_row, m->d_carry_val, (int)m->cols};
    if (m->index_format == FD2_INDEX_PACKED16)
        FD2_TRY((launch_stream_fmt<T, true>(m, a, x, y, st)));
    else
        FD2_TRY((launch_stream_fmt<T, false>(m, a, x, y, st)));
    spmv_fixup_kernel<<<(m->n_warps + 255) / 256, 256, 0, st>>>(m->n_warps, m->d_carry_row, m->d_carry_val,
                                                               a.row_scale, m->rows, y);
    FD2_CHECK_CUDA(cudaGetLastError());
    return FD2_OK;
}

template <typename T>
int transpose_typed(const fd2_matrix* m, fd2_matrix* t, cudaStream_t st) {
    const int64_t nnz = m->nnz;
    int32_t *keys_in = nullptr, *keys_out = nullptr;
    int64_t *perm_in = nullptr, *perm_out = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    int end_bit = 1;
    while (end_bit < 31 && ((int64_t)1 << end_bit) < m->cols) end_bit++;
    int rc = FD2_OK;
    cudaError_t e = cudaMalloc(&keys_in, nnz * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&keys_out, nnz * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&perm_in, nnz * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMalloc(&perm_out, nnz * sizeof(int64_t));
    if (e == cudaSuccess) {
        unpack_entries<T><<<grid_for(nnz), 256, 0, st>>>(m->d_off, m->rows, m->cols_view(), (const T*)m->d_val,
                                                         nullptr, FD2_SCALE_NONE, nnz, keys_in, nullptr);
        e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys_in, keys_out, perm_in, perm_out, nnz, 0, end_bit,
                                            st);
    }
    if (e == cudaSuccess) e = cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 16));
    if (e == cudaSuccess) {
        // stable sort by column: within a new row, entries keep ascending old-row order
        iota64<<<grid_for(nnz), 256, 0, st>>>(perm_in, nnz);
        e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys_in, keys_out, perm_in, perm_out, nnz, 0, end_bit,
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
    for (void* p : {(void*)keys_in, (void*)keys_out, (void*)perm_in, (void*)perm_out, tmp})
        if (p) cudaFree(p);
    return rc;
}

}  // namespace

int matrix_alloc(fd2_matrix* m, cudaStream_t st) {
    FD2_CHECK_CUDA(cudaMalloc(&m->d_off, (m->rows + 1) * sizeof(int64_t)));
    return matrix_alloc_entries(m, st);
}

int matrix_alloc_entries(fd2_matrix* m, cudaStream_t st) {
    const int64_t pad = round_chunk(m->nnz);
    FD2_CHECK_CUDA(cudaMalloc(&m->d_col, std::max<int64_t>(pad, 1) * sizeof(int32_t)));
    FD2_CHECK_CUDA(cudaMalloc(&m->d_val, std::max<int64_t>(pad, 1) * value_size(m->value_type)));
    if (pad > m->nnz) {  // the last chunk's padding: column 0, value 0
        FD2_CHECK_CUDA(cudaMemsetAsync(m->d_col + m->nnz, 0, (pad - m->nnz) * sizeof(int32_t), st));
        FD2_CHECK_CUDA(cudaMemsetAsync((char*)m->d_val + m->nnz * value_size(m->value_type), 0,
                                       (pad - m->nnz) * value_size(m->value_type), st));
    }
    if (m->scale_axis != FD2_SCALE_NONE) {
        const int64_t n = m->scale_axis == FD2_SCALE_ROWS ? m->rows : m->cols;
        FD2_CHECK_CUDA(cudaMalloc(&m->d_scale, std::max<int64_t>(n, 1) * sizeof(float)));
    }
    return FD2_OK;
}

void matrix_free(fd2_matrix* m) {
    for (void* p : {(void*)m->d_off, (void*)m->d_col, (void*)m->d_col16, (void*)m->d_cbase, (void*)m->d_exc, m->d_val,
                    (void*)m->d_scale, (void*)m->d_head, (void*)m->d_chunk_h, (void*)m->d_chunk_row0, (void*)m->d_nzrow,
                    (void*)m->d_carry_row, (void*)m->d_carry_val, (void*)m->d_xs})
        if (p) cudaFree(p);
    m->d_off = nullptr;
    m->d_col = nullptr;
    m->d_col16 = nullptr;
    m->d_cbase = m->d_exc = nullptr;
    m->d_val = nullptr;
    m->d_scale = nullptr;
    m->d_head = nullptr;
    m->d_chunk_h = m->d_chunk_row0 = m->d_nzrow = nullptr;
    m->d_carry_row = nullptr;
    m->d_carry_val = m->d_xs = nullptr;
}

// Warps of one full wave of the stream kernel for this matrix's instance: every
// warp owns one contiguous range, so there is no second, partial wave.  A
// matrix whose x fits in shared memory (cols x 4 bytes <= kSmemXMaxBytes) uses
// the x-in-shared-memory instance, one block of kSmemThreads per SM.
template <typename T, bool kPacked>
int resident_warps(fd2_matrix* m, int sm_count) {
    int per_sm = 0;
    const int64_t xb = m->cols * (int64_t)sizeof(float);
    m->x_in_smem = false;
    if (xb > 0 && xb <= kSmemXMaxBytes && allow_smem_x<T, kPacked>() == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spmv_stream_kernel<T, kPacked, true>, kSmemThreads,
                                                      (size_t)xb) == cudaSuccess &&
        per_sm >= 1) {
        m->x_in_smem = true;
        return per_sm * sm_count * (kSmemThreads / 32);
    }
    cudaGetLastError();  // a refused attribute or query leaves the global-gather instance
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spmv_stream_kernel<T, kPacked, false>, kStreamThreads,
                                                      0) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    return per_sm * sm_count * (kStreamThreads / 32);
}

int stream_warps(fd2_matrix* m) {
    const int sms = m->ctx->sm_count > 0 ? m->ctx->sm_count : 148;
    const bool pk = m->index_format == FD2_INDEX_PACKED16;
    int w;
    switch (m->value_type) {
        case FD2_VALUES_F16:
            w = pk ? resident_warps<__half, true>(m, sms) : resident_warps<__half, false>(m, sms);
            break;
        case FD2_VALUES_BF16:
            w = pk ? resident_warps<__nv_bfloat16, true>(m, sms) : resident_warps<__nv_bfloat16, false>(m, sms);
            break;
        default: w = pk ? resident_warps<float, true>(m, sms) : resident_warps<float, false>(m, sms);
    }
    return std::min(w, kMaxStreamWarps);
}

int matrix_finalize(fd2_matrix* m, cudaStream_t st) {
    m->n_chunks = round_chunk(m->nnz) / kChunk;
    m->n_warps = (int)std::max<int64_t>(1, std::min<int64_t>(m->n_chunks, stream_warps(m)));
    FD2_CHECK_CUDA(cudaMalloc(&m->d_head, std::max<int64_t>(m->n_chunks * kChunkWords, 1) * sizeof(uint32_t)));
    FD2_CHECK_CUDA(cudaMalloc(&m->d_chunk_h, std::max<int64_t>(m->n_chunks, 1) * sizeof(int32_t)));
    FD2_CHECK_CUDA(cudaMalloc(&m->d_chunk_row0, std::max<int64_t>(m->n_chunks, 1) * sizeof(int32_t)));
    FD2_CHECK_CUDA(cudaMalloc(&m->d_carry_row, m->n_warps * sizeof(int64_t)));
    FD2_CHECK_CUDA(cudaMalloc(&m->d_carry_val, m->n_warps * sizeof(float)));
    if (m->scale_axis == FD2_SCALE_COLS)
        FD2_CHECK_CUDA(cudaMalloc(&m->d_xs, std::max<int64_t>(m->cols, 1) * sizeof(float)));
    FD2_CHECK_CUDA(cudaMemsetAsync(m->d_head, 0, std::max<int64_t>(m->n_chunks * kChunkWords, 1) * sizeof(uint32_t),
                                   st));
    // row starts, non-empty rows, row starts before each chunk
    int32_t *ne = nullptr, *pos = nullptr, *cnt = nullptr;
    auto cleanup = [&]() {
        for (void* p : {(void*)ne, (void*)pos, (void*)cnt})
            if (p) cudaFree(p);
    };
    const int64_t rows1 = std::max<int64_t>(m->rows, 1);
    if (cudaMalloc(&ne, rows1 * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&pos, rows1 * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&cnt, std::max<int64_t>(m->n_chunks, 1) * sizeof(int32_t)) != cudaSuccess) {
        cleanup();
        set_error("matrix_finalize: out of device memory");
        return FD2_ERR_OUT_OF_MEMORY;
    }
    int rc = FD2_OK;
    if (m->rows) mark_row_starts<<<grid_for(m->rows), 256, 0, st>>>(m->d_off, m->rows, m->d_head, ne);
    if (m->rows) rc = exclusive_scan(ne, pos, m->rows, st);
    int32_t last_ne = 0, last_pos = 0;
    if (!rc && m->rows) {
        if (cudaMemcpy(&last_ne, ne + m->rows - 1, 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(&last_pos, pos + m->rows - 1, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = FD2_ERR_CUDA;
    }
    m->n_nzrows = (int64_t)last_pos + last_ne;
    if (!rc && cudaMalloc(&m->d_nzrow, std::max<int64_t>(m->n_nzrows, 1) * sizeof(int32_t)) != cudaSuccess)
        rc = FD2_ERR_OUT_OF_MEMORY;
    if (!rc && m->rows) scatter_rows<<<grid_for(m->rows), 256, 0, st>>>(ne, pos, m->rows, m->d_nzrow);
    if (!rc && m->n_chunks) {
        chunk_head_counts<<<grid_for(m->n_chunks), 256, 0, st>>>(m->d_head, m->n_chunks, cnt);
        rc = exclusive_scan(cnt, m->d_chunk_h, m->n_chunks, st);
        if (!rc)
            chunk_first_rows<<<grid_for(m->n_chunks), 256, 0, st>>>(cnt, m->d_chunk_h, m->d_nzrow, m->n_chunks,
                                                                   m->d_chunk_row0);
    }
    // 16-bit column packing
    if (!rc && m->index_format == FD2_INDEX_PACKED16 && m->n_chunks) {
        int32_t *wide = ne, *eslot = pos;  // reuse when large enough
        bool own = m->n_chunks > rows1;
        if (own && (cudaMalloc(&wide, m->n_chunks * sizeof(int32_t)) != cudaSuccess ||
                    cudaMalloc(&eslot, m->n_chunks * sizeof(int32_t)) != cudaSuccess))
            rc = FD2_ERR_OUT_OF_MEMORY;
        if (!rc && cudaMalloc(&m->d_cbase, m->n_chunks * sizeof(int32_t)) != cudaSuccess) rc = FD2_ERR_OUT_OF_MEMORY;
        if (!rc) {
            chunk_span<<<(unsigned)((m->n_chunks * 32 + 255) / 256), 256, 0, st>>>(m->d_col, m->nnz, m->n_chunks,
                                                                                 m->d_cbase, wide);
            rc = exclusive_scan(wide, eslot, m->n_chunks, st);
        }
        int32_t lw = 0, ls = 0;
        if (!rc && (cudaMemcpy(&lw, wide + m->n_chunks - 1, 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
                    cudaMemcpy(&ls, eslot + m->n_chunks - 1, 4, cudaMemcpyDeviceToHost) != cudaSuccess))
            rc = FD2_ERR_CUDA;
        m->n_exc = (int64_t)lw + ls;
        if (!rc && (cudaMalloc(&m->d_col16, m->n_chunks * kChunk * sizeof(uint16_t)) != cudaSuccess ||
                    cudaMalloc(&m->d_exc, std::max<int64_t>(m->n_exc, 1) * kChunk * sizeof(int32_t)) != cudaSuccess))
            rc = FD2_ERR_OUT_OF_MEMORY;
        if (!rc) {
            pack_columns<<<grid_for(m->n_chunks * kChunk), 256, 0, st>>>(m->d_col, m->nnz, m->n_chunks, wide, eslot,
                                                                        m->d_cbase, m->d_col16, m->d_exc);
            mark_wide_bases<<<grid_for(m->n_chunks), 256, 0, st>>>(wide, eslot, m->n_chunks, m->d_cbase);
            if (cudaStreamSynchronize(st) != cudaSuccess) rc = FD2_ERR_CUDA;
        }
        if (own) {
            if (wide) cudaFree(wide);
            if (eslot) cudaFree(eslot);
        }
        if (!rc) {  // the int32 columns are no longer needed
            cudaFree(m->d_col);
            m->d_col = nullptr;
        }
    } else if (!rc && m->index_format == FD2_INDEX_PACKED16) {
        cudaFree(m->d_col);  // empty matrix: nothing to pack
        m->d_col = nullptr;
        if (cudaMalloc(&m->d_cbase, sizeof(int32_t)) != cudaSuccess ||
            cudaMalloc(&m->d_col16, kChunk * sizeof(uint16_t)) != cudaSuccess ||
            cudaMalloc(&m->d_exc, kChunk * sizeof(int32_t)) != cudaSuccess)
            rc = FD2_ERR_OUT_OF_MEMORY;
    }
    // values (and int32 columns) to storage order
    if (!rc && m->n_chunks) {
        const int64_t pad = m->n_chunks * kChunk;
        const size_t vs = value_size(m->value_type);
        void* tmp = nullptr;
        if (cudaMalloc(&tmp, pad * vs) != cudaSuccess) {
            rc = FD2_ERR_OUT_OF_MEMORY;
        } else {
            if (vs == 4)
                to_storage_order<uint32_t><<<grid_for(pad), 256, 0, st>>>((const uint32_t*)m->d_val, (uint32_t*)tmp, pad);
            else
                to_storage_order<uint16_t><<<grid_for(pad), 256, 0, st>>>((const uint16_t*)m->d_val, (uint16_t*)tmp, pad);
            if (cudaStreamSynchronize(st) != cudaSuccess) rc = FD2_ERR_CUDA;
            cudaFree(m->d_val);
            m->d_val = tmp;
        }
        if (!rc && m->d_col) {
            int32_t* tc = nullptr;
            if (cudaMalloc(&tc, pad * sizeof(int32_t)) != cudaSuccess) {
                rc = FD2_ERR_OUT_OF_MEMORY;
            } else {
                to_storage_order<int32_t><<<grid_for(pad), 256, 0, st>>>(m->d_col, tc, pad);
                if (cudaStreamSynchronize(st) != cudaSuccess) rc = FD2_ERR_CUDA;
                cudaFree(m->d_col);
                m->d_col = tc;
            }
        }
    }
    if (!rc && cudaStreamSynchronize(st) != cudaSuccess) rc = FD2_ERR_CUDA;
    cleanup();
    if (rc && rc != FD2_ERR_OUT_OF_MEMORY) set_error("matrix_finalize: %s", cudaGetErrorString(cudaGetLastError()));
    return rc;
}

int matrix_spmv(const fd2_matrix* m, const float* x, float* y, cudaStream_t st) {
    if (m->rows == 0) return FD2_OK;
    FD2_CHECK_CUDA(cudaMemsetAsync(y, 0, m->rows * sizeof(float), st));  // empty rows, and rows only carries reach
    if (m->n_chunks == 0) return FD2_OK;
    if (m->scale_axis == FD2_SCALE_COLS) {
        scale_vector_kernel<<<grid_for(m->cols), 256, 0, st>>>(m->d_scale, x, m->d_xs, m->cols);
        FD2_CHECK_CUDA(cudaGetLastError());
        x = m->d_xs;
        m->ctx->launches += 1;
    }
    m->ctx->launches += 2;
    switch (m->value_type) {
        case FD2_VALUES_F16: return launch_stream<__half>(m, x, y, st);
        case FD2_VALUES_BF16: return launch_stream<__nv_bfloat16>(m, x, y, st);
        default: return launch_stream<float>(m, x, y, st);
    }
}

}  // namespace fd2

using namespace fd2;

extern "C" {

int fd2_matrix_create(fd2_context* ctx, int64_t rows, int64_t cols, int64_t nnz, const int64_t* h_off,
                      const int64_t* h_col, const float* h_val, int value_type, int index_format,
                      fd2_matrix** out) {
    FD2_REQUIRE(ctx && h_off && out && (nnz == 0 || (h_col && h_val)), FD2_ERR_INVALID_ARGUMENT,
                "matrix_create: null argument");
    FD2_REQUIRE(rows >= 0 && rows < ((int64_t)1 << 31) && cols >= 0 && cols < ((int64_t)1 << 31) && nnz >= 0,
                FD2_ERR_INVALID_ARGUMENT, "matrix_create: sizes rows=%lld cols=%lld nnz=%lld", (long long)rows,
                (long long)cols, (long long)nnz);
    FD2_REQUIRE(value_type >= FD2_VALUES_F32 && value_type <= FD2_VALUES_BF16, FD2_ERR_INVALID_ARGUMENT,
                "matrix_create: value type %d", value_type);
    FD2_REQUIRE(index_format == FD2_INDEX_I32 || index_format == FD2_INDEX_PACKED16, FD2_ERR_INVALID_ARGUMENT,
                "matrix_create: index format %d", index_format);
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
    m->index_format = index_format;
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
    int rc = matrix_alloc(m, st);
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
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // host staging buffers must outlive the copies
    if (e != cudaSuccess) {
        set_error("matrix_create: %s", cudaGetErrorString(e));
        return fail(e == cudaErrorMemoryAllocation ? FD2_ERR_OUT_OF_MEMORY : FD2_ERR_CUDA);
    }
    rc = matrix_finalize(m, st);
    if (rc) return fail(rc);
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
    info->index_format = m->index_format;
    info->x_in_shared = m->x_in_smem ? 1 : 0;
    info->exception_chunks = m->n_exc;
    const int64_t pad = m->n_chunks * kChunk;
    const int64_t ns = m->scale_axis == FD2_SCALE_ROWS ? m->rows : m->scale_axis == FD2_SCALE_COLS ? m->cols : 0;
    const int64_t col_bytes =
        m->index_format == FD2_INDEX_PACKED16 ? pad * 2 + m->n_chunks * 4 + m->n_exc * kChunk * 4 : pad * 4;
    info->device_bytes = pad * (int64_t)value_size(m->value_type) + col_bytes + pad / 8 + m->n_chunks * 8 +
                         m->n_nzrows * 4 + ns * (int64_t)sizeof(float);
    return FD2_OK;
}

int fd2_matrix_to_host(const fd2_matrix* m, int64_t* h_off, int32_t* h_col, float* h_val) {
    FD2_REQUIRE(m && h_off && (m->nnz == 0 || (h_col && h_val)), FD2_ERR_INVALID_ARGUMENT,
                "matrix_to_host: null argument");
    cudaStream_t st = m->ctx->stream;
    FD2_CHECK_CUDA(cudaMemcpyAsync(h_off, m->d_off, (m->rows + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    if (m->nnz) {
        float* d_f = nullptr;
        int32_t* d_c = nullptr;
        cudaError_t e = cudaMalloc(&d_f, m->nnz * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&d_c, m->nnz * sizeof(int32_t));
        if (e == cudaSuccess) {
            switch (m->value_type) {
                case FD2_VALUES_F16:
                    unpack_entries<__half><<<grid_for(m->nnz), 256, 0, st>>>(
                        m->d_off, m->rows, m->cols_view(), (const __half*)m->d_val, m->d_scale, m->scale_axis, m->nnz,
                        d_c, d_f);
                    break;
                case FD2_VALUES_BF16:
                    unpack_entries<__nv_bfloat16><<<grid_for(m->nnz), 256, 0, st>>>(
                        m->d_off, m->rows, m->cols_view(), (const __nv_bfloat16*)m->d_val, m->d_scale, m->scale_axis,
                        m->nnz, d_c, d_f);
                    break;
                default:
                    unpack_entries<float><<<grid_for(m->nnz), 256, 0, st>>>(m->d_off, m->rows, m->cols_view(),
                                                                            (const float*)m->d_val, m->d_scale,
                                                                            m->scale_axis, m->nnz, d_c, d_f);
            }
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_val, d_f, m->nnz * sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_col, d_c, m->nnz * sizeof(int32_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (d_f) cudaFree(d_f);
        if (d_c) cudaFree(d_c);
        FD2_CHECK_CUDA(e);
    }
    FD2_CHECK_CUDA(cudaStreamSynchronize(st));
    return FD2_OK;
}

int fd2_matrix_transpose(const fd2_matrix* m, fd2_matrix** out) {
    FD2_REQUIRE(m && out, FD2_ERR_INVALID_ARGUMENT, "matrix_transpose: null argument");
    return matrix_transpose_fmt(m, m->index_format, out);
}

}  // extern "C"

int fd2::matrix_transpose_fmt(const fd2_matrix* m, int index_format, fd2_matrix** out) {
    auto* t = new fd2_matrix();
    t->ctx = m->ctx;
    t->rows = m->cols;
    t->cols = m->rows;
    t->nnz = m->nnz;
    t->value_type = m->value_type;
    t->index_format = index_format;
    t->scale_axis = m->scale_axis == FD2_SCALE_ROWS   ? FD2_SCALE_COLS
                    : m->scale_axis == FD2_SCALE_COLS ? FD2_SCALE_ROWS
                                                      : FD2_SCALE_NONE;
    cudaStream_t st = m->ctx->stream;
    int rc = matrix_alloc(t, st);
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
    if (rc == FD2_OK) rc = matrix_finalize(t, st);
    if (rc) {
        matrix_free(t);
        delete t;
        return rc;
    }
    *out = t;
    return FD2_OK;
}

extern "C" int fd2_matrix_spmv(const fd2_matrix* m, const float* d_x, float* d_y, void* stream) {
    FD2_REQUIRE(m && d_y && (m->cols == 0 || d_x), FD2_ERR_INVALID_ARGUMENT, "matrix_spmv: null argument");
    return matrix_spmv(m, d_x, d_y, (cudaStream_t)stream);
}
