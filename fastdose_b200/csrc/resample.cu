// resample.cu -- BEV -> PVCS resampling: dense trilinear volumes and the
// per-beamlet sparse dose columns of the dose-loading matrix.
//
// Dense: d_BEV2PVCS (FastDoseLib/src/TermaComp.cu:124-150) and
// d_BEV2PVCS_SuperSampling (FastDoseLib/src/geom.cu:412-474).  Each voxel centre
// (or ss^3 sub-voxel sample) is rotated into the beam frame, projected onto the
// divergent BEV grid and sampled trilinearly (texel centres at i+0.5, zero
// outside), as the reference's linear/border texture does.
//
// Sparse columns: d_voxelInterp (IMRTOpt/src/IMRTgeom.cu:370-468).  A voxel within
// extent + half its diagonal of the beamlet axis takes the mean of ss^3 point
// samples of the beamlet's BEV dose; samples outside the fluence map laterally
// are skipped, samples outside [0, long_dim) in depth read zero.  The reference
// evaluates every (voxel, beamlet) pair of a beam into a dense
// [beamlets x voxels] matrix and then converts it with cusparseDenseToSparse;
// here each beamlet visits only the voxels of a conservative box around its
// frustum, tests them against a cheap bound, and emits its nonzeros straight
// into CSR order (voxel index ascending) with a block-wide scan.
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

#include "fd2_internal.cuh"
#include "resample.cuh"

namespace fd2 {

namespace {

__device__ __forceinline__ float3 rot(const float* R, float3 v) {
    return make_float3(R[0] * v.x + R[1] * v.y + R[2] * v.z, R[3] * v.x + R[4] * v.y + R[5] * v.z,
                       R[6] * v.x + R[7] * v.y + R[8] * v.z);
}

__device__ __forceinline__ float bev_fetch(const float* __restrict__ bev, int fx, int fy, int L, int i, int j, int k) {
    if ((unsigned)i >= (unsigned)fx || (unsigned)j >= (unsigned)fy || (unsigned)k >= (unsigned)L) return 0.0f;
    return __ldg(bev + (size_t)i + (size_t)fx * ((size_t)j + (size_t)fy * k));
}

__device__ __forceinline__ float bev_trilinear(const float* __restrict__ bev, int fx, int fy, int L, float u, float v,
                                               float w) {
    float xb = u - 0.5f, yb = v - 0.5f, zb = w - 0.5f;
    float fi = floorf(xb), fj = floorf(yb), fk = floorf(zb);
    float ax = xb - fi, ay = yb - fj, az = zb - fk;
    int i = (int)fi, j = (int)fj, k = (int)fk;
    float c00 = bev_fetch(bev, fx, fy, L, i, j, k) * (1 - ax) + bev_fetch(bev, fx, fy, L, i + 1, j, k) * ax;
    float c10 = bev_fetch(bev, fx, fy, L, i, j + 1, k) * (1 - ax) + bev_fetch(bev, fx, fy, L, i + 1, j + 1, k) * ax;
    float c01 = bev_fetch(bev, fx, fy, L, i, j, k + 1) * (1 - ax) + bev_fetch(bev, fx, fy, L, i + 1, j, k + 1) * ax;
    float c11 =
        bev_fetch(bev, fx, fy, L, i, j + 1, k + 1) * (1 - ax) + bev_fetch(bev, fx, fy, L, i + 1, j + 1, k + 1) * ax;
    return (c00 * (1 - ay) + c10 * ay) * (1 - az) + (c01 * (1 - ay) + c11 * ay) * az;
}

// PVCS point -> normalised BEV coordinates (x lateral, y depth, z lateral).
__device__ __forceinline__ float3 to_bev_grid(const ColumnInfo& ci, float3 p) {
    float3 v = rot(ci.R, make_float3(p.x - ci.src[0], p.y - ci.src[1], p.z - ci.src[2]));
    float k = v.y * ci.inv_sad;
    return make_float3(v.x / (ci.bsx * k) + ci.hx, (v.y - ci.lim_min) * ci.inv_ls, v.z / (ci.bsy * k) + ci.hy);
}

__global__ void bev2pvcs_kernel(ColumnInfo ci, const float* __restrict__ bev, float* __restrict__ out, size_t pitch,
                                int nx, int ny, int nz, float vx, float vy, float vz) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y,
        z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= nx || y >= ny || z >= nz) return;
    float3 cn = to_bev_grid(ci, make_float3((x + 0.5f) * vx, (y + 0.5f) * vy, (z + 0.5f) * vz));
    out[(size_t)x + pitch * ((size_t)y + (size_t)ny * z)] = bev_trilinear(bev, ci.fx, ci.fy, ci.L, cn.x, cn.z, cn.y);
}

__global__ void bev2pvcs_ss_kernel(ColumnInfo ci, const float* __restrict__ bev, float* __restrict__ out, size_t pitch,
                                   int nx, int ny, int nz, float vx, float vy, float vz, int ss, float extent) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y,
        z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= nx || y >= ny || z >= nz) return;
    float3 c = make_float3((x + 0.5f) * vx, (y + 0.5f) * vy, (z + 0.5f) * vz);
    float3 v = rot(ci.R, make_float3(c.x - ci.src[0], c.y - ci.src[1], c.z - ci.src[2]));
    if (v.x * v.x + v.z * v.z > extent * extent) return;
    float inv = 1.0f / ss, acc = 0.0f;
    for (int k = 0; k < ss; k++)
        for (int j = 0; j < ss; j++)
            for (int i = 0; i < ss; i++) {
                float3 cn = to_bev_grid(ci, make_float3((x + (i + 0.5f) * inv) * vx, (y + (j + 0.5f) * inv) * vy,
                                                        (z + (k + 0.5f) * inv) * vz));
                acc += bev_trilinear(bev, ci.fx, ci.fy, ci.L, cn.x, cn.z, cn.y);
            }
    if (acc < 1e-4f) return;
    out[(size_t)x + pitch * ((size_t)y + (size_t)ny * z)] = acc / (float)(ss * ss * ss);
}

// Conservative candidate test for a voxel centre c: could any point within
// hdiag of c carry a nonzero column value?
__device__ __forceinline__ bool candidate(const ColumnInfo& ci, float3 c, float hdiag, float extent) {
    float3 v = rot(ci.R, make_float3(c.x - ci.src[0], c.y - ci.src[1], c.z - ci.src[2]));
    const float slack = 1e-3f;
    if (sqrtf(v.x * v.x + v.z * v.z) > hdiag + extent + slack) return false;
    float ymax = v.y + hdiag + slack;
    if (ymax < ci.lim_min || v.y - hdiag - slack >= ci.lim_min + ci.L * ci.ls) return false;
    float k = ymax * ci.inv_sad;
    if (fabsf(v.x) - hdiag - slack > ci.hx * ci.bsx * k) return false;
    if (fabsf(v.z) - hdiag - slack > ci.hy * ci.bsy * k) return false;
    return true;
}

// Mean of ss^3 point samples (d_voxelInterp), or 0 when the voxel centre is
// farther than extent + hdiag from the beamlet axis.
__device__ __forceinline__ float column_value(const ColumnInfo& ci, const float* __restrict__ bev, int x, int y,
                                              int z, float3 vs, float hdiag, float extent, int ss) {
    float3 c = make_float3((x + 0.5f) * vs.x, (y + 0.5f) * vs.y, (z + 0.5f) * vs.z);
    float3 v = rot(ci.R, make_float3(c.x - ci.src[0], c.y - ci.src[1], c.z - ci.src[2]));
    if (sqrtf(v.x * v.x + v.z * v.z) > hdiag + extent) return 0.0f;
    const float inv = 1.0f / ss;
    const float ffx = (float)ci.fx, ffy = (float)ci.fy;
    float acc = 0.0f;
    for (int kk = 0; kk < ss; kk++) {
        const float pz = (z + (kk + 0.5f) * inv) * vs.z;
        for (int jj = 0; jj < ss; jj++) {
            const float py = (y + (jj + 0.5f) * inv) * vs.y;
            for (int ii = 0; ii < ss; ii++) {
                const float px = (x + (ii + 0.5f) * inv) * vs.x;
                float3 cn = to_bev_grid(ci, make_float3(px, py, pz));
                if (cn.x < 0.0f || cn.x > ffx || cn.z < 0.0f || cn.z > ffy) continue;
                acc += bev_fetch(bev, ci.fx, ci.fy, ci.L, (int)floorf(cn.x), (int)floorf(cn.z), (int)floorf(cn.y));
            }
        }
    }
    return acc * (inv * inv * inv);
}

constexpr int kColThreads = 256;

// Pass 1: number of candidate voxels of each beamlet (its row capacity).
__global__ void __launch_bounds__(kColThreads) column_count_kernel(const ColumnInfo* __restrict__ infos,
                                                                  uint32_t* __restrict__ counts, int nx, int ny,
                                                                  float3 vs, float hdiag, float extent) {
    const ColumnInfo ci = infos[blockIdx.x];
    const int bx = ci.box[3] - ci.box[0], by = ci.box[4] - ci.box[1], bz = ci.box[5] - ci.box[2];
    const long long n = (long long)bx * by * bz;
    uint32_t cnt = 0;
    for (long long i = threadIdx.x; i < n; i += kColThreads) {
        int x = ci.box[0] + (int)(i % bx), y = ci.box[1] + (int)((i / bx) % by), z = ci.box[2] + (int)(i / ((long long)bx * by));
        cnt += candidate(ci, make_float3((x + 0.5f) * vs.x, (y + 0.5f) * vs.y, (z + 0.5f) * vs.z), hdiag, extent);
    }
    typedef cub::BlockReduce<uint32_t, kColThreads> Reduce;
    __shared__ typename Reduce::TempStorage tmp;
    uint32_t tot = Reduce(tmp).Sum(cnt);
    if (threadIdx.x == 0) counts[blockIdx.x] = tot;
    (void)nx; (void)ny;
}

// Pass 2: values of the candidates, nonzeros compacted in voxel order into
// the beamlet's temporary segment; writes the row's nnz and max |value|.
__global__ void __launch_bounds__(kColThreads) column_value_kernel(
    const ColumnInfo* __restrict__ infos, const float* const* __restrict__ dose, const uint64_t* __restrict__ cap_off,
    int32_t* __restrict__ tmp_col, float* __restrict__ tmp_val, uint32_t* __restrict__ row_nnz,
    float* __restrict__ row_max, int nx, int ny, float3 vs, float hdiag, float extent, int ss) {
    const ColumnInfo ci = infos[blockIdx.x];
    const float* __restrict__ bev = dose[blockIdx.x];
    const int bx = ci.box[3] - ci.box[0], by = ci.box[4] - ci.box[1], bz = ci.box[5] - ci.box[2];
    const long long n = (long long)bx * by * bz;
    const uint64_t base = cap_off[blockIdx.x];
    const uint64_t cap = cap_off[blockIdx.x + 1] - base;
    typedef cub::BlockScan<uint32_t, kColThreads> Scan;
    typedef cub::BlockReduce<float, kColThreads> RMax;
    __shared__ typename Scan::TempStorage scan_tmp;
    __shared__ typename RMax::TempStorage max_tmp;
    uint32_t written = 0;  // uniform across the block
    float vmax = 0.0f;
    for (long long i0 = 0; i0 < n; i0 += kColThreads) {
        long long i = i0 + threadIdx.x;
        float val = 0.0f;
        int32_t col = 0;
        if (i < n) {
            int x = ci.box[0] + (int)(i % bx), y = ci.box[1] + (int)((i / bx) % by),
                z = ci.box[2] + (int)(i / ((long long)bx * by));
            col = x + nx * (y + ny * z);
            if (candidate(ci, make_float3((x + 0.5f) * vs.x, (y + 0.5f) * vs.y, (z + 0.5f) * vs.z), hdiag, extent))
                val = column_value(ci, bev, x, y, z, vs, hdiag, extent, ss);
        }
        uint32_t nz = val != 0.0f, pos, total;
        Scan(scan_tmp).ExclusiveSum(nz, pos, total);
        if (nz && written + pos < cap) {
            tmp_col[base + written + pos] = col;
            tmp_val[base + written + pos] = val;
        }
        vmax = fmaxf(vmax, fabsf(val));
        written += total;
        __syncthreads();  // scan_tmp reuse
    }
    float m = RMax(max_tmp).Reduce(vmax, cub::Max());
    if (threadIdx.x == 0) {
        row_nnz[blockIdx.x] = written;
        row_max[blockIdx.x] = m;
    }
}

template <typename VT>
__device__ __forceinline__ VT encode(float v, float inv_scale);
template <>
__device__ __forceinline__ float encode<float>(float v, float) { return v; }
template <>
__device__ __forceinline__ __half encode<__half>(float v, float s) { return __float2half_rn(v * s); }
template <>
__device__ __forceinline__ __nv_bfloat16 encode<__nv_bfloat16>(float v, float s) { return __float2bfloat16_rn(v * s); }

// Pass 3: copy each row's segment to its final CSR position.
template <typename VT>
__global__ void column_gather_kernel(const uint64_t* __restrict__ cap_off, const int64_t* __restrict__ row_off,
                                     const int32_t* __restrict__ tmp_col, const float* __restrict__ tmp_val,
                                     const float* __restrict__ inv_scale, int32_t* __restrict__ col,
                                     VT* __restrict__ val) {
    const int r = blockIdx.x;
    const uint64_t src = cap_off[r];
    const int64_t dst = row_off[r], n = row_off[r + 1] - row_off[r];
    const float s = inv_scale ? inv_scale[r] : 1.0f;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        col[dst + i] = tmp_col[src + i];
        val[dst + i] = encode<VT>(tmp_val[src + i], s);
    }
}

}  // namespace

int launch_bev2pvcs(const ColumnInfo& ci, const fd2_volume_t& v, const float* d_bev, float* d_out, size_t pitch,
                    int ss, float extent, cudaStream_t stream) {
    dim3 block(8, 8, 4);
    dim3 grid((v.dim[0] + 7) / 8, (v.dim[1] + 7) / 8, (v.dim[2] + 3) / 4);
    if (ss <= 0)
        bev2pvcs_kernel<<<grid, block, 0, stream>>>(ci, d_bev, d_out, pitch, v.dim[0], v.dim[1], v.dim[2],
                                                    v.voxel_size[0], v.voxel_size[1], v.voxel_size[2]);
    else
        bev2pvcs_ss_kernel<<<grid, block, 0, stream>>>(ci, d_bev, d_out, pitch, v.dim[0], v.dim[1], v.dim[2],
                                                       v.voxel_size[0], v.voxel_size[1], v.voxel_size[2], ss, extent);
    FD2_CHECK_CUDA(cudaGetLastError());
    return FD2_OK;
}

int launch_column_count(const ColumnInfo* d_infos, size_t n, uint32_t* d_counts, const fd2_volume_t& v, float extent,
                        cudaStream_t stream) {
    if (!n) return FD2_OK;
    float3 vs = make_float3(v.voxel_size[0], v.voxel_size[1], v.voxel_size[2]);
    float hdiag = 0.5f * sqrtf(vs.x * vs.x + vs.y * vs.y + vs.z * vs.z);
    column_count_kernel<<<(unsigned)n, kColThreads, 0, stream>>>(d_infos, d_counts, v.dim[0], v.dim[1], vs, hdiag,
                                                                 extent);
    FD2_CHECK_CUDA(cudaGetLastError());
    return FD2_OK;
}

int launch_column_values(const ColumnInfo* d_infos, size_t n, const float* const* d_dose, const uint64_t* d_cap_off,
                         int32_t* d_tmp_col, float* d_tmp_val, uint32_t* d_row_nnz, float* d_row_max,
                         const fd2_volume_t& v, float extent, int ss, cudaStream_t stream) {
    if (!n) return FD2_OK;
    float3 vs = make_float3(v.voxel_size[0], v.voxel_size[1], v.voxel_size[2]);
    float hdiag = 0.5f * sqrtf(vs.x * vs.x + vs.y * vs.y + vs.z * vs.z);
    column_value_kernel<<<(unsigned)n, kColThreads, 0, stream>>>(d_infos, d_dose, d_cap_off, d_tmp_col, d_tmp_val,
                                                                 d_row_nnz, d_row_max, v.dim[0], v.dim[1], vs, hdiag,
                                                                 extent, ss);
    FD2_CHECK_CUDA(cudaGetLastError());
    return FD2_OK;
}

int launch_column_gather(size_t n, const uint64_t* d_cap_off, const int64_t* d_row_off, const int32_t* d_tmp_col,
                         const float* d_tmp_val, const float* d_inv_scale, int32_t* d_col, void* d_val,
                         int value_type, cudaStream_t stream) {
    if (!n) return FD2_OK;
    if (value_type == FD2_VALUES_F16)
        column_gather_kernel<__half><<<(unsigned)n, 256, 0, stream>>>(d_cap_off, d_row_off, d_tmp_col, d_tmp_val,
                                                                      d_inv_scale, d_col, (__half*)d_val);
    else if (value_type == FD2_VALUES_BF16)
        column_gather_kernel<__nv_bfloat16><<<(unsigned)n, 256, 0, stream>>>(
            d_cap_off, d_row_off, d_tmp_col, d_tmp_val, d_inv_scale, d_col, (__nv_bfloat16*)d_val);
    else
        column_gather_kernel<float><<<(unsigned)n, 256, 0, stream>>>(d_cap_off, d_row_off, d_tmp_col, d_tmp_val,
                                                                     nullptr, d_col, (float*)d_val);
    FD2_CHECK_CUDA(cudaGetLastError());
    return FD2_OK;
}

}  // namespace fd2
