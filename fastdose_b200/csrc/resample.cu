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
// farther than extent + hdiag from the beamlet axis.  Sample positions are
// affine in the sub-sample indices, so the beam-frame coordinates are stepped
// incrementally; one reciprocal of the depth per sample gives the divergent
// lateral scale.  SS > 0: ss == SS known at compile time, the innermost line
// of samples unrolled -- independent samples whose loads are predicated
// rather than branched around; SS == 0: any ss, consecutive samples that land
// in the same texel reuse it.  Both add the same values in the same order.
template <int SS>
__device__ __forceinline__ float column_value(const ColumnInfo& ci, const float* __restrict__ bev, int x, int y,
                                              int z, float3 vs, float hdiag, float extent, int ss_rt) {
    const int ss = SS > 0 ? SS : ss_rt;
    const float3 c = make_float3((x + 0.5f) * vs.x, (y + 0.5f) * vs.y, (z + 0.5f) * vs.z);
    const float3 v = rot(ci.R, make_float3(c.x - ci.src[0], c.y - ci.src[1], c.z - ci.src[2]));
    if (sqrtf(v.x * v.x + v.z * v.z) > hdiag + extent) return 0.0f;
    const float inv = 1.0f / ss;
    const float ffx = (float)ci.fx, ffy = (float)ci.fy;
    const float a = inv * vs.x, b = inv * vs.y, cz = inv * vs.z;
    const float3 dI = make_float3(ci.R[0] * a, ci.R[3] * a, ci.R[6] * a);
    const float3 dJ = make_float3(ci.R[1] * b, ci.R[4] * b, ci.R[7] * b);
    const float3 dK = make_float3(ci.R[2] * cz, ci.R[5] * cz, ci.R[8] * cz);
    const float3 p0 = make_float3((x + 0.5f * inv) * vs.x - ci.src[0], (y + 0.5f * inv) * vs.y - ci.src[1],
                                  (z + 0.5f * inv) * vs.z - ci.src[2]);
    const float3 u0 = rot(ci.R, p0);
    const float sx = 1.0f / (ci.bsx * ci.inv_sad), sz = 1.0f / (ci.bsy * ci.inv_sad);
    const int plane = ci.fx * ci.fy;
    int last = -1;
    float last_v = 0.0f, acc = 0.0f;
    for (int kk = 0; kk < ss; kk++) {
        const float3 uk = make_float3(u0.x + kk * dK.x, u0.y + kk * dK.y, u0.z + kk * dK.z);
        for (int jj = 0; jj < ss; jj++) {
            const float3 ukj = make_float3(uk.x + jj * dJ.x, uk.y + jj * dJ.y, uk.z + jj * dJ.z);
            if constexpr (SS > 0) {
#pragma unroll
                for (int ii = 0; ii < SS; ii++) {
                    const float ux = ukj.x + ii * dI.x, uy = ukj.y + ii * dI.y, uz = ukj.z + ii * dI.z;
                    const float r = __fdividef(1.0f, uy);
                    const float cnx = ux * r * sx + ci.hx, cnz = uz * r * sz + ci.hy;
                    const int tx = __float2int_rd(cnx), ty = __float2int_rd(cnz);
                    const int tz = __float2int_rd((uy - ci.lim_min) * ci.inv_ls);
                    const bool in = !(cnx < 0.0f || cnx > ffx || cnz < 0.0f || cnz > ffy) && tx < ci.fx &&
                                    ty < ci.fy && (unsigned)tz < (unsigned)ci.L;
                    if (in) acc += __ldg(bev + (tx + ci.fx * ty + plane * tz));
                }
            } else {
                for (int ii = 0; ii < ss; ii++) {
                    const float ux = ukj.x + ii * dI.x, uy = ukj.y + ii * dI.y, uz = ukj.z + ii * dI.z;
                    const float r = __fdividef(1.0f, uy);
                    const float cnx = ux * r * sx + ci.hx, cnz = uz * r * sz + ci.hy;
                    if (cnx < 0.0f || cnx > ffx || cnz < 0.0f || cnz > ffy) continue;
                    const int tx = __float2int_rd(cnx), ty = __float2int_rd(cnz);
                    const int tz = __float2int_rd((uy - ci.lim_min) * ci.inv_ls);
                    if (tx >= ci.fx || ty >= ci.fy || (unsigned)tz >= (unsigned)ci.L) continue;
                    const int idx = tx + ci.fx * ty + plane * tz;
                    if (idx != last) {
                        last = idx;
                        last_v = __ldg(bev + idx);
                    }
                    acc += last_v;
                }
            }
        }
    }
    return acc * (inv * inv * inv);
}

constexpr int kColThreads = 256;
constexpr int kPerThread = 4;
constexpr int kColChunk = kColThreads * kPerThread;

// Voxels of the row (y, z) of a beamlet's box that can be candidates: the
// candidate test requires the voxel centre within r0 = hdiag + extent + slack
// of the beamlet axis, and along a row the squared distance to the axis is a
// quadratic in x, so the admissible x form one interval.  It is solved in
// double and widened by one voxel on each side, so it contains every x the
// float test accepts; the exact test still runs on each voxel of it.
__device__ __forceinline__ void row_interval(const ColumnInfo& ci, int y, int z, float3 vs, float r0, int& xa,
                                             int& xb) {
    const double cx0 = 0.5 * vs.x - ci.src[0], cy = (y + 0.5) * vs.y - ci.src[1], cz = (z + 0.5) * vs.z - ci.src[2];
    const double A0 = ci.R[0] * cx0 + ci.R[1] * cy + ci.R[2] * cz, A1 = (double)ci.R[0] * vs.x;
    const double C0 = ci.R[6] * cx0 + ci.R[7] * cy + ci.R[8] * cz, C1 = (double)ci.R[6] * vs.x;
    const double a = A1 * A1 + C1 * C1, b = A0 * A1 + C0 * C1, c = A0 * A0 + C0 * C0 - (double)r0 * r0;
    xa = ci.box[0];
    xb = ci.box[3];
    if (a < 1e-12) {  // row parallel to the beamlet axis
        if (c > 1e-6 * r0 * r0) xb = xa;
        return;
    }
    const double disc = b * b - a * c;
    if (disc < 0.0) {
        xb = xa;
        return;
    }
    const double s = sqrt(disc);
    const double lo = (-b - s) / a, hi = (-b + s) / a;
    xa = max(xa, (int)floor(lo) - 1);
    xb = min(xb, (int)ceil(hi) + 2);
    if (xb < xa) xb = xa;
}

// Pass 1: number of candidate voxels of each beamlet (its row capacity).
__global__ void __launch_bounds__(kColThreads) column_count_kernel(const ColumnInfo* __restrict__ infos,
                                                                  uint32_t* __restrict__ counts, int nx, int ny,
                                                                  float3 vs, float hdiag, float extent) {
    const ColumnInfo ci = infos[blockIdx.x];
    const int by = ci.box[4] - ci.box[1], bz = ci.box[5] - ci.box[2];
    const int rows = by * bz;
    const float r0 = hdiag + extent + 2e-3f;
    uint32_t cnt = 0;
    for (int r = threadIdx.x; r < rows; r += kColThreads) {
        const int y = ci.box[1] + r % by, z = ci.box[2] + r / by;
        int xa, xb;
        row_interval(ci, y, z, vs, r0, xa, xb);
        for (int x = xa; x < xb; x++)
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
// Rows (y, z) of the box are taken kColThreads at a time in voxel order; their
// admissible x intervals are concatenated by a scan, and the concatenation is
// tested kColChunk voxels at a time with an order-preserving compaction.  The
// candidates gather in shared memory across chunks and row groups until at
// least kColChunk wait; then all threads compute their values (a few per
// thread, so the block barrier after them waits on a balanced share) and the
// nonzeros are compacted in order into the segment.
__global__ void __launch_bounds__(kColThreads) column_value_kernel(
    const ColumnInfo* __restrict__ infos, const float* const* __restrict__ dose, const uint64_t* __restrict__ cap_off,
    int32_t* __restrict__ tmp_col, float* __restrict__ tmp_val, uint32_t* __restrict__ row_nnz,
    float* __restrict__ row_max, int nx, int ny, float3 vs, float hdiag, float extent, int ss) {
    const ColumnInfo ci = infos[blockIdx.x];
    const float* __restrict__ bev = dose[blockIdx.x];
    const int by = ci.box[4] - ci.box[1], bz = ci.box[5] - ci.box[2];
    const int rows = by * bz;
    const float r0 = hdiag + extent + 2e-3f;
    const uint64_t base = cap_off[blockIdx.x];
    const uint64_t cap = cap_off[blockIdx.x + 1] - base;
    typedef cub::BlockScan<uint32_t, kColThreads> Scan;
    typedef cub::BlockReduce<float, kColThreads> RMax;
    __shared__ typename Scan::TempStorage scan_tmp;
    __shared__ typename RMax::TempStorage max_tmp;
    __shared__ uint32_t s_roff[kColThreads + 1];  // start of each row's interval in the concatenation
    __shared__ int s_rx[kColThreads];             // first x of the row's interval
    __shared__ int s_cand[2 * kColChunk];         // voxel index of the waiting candidates, in order
    __shared__ float s_val[2 * kColChunk];
    uint32_t written = 0;  // uniform across the block
    uint32_t pend = 0;     // candidates waiting in s_cand (uniform)
    float vmax = 0.0f;
    // values of the waiting candidates, then their nonzeros in order
    auto flush = [&]() {
        for (uint32_t k = threadIdx.x; k < pend; k += kColThreads) {
            const int v = s_cand[k];
            const int x = v % nx, y = (v / nx) % ny, z = v / (nx * ny);
            s_val[k] = ss == 5 ? column_value<5>(ci, bev, x, y, z, vs, hdiag, extent, ss)
                               : column_value<0>(ci, bev, x, y, z, vs, hdiag, extent, ss);
        }
        __syncthreads();
        const uint32_t per = (pend + kColThreads - 1) / kColThreads;  // a contiguous run per thread
        const uint32_t k0 = min(pend, threadIdx.x * per), k1 = min(pend, k0 + per);
        uint32_t nzc = 0;
        for (uint32_t k = k0; k < k1; k++) nzc += s_val[k] != 0.0f;
        uint32_t npos, n_nz;
        Scan(scan_tmp).ExclusiveSum(nzc, npos, n_nz);
        for (uint32_t k = k0; k < k1; k++) {
            if (s_val[k] != 0.0f) {
                if (written + npos < cap) {
                    tmp_col[base + written + npos] = s_cand[k];
                    tmp_val[base + written + npos] = s_val[k];
                }
                vmax = fmaxf(vmax, fabsf(s_val[k]));
                npos++;
            }
        }
        written += n_nz;
        pend = 0;
        __syncthreads();  // s_cand / s_val / scan_tmp reuse
    };
    for (int r0w = 0; r0w < rows; r0w += kColThreads) {
        const int r = r0w + threadIdx.x;
        int xa = 0, xb = 0;
        if (r < rows) row_interval(ci, ci.box[1] + r % by, ci.box[2] + r / by, vs, r0, xa, xb);
        uint32_t off, total;
        Scan(scan_tmp).ExclusiveSum((uint32_t)(xb - xa), off, total);
        s_roff[threadIdx.x] = off;
        s_rx[threadIdx.x] = xa;
        if (threadIdx.x == 0) s_roff[kColThreads] = total;
        __syncthreads();
        for (uint32_t f0 = 0; f0 < total; f0 += kColChunk) {
            // candidate test, kPerThread consecutive voxels per thread
            uint32_t flags = 0, cnt = 0;
            int vox[kPerThread];
#pragma unroll
            for (int q = 0; q < kPerThread; q++) {
                const uint32_t f = f0 + threadIdx.x * kPerThread + q;
                vox[q] = -1;
                if (f < total) {
                    int lo = 0, hi = kColThreads;  // last row whose start is <= f
                    while (hi - lo > 1) {
                        const int mid = (lo + hi) >> 1;
                        if (s_roff[mid] <= f) lo = mid; else hi = mid;
                    }
                    const int rr = r0w + lo;
                    const int x = s_rx[lo] + (int)(f - s_roff[lo]), y = ci.box[1] + rr % by, z = ci.box[2] + rr / by;
                    if (candidate(ci, make_float3((x + 0.5f) * vs.x, (y + 0.5f) * vs.y, (z + 0.5f) * vs.z), hdiag,
                                  extent)) {
                        flags |= 1u << q;
                        cnt++;
                        vox[q] = x + nx * (y + ny * z);
                    }
                }
            }
            uint32_t pos, n_cand;
            Scan(scan_tmp).ExclusiveSum(cnt, pos, n_cand);
#pragma unroll
            for (int q = 0; q < kPerThread; q++)  // pend < kColChunk and n_cand <= kColChunk
                if (flags & (1u << q)) s_cand[pend + pos++] = vox[q];
            pend += n_cand;
            __syncthreads();
            if (pend >= (uint32_t)kColChunk) flush();
        }
        __syncthreads();  // s_roff / s_rx reuse
    }
    if (pend) flush();
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

// Row offsets of a batch from its per-row nonzero counts, on the device:
// row_off[0] holds the batch's first offset; row_off[1..n] = row_off[0] +
// inclusive prefix sums.  For 16-bit values also the row scales (row maximum,
// 1 for an empty row) and their reciprocals.
__global__ void __launch_bounds__(1024) column_rows_kernel(const uint32_t* __restrict__ nnz,
                                                           const float* __restrict__ vmax, int64_t n,
                                                           int64_t* __restrict__ row_off, float* __restrict__ scale,
                                                           float* __restrict__ inv_scale) {
    typedef cub::BlockScan<int64_t, 1024> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ int64_t s_carry;
    if (threadIdx.x == 0) s_carry = row_off[0];
    __syncthreads();
    for (int64_t i0 = 0; i0 < n; i0 += 1024) {
        const int64_t i = i0 + threadIdx.x;
        int64_t incl, total;
        Scan(tmp).InclusiveSum(i < n ? (int64_t)nnz[i] : 0, incl, total);
        if (i < n) {
            row_off[i + 1] = s_carry + incl;
            if (scale) {
                const float sc = vmax[i] > 0.0f ? vmax[i] : 1.0f;
                scale[i] = sc;
                inv_scale[i] = 1.0f / sc;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_carry += total;
        __syncthreads();
    }
}

}  // namespace

int launch_column_rows(size_t n, const uint32_t* d_nnz, const float* d_max, int64_t* d_row_off, float* d_scale,
                       float* d_inv_scale, cudaStream_t stream) {
    if (!n) return FD2_OK;
    column_rows_kernel<<<1, 1024, 0, stream>>>(d_nnz, d_max, (int64_t)n, d_row_off, d_scale, d_inv_scale);
    FD2_CHECK_CUDA(cudaGetLastError());
    return FD2_OK;
}

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
