// cccs.cu -- collapsed-cone convolution/superposition in beam's-eye view.
//
// Restates d_DoseComputeCollective (FastDoseLib/src/DoseComp.cu:217-392).  For
// every forward zenith bin theta (theta <= pi/2) and azimuth phi, the rays of
// all BEV pixels -- translates of one base ray starting at (0.5, 0.5, 0) in
// normalised BEV units -- march slice by slice through voxel boundaries.  Per
// segment of path length p (physical, with divergence) in voxel v:
//     dose[v] += (A/a * XA + B/b * XB) * p * rho[v]       (g == 1, quirk Q1)
//     sum_p[v] += p * rho[v]
//     X <- T[v] (1 - e^{-k p rho}) + e^{-k p rho} X          for (k, X) in {(a, XA), (b, XB)}
// with lateral wrap-around and the recursion reset on crossing an edge (Q4).
// After all azimuths of a slice, dose_bev[s] += sum_phi dose / (sum_p_lastphi + 1e-4)
// (Q2: the path sum of the last azimuth only).
//
// B200 design.  The reference runs one block per beamlet with one thread per
// pixel and a block barrier after every ray step, azimuths in sequence.  Here a
// block owns one beamlet (schedule 0: all zenith bins in turn) or one
// (beamlet, zenith bin) (schedule 1), and each WARP owns one azimuth: its 32
// lanes carry all P rays (P/32 independent recursions per lane, which the
// scheduler interleaves), every lane computes the shared base-ray step itself
// (the warp stays converged, no broadcast), and the only barriers are the
// three per slice that stage the slice's Terma/density pair into shared memory
// and reduce the azimuths.  Within one step the rays of a beamlet deposit into
// distinct voxels (a shift permutation), so the warp-private deposit buffer
// needs only a __syncwarp between steps.
//
// Boundary decisions (next voxel boundary, slice snap, lateral wrap) use
// correctly rounded float operations in the order the reference writes them,
// starting from cone directions computed on the host; the CPU oracle performs
// the identical operations, so both march the same segments bit for bit.
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <vector>

#include "fd2_internal.cuh"

namespace fd2 {

namespace {

constexpr int kStepCap = 1 << 20;  // per-slice step cap (the watchdog bound)
// The 16x16 march is compiled for at most 8 azimuth warps, with the register
// budget of 3 such blocks of 256 threads per SM: 80 registers, 4 blocks of
// 192 threads (6 azimuths).  On the 4pi plan that measured faster than 48,
// 64, 72, 96 and 126 registers (7, 5, 4, 3 and 2 blocks of 192).
constexpr int kFx16Threads = 256;

struct RayGeom {  // per-beamlet scalars the march needs
    float hx, hy;      // fmap_size / 2
    float bsx, bsy;    // beamlet_size
    float ls, lim_min, inv_sad;
    float ffx, ffy;    // fmap size as float
    int fx, fy, P, L;
};

// 1/x on the special-function unit (PTX rcp.approx.ftz.f32).
__device__ __forceinline__ float rcp_sfu(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// A cone direction with what the boundary step needs of it, formed once per
// (zenith, azimuth) pass: the sign of each component and the reciprocal of its
// magnitude (+inf for a zero component).
struct ConeDir {
    float3 d, sg, ra;
};

__device__ __forceinline__ ConeDir make_cone_dir(float3 d) {
    ConeDir k;
    k.d = d;
    k.sg = make_float3(d.x < 0.0f ? -1.0f : 1.0f, d.y < 0.0f ? -1.0f : 1.0f, d.z < 0.0f ? -1.0f : 1.0f);
    k.ra = make_float3(rcp_sfu(fabsf(d.x)), rcp_sfu(fabsf(d.y)), rcp_sfu(fabsf(d.z)));
    return k;
}

// The reference's step to the next boundary along one axis (its build uses
// -use_fast_math, whose a/b is a * rcp.approx(b)):
//     (ceil(c + 1e-3) - c) / d    for d > 0,
//     (floor(c - 1e-3) - c) / d   otherwise.
// With s = sign(d) and u = s c (exact), floor(c - 1e-3) - c = -(ceil(u + 1e-3) - u)
// (round-to-nearest is symmetric under negation) and the sign cancels against
// d's, so both cases are (ceil(u + 1e-3) - u) * rcp(|d|): one rounding
// function and no division per step.  u + 1e-3 and ceil(...) - u are single
// fused operations on the exact product s c, so they round as the
// reference's additions do.  A zero component gives rcp(0) = +inf, so an axis
// the ray does not move along never limits the step (the reference divides
// by zero there and the ray becomes NaN and never ends its slice).
__device__ __forceinline__ float step_to_boundary(float c, float s, float ra) {
    const float up = ceilf(__fmaf_rn(c, s, 1e-3f));
    return __fmul_rn(__fmaf_rn(-c, s, up), ra);
}

// d_nextPoint (DoseComp.cu:76-111): the next voxel-boundary point of the base ray.
__device__ __forceinline__ bool next_point(float3 c, const ConeDir& k, float3& np) {
    const float3 d = k.d;
    float sx = step_to_boundary(c.x, k.sg.x, k.ra.x), sy = step_to_boundary(c.y, k.sg.y, k.ra.y),
          sz = step_to_boundary(c.z, k.sg.z, k.ra.z);
    float take = fminf(fminf(sx, sy), sz);
    np = make_float3(__fmaf_rn(take, d.x, c.x), __fmaf_rn(take, d.y, c.y), __fmaf_rn(take, d.z, c.z));
    bool flag = fabsf(__fsub_rn(np.z, roundf(np.z))) < 1e-4f;
    if (flag) {
        np = make_float3(__fmaf_rn(sz, d.x, c.x), __fmaf_rn(sz, d.y, c.y), roundf(__fmaf_rn(sz, d.z, c.z)));
    }
    return flag;
}

// Lateral voxel column of the segment midpoint (d_calcCoords, DoseComp.cu:147-164).
//
// The reference's r = fmodf(m, ff), plus ff when negative, is computed
// without fmodf: q = floor(m / ff) (the division may round q one off near a
// multiple of ff), r = m - q ff in one fused operation, then one correction by
// +-ff.  For m >= 0 the fused result is exact (the true remainder, or it minus
// or plus ff, all representable by Sterbenz's lemma) and the correction lands
// on the exact remainder, which is what fmodf returns.  For m < 0 the
// reference rounds fmod + ff once; the fused operation rounds the same exact
// value once, or, when q is one off, produces the exact fmod (Sterbenz) and the
// correction rounds fmod + ff once.  Both paths give the reference's float.
__device__ __forceinline__ int mid_index(float b, float n, float ff, int f) {
    const float m = __fmul_rn(__fadd_rn(b, n), 0.5f);
    const float q = floorf(__fdiv_rn(m, ff));
    float r = __fmaf_rn(-q, ff, m);
    if (r < 0.0f)
        r = __fadd_rn(r, ff);
    else if (r >= ff)
        r = __fsub_rn(r, ff);
    const int i = (int)floorf(r);
    return i < f ? i : f - 1;
}

__device__ __forceinline__ bool crosses_edge(float b, float n, float ff) {
    return floorf(__fdividef(b, ff)) != floorf(__fdividef(n, ff));
}

// The same two operations for a 16-pixel map axis.  Division by 16 is exact
// (the fast reciprocal of a power of two is exact), so b / 16 is b * 0.0625; the
// remainder m - 16*trunc(m/16) is exact by Sterbenz's lemma and equals fmodf.
__device__ __forceinline__ int mid_index16(float b, float n) {
    const float m = __fmul_rn(__fadd_rn(b, n), 0.5f);
    float r = __fsub_rn(m, __fmul_rn(16.0f, truncf(__fmul_rn(m, 0.0625f))));
    r = r < 0.0f ? __fadd_rn(r, 16.0f) : r;
    const int i = __float2int_rd(r);
    return i < 16 ? i : 15;
}

__device__ __forceinline__ bool crosses16(float b, float n) {
    return floorf(__fmul_rn(b, 0.0625f)) != floorf(__fmul_rn(n, 0.0625f));
}

// 4 bytes from global to shared memory without passing through registers
// (PTX cp.async), committed as one group per call site; and the wait for all
// of this thread's groups.
__device__ __forceinline__ void cp_async4(float* smem_dst, const float* gsrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// 2^x on the special-function unit (PTX ex2.approx.ftz.f32).  The attenuation
// e^(-k p) is evaluated as 2^(-(k log2 e) p) with k log2 e formed once per
// zenith bin: one multiply and one MUFU operation per exponential.
__device__ __forceinline__ float exp2_sfu(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Segment length sqrt(l2) as l2 * rsqrt(l2) with the SFU reciprocal square
// root (PTX rsqrt.approx.ftz.f32); l2 > 0 for every segment the march takes.
__device__ __forceinline__ float seg_length(float l2) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(l2));
    return l2 * r;
}

// Block: n_phi warps.  Dynamic shared memory: float2 tr[P] (Terma, density of
// the current slice) followed by float2 dp[n_phi][P] (per-azimuth dose and path
// sums); for kFx16 instead float4 wb[n_phi][P] (each azimuth's copy of the
// slice beside its sums) followed by float2 ytab[n_phi][16] (row tables).
// RPL = rays per lane (P <= 32 * RPL); kFx16: the map is 16 x 16.
// kCols: every map of the batch is F x F with F <= 32 -- each lane owns one
// column (lane % F) and the rows lane / F + k j (k = 32 / F lanes per column),
// so the x half of the voxel work is done once per lane and the y half once per
// row and shared by shuffles (16 x 16 maps share it through the row table);
// RPL >= ceil(F / k).
template <int RPL, bool kFx16, bool kCols = false, bool kTab = false>
__global__ void __launch_bounds__(kFx16 || kCols || kTab ? kFx16Threads : 768,
                                  kFx16 ? 3 : ((kCols || kTab) && RPL <= 8 ? 4 : (kCols || kTab ? 3 : 1)))
    cccs_kernel(const fd2_beam_t* __restrict__ beams,
                                                   const float* const* __restrict__ terma,
                                                   const float* const* __restrict__ dens,
                                                   float* const* __restrict__ dose,
                                                   const float4* __restrict__ dirs,  // [beam][n_tf][n_phi]
                                                   ConeParams cp, int split, float* __restrict__ split_out,
                                                   size_t split_stride, DeviceStatus* status,
                                                   const int* __restrict__ order) {
    extern __shared__ float2 smem[];
    __shared__ int s_ctrl[2];  // next slice index, abort flag
    int* s_next = &s_ctrl[0];
    int* s_abort = &s_ctrl[1];
    if (threadIdx.x == 0) *s_abort = 0;
    const int n_tf = cp.n_theta_fwd, n_phi = cp.n_phi;
    // order (optional, one block per beamlet only): the beamlet each block
    // marches, longest first, so the launch ends on short blocks
    const int bi = split ? blockIdx.x / n_tf : (order ? order[blockIdx.x] : blockIdx.x);
    const int t0 = split ? blockIdx.x % n_tf : 0;
    const int t1 = split ? t0 + 1 : n_tf;
    const fd2_beam_t& b = beams[bi];
    RayGeom g;
    g.fx = b.fmap_size[0];
    g.fy = b.fmap_size[1];
    g.P = g.fx * g.fy;
    g.L = (int)b.long_dim;
    g.ffx = (float)g.fx;
    g.ffy = (float)g.fy;
    g.hx = g.fx * 0.5f;
    g.hy = g.fy * 0.5f;
    g.bsx = b.beamlet_size[0];
    g.bsy = b.beamlet_size[1];
    g.ls = b.long_spacing;
    g.lim_min = b.lim_min;
    g.inv_sad = 1.0f / b.sad;
    const size_t pitch = b.TermaBEV_pitch / sizeof(float);

    // kTab: per block, the (column, row) table entries of ray j of each lane
    // (x entry = column, y entry = F + row; all ones past the map), and per
    // azimuth warp the step's 2F halves
    __shared__ uint32_t s_pairs[kTab ? RPL * 32 : 1];
    __shared__ float2 s_htab[kTab ? 8 * 64 : 1];
    if constexpr (kTab) {
        for (int i = threadIdx.x; i < RPL * 32; i += blockDim.x)  // ray i / 32 of lane i % 32 is cell i
            s_pairs[i] = i < g.P ? (uint32_t)(i % g.fx) | (uint32_t)(g.fx + i / g.fx) << 16 : 0xffffffffu;
    }  // visible after the first slice's barrier

    float2* tr = smem;
    float2* dp = smem + g.P;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float2* mydp = dp + (size_t)warp * g.P;
    // kFx16: every azimuth warp keeps its own copy of the slice beside its sums,
    // wb[warp][v] = {Terma, density, dose, path sum}, so a ray step reads all
    // four with one 16-byte load; behind them, each warp's 16-entry row table.
    float4* wb = reinterpret_cast<float4*>(smem);
    float4* mywb = wb + (size_t)warp * g.P;
    float2* ytab = reinterpret_cast<float2*>(wb + (size_t)n_phi * g.P) + 16 * warp;
    const float* __restrict__ T = terma[bi];
    const float* __restrict__ R = dens[bi];
    float* __restrict__ D = dose[bi];

    // per-ray constant pixel coordinates
    float fix[RPL], fiy[RPL];
    bool act[RPL];
    if constexpr (!kFx16 && !kCols) {
#pragma unroll
        for (int j = 0; j < RPL; j++) {
            int r = j * 32 + lane;
            act[j] = r < g.P;
            fix[j] = (float)(r % g.fx);
            fiy[j] = (float)(r / g.fx);
        }
    }
    // kCols: this lane's column and first row, the lanes per column, and the
    // row whose y half this lane computes for the others
    const int kgrp = kCols ? 32 / g.fx : 1;
    const int ccol = kCols ? lane % g.fx : 0, cgrp = kCols ? lane / g.fx : 0;
    const bool clane = kCols && lane < kgrp * g.fx;
    const float fcol = (float)ccol, frow = (float)(kCols && lane < g.fy ? lane : 0);

    // The slice most likely to come next (s + 1, or slice 0 of the next zenith
    // pass), copied by cp.async into s_stage (Terma, then density) during the
    // march and used only if that slice is the one taken.  Each thread copies
    // and later reads the same pixels, so no barrier stands between the two.
    constexpr int kStageP = kFx16 ? 256 : 1024;
    __shared__ float s_stage[2 * kStageP];
    int st_s = -1;

    for (int t = t0; t < t1; t++) {
        const float Aa = cp.A_a[t], Bb = cp.B_b[t];
        const float ka = -cp.a[t] * 1.4426950408889634f, kb = -cp.b[t] * 1.4426950408889634f;  // -k log2(e)
        const float4 d4 = dirs[((size_t)bi * n_tf + t) * n_phi + warp];
        const ConeDir cd = make_cone_dir(make_float3(d4.x, d4.y, d4.z));
        float3 c = make_float3(0.5f, 0.5f, 0.0f);
        float fs = (c.z * g.ls + g.lim_min) * g.inv_sad;  // divergence factor at c, carried step to step
        float XA[RPL], XB[RPL];
#pragma unroll
        for (int j = 0; j < RPL; j++) XA[j] = XB[j] = 0.0f;

        // The slice of every pass is the rounded z of the first azimuth's base
        // ray (DoseComp.cu:300): when that ray ends a slice within 1e-3 below
        // the next plane it steps over it, and the reference skips that slice
        // for this zenith bin; the other azimuths keep marching from wherever
        // they stopped.
        if (threadIdx.x == 0) *s_next = 0;
        __syncthreads();  // the previous pass has finished; s_next is visible
        int s = *s_next;
        while (s < g.L) {
            if constexpr (kFx16) {
                // each pixel's pair goes to every azimuth's copy, sums cleared
                cp_async_wait_all();  // this thread's staged pixels have landed
                for (int v = threadIdx.x; v < g.P; v += blockDim.x) {
                    const float2 t = s == st_s ? make_float2(s_stage[v], s_stage[kStageP + v])
                                               : make_float2(__ldg(T + (size_t)s * pitch + v),
                                                             __ldg(R + (size_t)s * pitch + v));
                    for (int w = 0; w < n_phi; w++) wb[(size_t)w * g.P + v] = make_float4(t.x, t.y, 0.0f, 0.0f);
                }
            } else {
                cp_async_wait_all();  // this thread's staged pixels have landed
                for (int v = threadIdx.x; v < g.P; v += blockDim.x)
                    tr[v] = s == st_s ? make_float2(s_stage[v], s_stage[kStageP + v])
                                      : make_float2(__ldg(T + (size_t)s * pitch + v), __ldg(R + (size_t)s * pitch + v));
                for (int v = lane; v < g.P; v += 32) mydp[v] = make_float2(0.0f, 0.0f);
            }
            __syncthreads();
            st_s = s + 1 < g.L ? s + 1 : (t + 1 < t1 ? 0 : -1);
            if (st_s >= 0)
                for (int v = threadIdx.x; v < g.P; v += blockDim.x) {
                    cp_async4(&s_stage[v], T + (size_t)st_s * pitch + v);
                    cp_async4(&s_stage[kStageP + v], R + (size_t)st_s * pitch + v);
                }
            cp_async_commit();

            int guard = 0;
            for (;;) {
                float3 np;
                const bool flag = next_point(c, cd, np);
                const float fe = (np.z * g.ls + g.lim_min) * g.inv_sad;
                const float dzp = (np.z - c.z) * g.ls;
                if constexpr (kFx16) {
                    // 16x16 map.  A lane's rays share their column, and the rays of
                    // one row share their row: the voxel/edge/length work splits into
                    // an x half per column and a y half per row, 16 of each per step.
                    // Lanes 0-15 evaluate the x half of column `lane`, lanes 16-31 the
                    // y half of row `lane - 16`, in the same instructions (the same
                    // operations on the same inputs as a per-ray evaluation, done once
                    // per column or row instead of per ray).  The half's edge
                    // crossing travels as the sign bit of its |offset|, which enters
                    // the length only squared.  Rows go to the warp's row table
                    // {+-|dy|, 256 * row} (bytes into the slice copy), rows of one
                    // parity together, so a lane reads its eight rows (of its parity)
                    // with four 16-byte loads; lanes 16-31 take their column's x half
                    // from lanes 0-15 by shuffle.
                    const float lx = (float)(lane & 15);
                    const bool yl = lane >= 16;
                    const float hb = __fadd_rn(yl ? c.y : c.x, lx), hn = __fadd_rn(yl ? np.y : np.x, lx);
                    const float bs = yl ? g.bsy : g.bsx;
                    const int hi = mid_index16(hb, hn);
                    const float hq = fabsf((hn - 8.0f) * bs * fe - (hb - 8.0f) * bs * fs);
                    const float hs = crosses16(hb, hn) ? -hq : hq;
                    if (yl) ytab[(lane & 1) * 8 + ((lane & 15) >> 1)] = make_float2(hs, __int_as_float(hi << 8));
                    const int cx = __shfl_sync(0xffffffffu, hi, lane & 15);
                    const float dxs = __shfl_sync(0xffffffffu, hs, lane & 15);
                    const float dxz2 = dxs * dxs + dzp * dzp;
                    const int wx = __float_as_int(dxs);
                    const char* col = reinterpret_cast<const char*>(mywb) + (cx << 4);
                    __syncwarp();
                    const float4* yrow = reinterpret_cast<const float4*>(ytab) + 4 * (lane >> 4);
                    // ray j of this lane: row (lane >> 4) + 2 j
                    auto ray = [&](int j, float dys, int yoff) {
                        const bool wrap = (__float_as_int(dys) | wx) < 0;
                        const float l2 = dxz2 + dys * dys;
                        const float len = seg_length(l2);
                        float4* v = const_cast<float4*>(reinterpret_cast<const float4*>(col + yoff));
                        const float4 e = *v;  // Terma, density, dose, path sum
                        const float p = len * e.y;
                        const float ea = exp2_sfu(ka * p), eb = exp2_sfu(kb * p);
                        const float dep = (Aa * XA[j] + Bb * XB[j]) * p;
                        *reinterpret_cast<float2*>(&v->z) = make_float2(e.z + dep, e.w + p);
                        XA[j] = wrap ? 0.0f : __fmaf_rn(ea, XA[j] - e.x, e.x);
                        XB[j] = wrap ? 0.0f : __fmaf_rn(eb, XB[j] - e.x, e.x);
                    };
#pragma unroll
                    for (int q = 0; q < RPL / 2; q++) {
                        const float4 y2 = yrow[q];
                        ray(2 * q, y2.x, __float_as_int(y2.y));
                        ray(2 * q + 1, y2.z, __float_as_int(y2.w));
                    }
                } else if constexpr (kCols) {
                    const float btx = __fadd_rn(c.x, fcol), ntx = __fadd_rn(np.x, fcol);
                    const int cx = mid_index(btx, ntx, g.ffx, g.fx);
                    const bool wrapx = crosses_edge(btx, ntx, g.ffx);
                    const float dxp = (ntx - g.hx) * g.bsx * fe - (btx - g.hx) * g.bsx * fs;
                    const float dxz2 = dxp * dxp + dzp * dzp;
                    const float bty = __fadd_rn(c.y, frow), nty = __fadd_rn(np.y, frow);
                    const int ycode = mid_index(bty, nty, g.ffy, g.fy) | (crosses_edge(bty, nty, g.ffy) ? 64 : 0);
                    const float dyq = (nty - g.hy) * g.bsy * fe - (bty - g.hy) * g.bsy * fs;
#pragma unroll
                    for (int j = 0; j < RPL; j++) {
                        const int y = cgrp + kgrp * j;
                        const bool on = clane && y < g.fy;
                        const int yc = __shfl_sync(0xffffffffu, ycode, on ? y : 0);
                        const float dyp = __shfl_sync(0xffffffffu, dyq, on ? y : 0);
                        const int mi = on ? cx + g.fx * (yc & 63) : 0;
                        const bool wrap = wrapx || (yc & 64);
                        const float l2 = dxz2 + dyp * dyp;
                        const float len = seg_length(l2);
                        const float2 trv = tr[mi];
                        const float p = len * trv.y;
                        const float ea = exp2_sfu(ka * p), eb = exp2_sfu(kb * p);
                        const float dep = (Aa * XA[j] + Bb * XB[j]) * p;
                        if (on) {
                            float2 acc = mydp[mi];
                            acc.x += dep;
                            acc.y += p;
                            mydp[mi] = acc;
                        }
                        XA[j] = wrap ? 0.0f : __fmaf_rn(ea, XA[j] - trv.x, trv.x);
                        XB[j] = wrap ? 0.0f : __fmaf_rn(eb, XB[j] - trv.x, trv.x);
                    }
                } else if constexpr (kTab) {
                    // F x F map, F <= 24: the rays of lane l are the cells l + 32 j,
                    // so all 32 lanes carry rays whatever F.  The step's 2F halves
                    // (x of each column, y of each row) are evaluated once, one per
                    // lane and round, into the warp's half table {+-|offset|,
                    // bytes into the slice}, the edge crossing as the sign bit;
                    // each ray then reads its column's and its row's entry.
                    float2* ht = s_htab + 64 * warp;
                    for (int h = lane; h < 2 * g.fx; h += 32) {
                        const bool yh = h >= g.fx;
                        const float off = (float)(yh ? h - g.fx : h);
                        const float hb = __fadd_rn(yh ? c.y : c.x, off), hn = __fadd_rn(yh ? np.y : np.x, off);
                        const float ff = yh ? g.ffy : g.ffx, hh = yh ? g.hy : g.hx, bs = yh ? g.bsy : g.bsx;
                        const int hi = mid_index(hb, hn, ff, yh ? g.fy : g.fx);
                        const float hq = fabsf((hn - hh) * bs * fe - (hb - hh) * bs * fs);
                        const float hs = crosses_edge(hb, hn, ff) ? -hq : hq;
                        const int bytes = (int)sizeof(float2) * (yh ? hi * g.fx : hi);
                        ht[h] = make_float2(hs, __int_as_float(bytes));
                    }
                    __syncwarp();
                    const float dz2 = dzp * dzp;
#pragma unroll
                    for (int j = 0; j < RPL; j++) {
                        const uint32_t pr = s_pairs[32 * j + lane];
                        const bool on = pr != 0xffffffffu;
                        const float2 xe = ht[on ? (pr & 0xffffu) : 0], ye = ht[on ? (pr >> 16) : 0];
                        const bool wrap = (__float_as_int(xe.x) | __float_as_int(ye.x)) < 0;
                        const int mb = __float_as_int(xe.y) + __float_as_int(ye.y);
                        const float dxz2 = xe.x * xe.x + dz2;
                        const float l2 = dxz2 + ye.x * ye.x;
                        const float len = seg_length(l2);
                        const float2 trv = *reinterpret_cast<const float2*>(reinterpret_cast<const char*>(tr) + mb);
                        const float p = len * trv.y;
                        const float ea = exp2_sfu(ka * p), eb = exp2_sfu(kb * p);
                        const float dep = (Aa * XA[j] + Bb * XB[j]) * p;
                        if (on) {
                            float2* acc_p = reinterpret_cast<float2*>(reinterpret_cast<char*>(mydp) + mb);
                            float2 acc = *acc_p;
                            acc.x += dep;
                            acc.y += p;
                            *acc_p = acc;
                        }
                        XA[j] = wrap ? 0.0f : __fmaf_rn(ea, XA[j] - trv.x, trv.x);
                        XB[j] = wrap ? 0.0f : __fmaf_rn(eb, XB[j] - trv.x, trv.x);
                    }
                } else {
#pragma unroll
                for (int j = 0; j < RPL; j++) {
                    const float btx = __fadd_rn(c.x, fix[j]), ntx = __fadd_rn(np.x, fix[j]);
                    const float bty = __fadd_rn(c.y, fiy[j]), nty = __fadd_rn(np.y, fiy[j]);
                    const int cx = mid_index(btx, ntx, g.ffx, g.fx);
                    const int cy = mid_index(bty, nty, g.ffy, g.fy);
                    const int mi = cx + cy * g.fx;
                    const bool wrap = crosses_edge(btx, ntx, g.ffx) || crosses_edge(bty, nty, g.ffy);
                    // physical segment length (d_calcLineSeg, DoseComp.cu:114-144)
                    const float dxp = (ntx - g.hx) * g.bsx * fe - (btx - g.hx) * g.bsx * fs;
                    const float dyp = (nty - g.hy) * g.bsy * fe - (bty - g.hy) * g.bsy * fs;
                    const float l2 = dxp * dxp + dyp * dyp + dzp * dzp;
                    const float len = seg_length(l2);
                    const float2 trv = tr[act[j] ? mi : 0];
                    const float p = len * trv.y;
                    const float ea = exp2_sfu(ka * p), eb = exp2_sfu(kb * p);
                    const float dep = (Aa * XA[j] + Bb * XB[j]) * p;
                    if (act[j]) {
                        float2 acc = mydp[mi];
                        acc.x += dep;
                        acc.y += p;
                        mydp[mi] = acc;
                    }
                    XA[j] = wrap ? 0.0f : __fmaf_rn(ea, XA[j] - trv.x, trv.x);
                    XB[j] = wrap ? 0.0f : __fmaf_rn(eb, XB[j] - trv.x, trv.x);
                }
                }
                c = np;
                fs = fe;
                __syncwarp();
                if (flag) break;
                if (++guard >= kStepCap) {
                    if (lane == 0) {
                        atomicExch(&status->code, (int)FD2_ERR_WATCHDOG);
                        *s_abort = 1;
                    }
                    break;
                }
            }
            if (threadIdx.x == 0) {
                // the first azimuth's plane after this slice; it always lies ahead
                const int nxt = (int)roundf(c.z);
                *s_next = nxt > s ? nxt : g.L;
            }
            __syncthreads();
            const int s_new = *s_abort ? g.L : *s_next;
            // reduce azimuths in order; normalise by the last azimuth's path sum
            for (int v = threadIdx.x; v < g.P; v += blockDim.x) {
                float sum = 0.0f, last_sum_p;
                if constexpr (kFx16) {
                    for (int w = 0; w < n_phi; w++) sum += wb[(size_t)w * g.P + v].z;
                    last_sum_p = wb[(size_t)(n_phi - 1) * g.P + v].w;
                } else {
                    for (int w = 0; w < n_phi; w++) sum += dp[(size_t)w * g.P + v].x;
                    last_sum_p = dp[(size_t)(n_phi - 1) * g.P + v].y;
                }
                const float val = sum / (last_sum_p + 1e-4f);
                if (split)
                    split_out[(size_t)blockIdx.x * split_stride + (size_t)s * g.P + v] = val;
                else
                    // this block alone owns beam bi's dose and each (s, v) stays with
                    // one thread, so a fire-and-forget add gives D + val in pass order
                    // without waiting for D's old value
                    atomicAdd(D + (size_t)s * pitch + v, val);
            }
            __syncthreads();  // the sums and the slice are read; s_next was read by every thread
            s = s_new;
        }
    }
    cp_async_wait_all();  // a staged slice that was not taken
}

// dose_bev[s][v] += sum_t planes[t][s][v] (zenith bins in order)
__global__ void cccs_split_reduce(const fd2_beam_t* __restrict__ beams, float* const* __restrict__ dose,
                                  const float* __restrict__ planes, size_t stride, int n_tf) {
    const int bi = blockIdx.y;
    const fd2_beam_t& b = beams[bi];
    const int P = b.fmap_size[0] * b.fmap_size[1];
    const size_t n = (size_t)P * b.long_dim;
    const size_t pitch = b.TermaBEV_pitch / sizeof(float);
    float* D = dose[bi];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        size_t s = i / P, v = i % P;
        float acc = 0.0f;
        for (int t = 0; t < n_tf; t++) acc += planes[((size_t)bi * n_tf + t) * stride + i];
        D[s * pitch + v] += acc;
    }
}

template <int RPL, bool kFx16, bool kCols, bool kTab = false>
int launch_instance(unsigned blocks, int threads, size_t shm, cudaStream_t st, const fd2_beam_t* d_beams,
                    const float* const* T, const float* const* R, float* const* D, const float4* dirs,
                    const ConeParams& cp, int split, float* planes, size_t plane_stride, DeviceStatus* status,
                    const int* order) {
    FD2_CHECK_CUDA(cudaFuncSetAttribute(cccs_kernel<RPL, kFx16, kCols, kTab>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)shm));
    cccs_kernel<RPL, kFx16, kCols, kTab><<<blocks, threads, shm, st>>>(d_beams, T, R, D, dirs, cp, split, planes,
                                                                 plane_stride, status, order);
    FD2_CHECK_CUDA(cudaGetLastError());
    return FD2_OK;
}

// The march for a batch.  map: the common map side F when every map of the
// batch is F x F, else 0.  16 x 16 maps take the 16-pixel instance; other
// common sides up to 32 the shared-column instance (both need 4..8 azimuth
// warps); anything else the general per-ray instance.
int launch_march(int map, int maxP, int n_phi, unsigned blocks, cudaStream_t st, const fd2_beam_t* d_beams,
                 const float* const* T, const float* const* R, float* const* D, const float4* dirs,
                 const ConeParams& cp, int split, float* planes, size_t plane_stride, DeviceStatus* status,
                 const int* order = nullptr) {
    const int threads = 32 * n_phi;
    const size_t shm = (size_t)(1 + n_phi) * maxP * sizeof(float2);
    const bool warps_ok = threads >= 128 && threads <= kFx16Threads;
    if (map == 16 && threads <= kFx16Threads)
        return launch_instance<8, true, false>(blocks, threads, (size_t)n_phi * (256 * sizeof(float4) + 16 * sizeof(float2)),
                                               st, d_beams, T, R, D, dirs, cp, split, planes, plane_stride, status, order);
    if (map > 0 && map <= 24 && warps_ok) {  // half-table instance: rays per lane = ceil(F^2 / 32)
        const int P = map * map;
        if (P <= 64)
            return launch_instance<2, false, false, true>(blocks, threads, shm, st, d_beams, T, R, D, dirs, cp, split,
                                                          planes, plane_stride, status, order);
        if (P <= 160)
            return launch_instance<5, false, false, true>(blocks, threads, shm, st, d_beams, T, R, D, dirs, cp, split,
                                                          planes, plane_stride, status, order);
        if (P <= 256)
            return launch_instance<8, false, false, true>(blocks, threads, shm, st, d_beams, T, R, D, dirs, cp, split,
                                                          planes, plane_stride, status, order);
        if (P <= 416)
            return launch_instance<13, false, false, true>(blocks, threads, shm, st, d_beams, T, R, D, dirs, cp,
                                                           split, planes, plane_stride, status, order);
        return launch_instance<18, false, false, true>(blocks, threads, shm, st, d_beams, T, R, D, dirs, cp, split,
                                                       planes, plane_stride, status, order);
    }
    if (map > 0 && map <= 32 && warps_ok) {
        const int k = 32 / map, rows = (map + k - 1) / k;  // rows per lane
        if (rows <= 8)
            return launch_instance<8, false, true>(blocks, threads, shm, st, d_beams, T, R, D, dirs, cp, split,
                                                   planes, plane_stride, status, order);
        if (rows <= 20)
            return launch_instance<20, false, true>(blocks, threads, shm, st, d_beams, T, R, D, dirs, cp, split,
                                                    planes, plane_stride, status, order);
        if (rows <= 24)
            return launch_instance<24, false, true>(blocks, threads, shm, st, d_beams, T, R, D, dirs, cp, split,
                                                    planes, plane_stride, status, order);
        return launch_instance<32, false, true>(blocks, threads, shm, st, d_beams, T, R, D, dirs, cp, split, planes,
                                                plane_stride, status, order);
    }
    if (maxP <= 256)
        return launch_instance<8, false, false>(blocks, threads, shm, st, d_beams, T, R, D, dirs, cp, split, planes,
                                                plane_stride, status, order);
    return launch_instance<32, false, false>(blocks, threads, shm, st, d_beams, T, R, D, dirs, cp, split, planes,
                                             plane_stride, status, order);
}

// common map side of a batch (F when every map is F x F), else 0
int common_map(int side, const fd2_beam_t& b) {
    const int fx = (int)b.fmap_size[0], fy = (int)b.fmap_size[1];
    if (fx != fy) return 0;
    return side < 0 ? fx : (side == fx ? side : 0);
}

}  // namespace

int launch_cccs_host(fd2_context* ctx, size_t n_beams, const fd2_beam_t* h_beams, const fd2_beam_t* d_beams,
                     const float* const* d_terma, const float* const* d_dens, float* const* d_dose,
                     const fd2_cccs_kernel* k, int schedule, cudaStream_t stream, const int* d_order) {
    if (n_beams == 0) return FD2_OK;
    ConeParams cp{};
    std::vector<int> fwd;
    for (int t = 0; t < k->n_theta; t++)
        if ((double)k->theta[t] <= 1.5707963267948966) fwd.push_back(t);  // forward only, DoseComp.cu:265
    if (fwd.empty()) return FD2_OK;
    cp.n_theta_fwd = (int)fwd.size();
    cp.n_phi = k->n_phi;
    for (size_t i = 0; i < fwd.size(); i++) {
        int t = fwd[i];
        cp.a[i] = k->a[t];
        cp.b[i] = k->b[t];
        cp.A_a[i] = k->A[t] / k->a[t];
        cp.B_b[i] = k->B[t] / k->b[t];
    }
    int maxP = 0, maxL = 0;
    for (size_t i = 0; i < n_beams; i++) {
        FD2_REQUIRE(h_beams[i].TermaBEV_pitch == h_beams[i].DensityBEV_pitch, FD2_ERR_INVALID_ARGUMENT,
                    "dose_compute: Terma and density pitches differ");
        maxP = std::max(maxP, (int)(h_beams[i].fmap_size[0] * h_beams[i].fmap_size[1]));
        maxL = std::max(maxL, (int)h_beams[i].long_dim);
    }
    FD2_REQUIRE(maxP > 0 && maxP <= 1024, FD2_ERR_INVALID_ARGUMENT, "dose_compute: fmap of %d pixels (1..1024)", maxP);
    // direction table [beam][theta_fwd][phi] as float4, evaluated on the device
    ConeAngles ang{};
    ang.n_theta_fwd = (int)fwd.size();
    ang.n_phi = k->n_phi;
    for (size_t t = 0; t < fwd.size(); t++) ang.theta[t] = k->theta[fwd[t]];
    for (int f = 0; f < k->n_phi; f++) ang.phi[f] = k->phi[f];
    size_t dir_bytes = n_beams * fwd.size() * k->n_phi * sizeof(float4);
    size_t plane_stride = (size_t)maxP * maxL;
    size_t plane_bytes = schedule == 1 ? n_beams * fwd.size() * plane_stride * sizeof(float) : 0;
    void* scratch = nullptr;
    FD2_TRY(ctx_scratch(ctx, dir_bytes + plane_bytes + 256, stream, &scratch));
    float4* d_dirs = (float4*)scratch;
    float* d_planes = (float*)((char*)scratch + ((dir_bytes + 255) / 256) * 256);
    FD2_TRY(launch_cone_dirs(d_beams, n_beams, ang, d_dirs, stream));
    // slices a zenith pass skips must contribute zero
    if (plane_bytes) FD2_CHECK_CUDA(cudaMemsetAsync(d_planes, 0, plane_bytes, stream));
    const unsigned blocks = (unsigned)(schedule == 1 ? n_beams * fwd.size() : n_beams);
    int map = -1;
    for (size_t i = 0; i < n_beams && map != 0; i++) map = common_map(map, h_beams[i]);
    FD2_TRY(launch_march(map, maxP, k->n_phi, blocks, stream, d_beams, d_terma, d_dens, d_dose, d_dirs, cp, schedule,
                         d_planes, plane_stride, ctx->d_status, schedule == 1 ? nullptr : d_order));
    ctx->launches += 2;  // direction table + march
    if (schedule == 1) {
        dim3 grid(std::max(1, std::min(64, (int)((plane_stride + 255) / 256))), (unsigned)n_beams);
        cccs_split_reduce<<<grid, 256, 0, stream>>>(d_beams, d_dose, d_planes, plane_stride, (int)fwd.size());
        FD2_CHECK_CUDA(cudaGetLastError());
        ctx->launches += 1;
    }
    return FD2_OK;
}

size_t cccs_scratch_bytes(size_t n_beams, const fd2_beam_t* h_beams, const fd2_cccs_kernel* k, int schedule) {
    size_t n_fwd = 0;
    for (int t = 0; t < k->n_theta; t++)
        if ((double)k->theta[t] <= 1.5707963267948966) n_fwd++;
    size_t maxP = 0, maxL = 0;
    for (size_t i = 0; i < n_beams; i++) {
        maxP = std::max(maxP, (size_t)h_beams[i].fmap_size[0] * h_beams[i].fmap_size[1]);
        maxL = std::max(maxL, (size_t)h_beams[i].long_dim);
    }
    const size_t dir_bytes = n_beams * n_fwd * k->n_phi * sizeof(float4);
    const size_t plane_bytes = schedule == 1 ? n_beams * n_fwd * maxP * maxL * sizeof(float) : 0;
    return dir_bytes + plane_bytes + 256;
}

void cccs_longest_first(size_t n_beams, const fd2_beam_t* h_beams, int* order) {
    std::vector<int> idx(n_beams);
    for (size_t i = 0; i < n_beams; i++) idx[i] = (int)i;
    std::stable_sort(idx.begin(), idx.end(),
                     [&](int a, int b) { return h_beams[a].long_dim > h_beams[b].long_dim; });
    std::copy(idx.begin(), idx.end(), order);
}

// Automatic schedule: split the zenith bins across blocks when the beamlets
// alone cannot fill the device (fewer than ~4 blocks per SM).
int cccs_auto_schedule(const fd2_context* ctx, size_t n_beams) {
    return n_beams < (size_t)ctx->sm_count * 4 ? 1 : 0;
}

}  // namespace fd2

extern "C" int fd2_dose_compute(fd2_context* ctx, size_t fmap_npixels, size_t n_beams, const fd2_beam_t* d_beams,
                                float* const* d_terma, float* const* d_density_bev, float* const* d_dose,
                                const fd2_cccs_kernel* kernel, void* stream) {
    FD2_REQUIRE(ctx && d_beams && d_terma && d_density_bev && d_dose && kernel, FD2_ERR_INVALID_ARGUMENT,
                "dose_compute: null argument");
    FD2_REQUIRE(fmap_npixels > 0 && fmap_npixels <= 1024, FD2_ERR_INVALID_ARGUMENT,
                "dose_compute: fmap_npixels %zu outside 1..1024", fmap_npixels);
    if (n_beams == 0) return FD2_OK;
    // the cone directions are evaluated on the host from the beam descriptors
    std::vector<fd2_beam_t> hb(n_beams);
    cudaStream_t st = (cudaStream_t)stream;
    FD2_CHECK_CUDA(cudaMemcpyAsync(hb.data(), d_beams, n_beams * sizeof(fd2_beam_t), cudaMemcpyDeviceToHost, st));
    FD2_CHECK_CUDA(cudaStreamSynchronize(st));
    return fd2::launch_cccs_host(ctx, n_beams, hb.data(), d_beams, (const float* const*)d_terma,
                                 (const float* const*)d_density_bev, d_dose, kernel,
                                 fd2::cccs_auto_schedule(ctx, n_beams), st, nullptr);
}

extern "C" int fd2_cccs_cone_directions(fd2_context* ctx, const fd2_cccs_kernel* k, size_t n_beams,
                                        const fd2_beam_t* h_beams, float* h_out, size_t n_out) {
    FD2_REQUIRE(ctx && k && h_beams && h_out, FD2_ERR_INVALID_ARGUMENT, "cone_directions: null argument");
    fd2::ConeAngles ang{};
    for (int t = 0; t < k->n_theta; t++)
        if ((double)k->theta[t] <= 1.5707963267948966) ang.theta[ang.n_theta_fwd++] = k->theta[t];
    ang.n_phi = k->n_phi;
    for (int f = 0; f < k->n_phi; f++) ang.phi[f] = k->phi[f];
    const size_t n = n_beams * ang.n_theta_fwd * ang.n_phi;
    FD2_REQUIRE(n_out >= 4 * n, FD2_ERR_CAPACITY, "cone_directions: need %zu floats", 4 * n);
    if (!n) return FD2_OK;
    fd2_beam_t* d_beams = nullptr;
    float4* d_out = nullptr;
    FD2_CHECK_CUDA(cudaMalloc(&d_beams, n_beams * sizeof(fd2_beam_t)));
    cudaError_t e = cudaMalloc(&d_out, n * sizeof(float4));
    if (e == cudaSuccess) e = cudaMemcpy(d_beams, h_beams, n_beams * sizeof(fd2_beam_t), cudaMemcpyHostToDevice);
    int rc = FD2_OK;
    if (e == cudaSuccess) rc = fd2::launch_cone_dirs(d_beams, n_beams, ang, d_out, ctx->stream);
    if (e == cudaSuccess && rc == FD2_OK) e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess && rc == FD2_OK) e = cudaMemcpy(h_out, d_out, n * sizeof(float4), cudaMemcpyDeviceToHost);
    cudaFree(d_beams);
    if (d_out) cudaFree(d_out);
    if (rc) return rc;
    FD2_CHECK_CUDA(e);
    return FD2_OK;
}

// ---------------------------------------------------------------------------
// fd2_dose_compute_static: the CCCS march without any device allocation.
//
// fd2_dose_compute keeps its cone-direction table (and, for batches too small
// to fill the device, per-zenith planes) in the context's scratch buffer,
// which grows with cudaMalloc when a larger batch arrives.  Some hosts cannot
// allow that: a treatment-planning service that hands out every byte of device
// memory from its own pool sized at start-up, or a caller whose device memory
// is owned by another runtime that forbids foreign allocations once its pools
// are set.  Those callers get this entry point: no context, no cudaMalloc, no
// cudaFree, no allocating library.  What it needs beyond the caller's buffers
// -- the status word and the direction table -- lives in one fixed array in
// device global memory, defined below.  Its address belongs to the CUDA
// context that loaded this library's device code, so it is looked up with
// cudaGetSymbolAddress on the first call in each context (once per device
// under the runtime's primary context) and kept under that context's id.
//
// Limits: n_beams * n_forward_theta * n_phi * 16 bytes of directions must fit
// FD2_DOSE_STATIC_DIR_BYTES (256 KiB: 256 beams of an 8 x 8 cone kernel);
// larger batches are rejected with FD2_ERR_CAPACITY before any device work.
// Only schedule 0 runs (every zenith bin of a beamlet in one block, no
// planes), whose dose equals schedule 1's bit for bit.
//
// Every call shares the one array on its device: two calls whose work
// overlaps on the device (different streams, or different host threads with
// no ordering between them) overwrite each other's direction table and status
// word.  Serialise them (same stream, or synchronise in between).

// [0, 256): status word, cleared by every call before its launches (the only
// part that must start at zero); [256, 256 + FD2_DOSE_STATIC_DIR_BYTES):
// direction table [beam][theta_fwd][phi] as float4, fully rewritten by every call.
static __device__ __align__(256) unsigned char fd2_static_scratch[256 + FD2_DOSE_STATIC_DIR_BYTES];

namespace {

constexpr size_t kStaticStatusBytes = 256;  // fd2::DeviceStatus, padded to keep the table aligned
constexpr size_t kStaticDirBytes = FD2_DOSE_STATIC_DIR_BYTES;
constexpr size_t kBeamChunk = 32;  // beam descriptors read back per copy, on the host stack
static_assert(sizeof(fd2::DeviceStatus) <= kStaticStatusBytes, "status word outgrew its slot");

// Looked-up addresses, one per CUDA context.  A context is named by its
// driver-assigned id, which is never reused within a process: a second context
// on the same device, or the primary context recreated after cudaDeviceReset,
// gets a new id and so a fresh lookup (the module may load at another address).
struct StaticAddr {
    unsigned long long ctx_id;
    void* addr;
};
std::vector<StaticAddr> g_static_addr;
std::mutex g_static_mu;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;
std::once_flag g_ctx_fns_once;

// The id of the context current on this thread; false when none is current
// yet or the driver does not offer the query.  The driver functions come
// through the runtime's entry-point table, so the library does not link the
// driver library itself.
bool current_context_id(unsigned long long* id) {
    std::call_once(g_ctx_fns_once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_get_current = (CtxGetCurrentFn)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_get_id = (CtxGetIdFn)f;
    });
    if (!g_ctx_get_current || !g_ctx_get_id) return false;
    CUcontext c = nullptr;
    if (g_ctx_get_current(&c) != CUDA_SUCCESS || c == nullptr) return false;
    return g_ctx_get_id(c, id) == CUDA_SUCCESS;
}

// The device address of fd2_static_scratch in the current context.  Host
// code only sees a stand-in for the array's name, so the address is looked up
// with cudaGetSymbolAddress (which also makes the device's primary context
// current if none is) the first time a context calls, then reused.
int static_scratch_address(unsigned char** out) {
    unsigned long long id = 0;
    if (current_context_id(&id)) {
        std::lock_guard<std::mutex> lock(g_static_mu);
        for (const StaticAddr& s : g_static_addr)
            if (s.ctx_id == id) {
                *out = (unsigned char*)s.addr;
                return FD2_OK;
            }
    }
    void* p = nullptr;
    FD2_CHECK_CUDA(cudaGetSymbolAddress(&p, fd2_static_scratch));
    FD2_REQUIRE(p != nullptr && ((uintptr_t)p & 255) == 0, FD2_ERR_CUDA,
                "dose_compute_static: scratch address %p not 256-byte aligned", p);
    if (current_context_id(&id)) {
        std::lock_guard<std::mutex> lock(g_static_mu);
        g_static_addr.push_back({id, p});
    }
    *out = (unsigned char*)p;
    return FD2_OK;
}

}  // namespace

extern "C" int fd2_dose_compute_static(size_t fmap_npixels, size_t n_beams, const fd2_beam_t* d_beams,
                                       float* const* d_terma, float* const* d_density_bev, float* const* d_dose,
                                       const fd2_cccs_kernel* kernel, int* status_out, void* stream) {
    using namespace fd2;
    FD2_REQUIRE(d_beams && d_terma && d_density_bev && d_dose && kernel, FD2_ERR_INVALID_ARGUMENT,
                "dose_compute_static: null argument");
    FD2_REQUIRE(fmap_npixels > 0 && fmap_npixels <= 1024, FD2_ERR_INVALID_ARGUMENT,
                "dose_compute_static: fmap_npixels %zu outside 1..1024", fmap_npixels);
    if (n_beams == 0) return FD2_OK;
    const fd2_cccs_kernel* k = kernel;
    ConeParams cp{};
    ConeAngles ang{};
    for (int t = 0; t < k->n_theta; t++) {
        if ((double)k->theta[t] > 1.5707963267948966) continue;  // forward bins only, DoseComp.cu:265
        const int i = cp.n_theta_fwd++;
        cp.a[i] = k->a[t];
        cp.b[i] = k->b[t];
        cp.A_a[i] = k->A[t] / k->a[t];
        cp.B_b[i] = k->B[t] / k->b[t];
        ang.theta[i] = k->theta[t];
    }
    if (cp.n_theta_fwd == 0) return FD2_OK;
    cp.n_phi = ang.n_phi = k->n_phi;
    ang.n_theta_fwd = cp.n_theta_fwd;
    for (int f = 0; f < k->n_phi; f++) ang.phi[f] = k->phi[f];
    const size_t per_beam = (size_t)cp.n_theta_fwd * cp.n_phi * sizeof(float4);
    FD2_REQUIRE(n_beams <= kStaticDirBytes / per_beam, FD2_ERR_CAPACITY,
                "dose_compute_static: %zu beams x %d cones need %zu bytes of direction table; the fixed scratch "
                "holds %zu bytes (at most %zu beams of this kernel per call)",
                n_beams, cp.n_theta_fwd * cp.n_phi, n_beams * per_beam, kStaticDirBytes, kStaticDirBytes / per_beam);

    // map sizes of the batch, read back in chunks through a small stack buffer
    cudaStream_t st = (cudaStream_t)stream;
    fd2_beam_t hb[kBeamChunk];
    int maxP = 0;
    int map = -1;
    for (size_t i0 = 0; i0 < n_beams; i0 += kBeamChunk) {
        const size_t m = std::min(kBeamChunk, n_beams - i0);
        FD2_CHECK_CUDA(cudaMemcpyAsync(hb, d_beams + i0, m * sizeof(fd2_beam_t), cudaMemcpyDeviceToHost, st));
        FD2_CHECK_CUDA(cudaStreamSynchronize(st));
        for (size_t i = 0; i < m; i++) {
            FD2_REQUIRE(hb[i].TermaBEV_pitch == hb[i].DensityBEV_pitch, FD2_ERR_INVALID_ARGUMENT,
                        "dose_compute_static: Terma and density pitches differ");
            maxP = std::max(maxP, (int)(hb[i].fmap_size[0] * hb[i].fmap_size[1]));
            map = map == 0 ? 0 : common_map(map, hb[i]);
        }
    }
    FD2_REQUIRE(maxP > 0 && maxP <= 1024, FD2_ERR_INVALID_ARGUMENT,
                "dose_compute_static: fmap of %d pixels (1..1024)", maxP);

    unsigned char* base = nullptr;
    FD2_TRY(static_scratch_address(&base));
    DeviceStatus* d_status = (DeviceStatus*)base;
    float4* d_dirs = (float4*)(base + kStaticStatusBytes);
    FD2_CHECK_CUDA(cudaMemsetAsync(d_status, 0, sizeof(DeviceStatus), st));
    FD2_TRY(launch_cone_dirs(d_beams, n_beams, ang, d_dirs, st));
    const float* const* T = (const float* const*)d_terma;
    const float* const* R = (const float* const*)d_density_bev;
    FD2_TRY(launch_march(map, maxP, cp.n_phi, (unsigned)n_beams, st, d_beams, T, R, d_dose, d_dirs, cp, 0, nullptr, 0,
                         d_status));
    if (status_out)
        FD2_CHECK_CUDA(cudaMemcpyAsync(status_out, &d_status->code, sizeof(int), cudaMemcpyDefault, st));
    return FD2_OK;
}
