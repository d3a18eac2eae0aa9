// terma.cu -- polyenergetic Terma ray trace into beam's-eye-view (BEV) slabs.
//
// Restates d_TermaComputeCollective (FastDoseLib/src/TermaComp.cu:179-253): for
// every BEV pixel, a ray from the source through the pixel centre at the SAD
// plane is stepped long_spacing/4 along the central-axis projection; each
// sub-step samples the density trilinearly (texel centres at i+0.5, zero outside
// the volume), accumulates radiological path length, and adds
// sum_e fluence_e*E_e*mu_e*exp(-mu_e*rpl) / SXD^2.  Outputs are the slice means
// of Terma and density, [long_dim][pitch/4] per beam.
//
// B200 layout: one thread per (beam, pixel); the 256 pixels of a 16x16 beamlet
// map form one block, so every slice store is a fully coalesced 1 KB row.  The
// density volume is read through the read-only path (L1/L2); neighbouring rays
// touch neighbouring voxels.  Pixels with zero fluence skip the spectrum sum
// (their Terma is exactly zero in the reference too).
#include "fd2_internal.cuh"

namespace fd2 {

namespace {

constexpr int kSubSteps = 4;  // SUPER_SAMPLING, TermaComp.cu:65

__device__ __forceinline__ float fetch(const float* __restrict__ vol, int nx, int ny, int nz, int i, int j, int k) {
    if ((unsigned)i >= (unsigned)nx || (unsigned)j >= (unsigned)ny || (unsigned)k >= (unsigned)nz) return 0.0f;
    return __ldg(vol + (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * (size_t)k));
}

// Trilinear sample at unnormalised coordinates (u, v, w) in voxel units.
__device__ __forceinline__ float trilinear(const float* __restrict__ vol, int nx, int ny, int nz, float u, float v,
                                           float w) {
    float xb = u - 0.5f, yb = v - 0.5f, zb = w - 0.5f;
    float fi = floorf(xb), fj = floorf(yb), fk = floorf(zb);
    float ax = xb - fi, ay = yb - fj, az = zb - fk;
    int i = (int)fi, j = (int)fj, k = (int)fk;
    float c00 = fetch(vol, nx, ny, nz, i, j, k) * (1.0f - ax) + fetch(vol, nx, ny, nz, i + 1, j, k) * ax;
    float c10 = fetch(vol, nx, ny, nz, i, j + 1, k) * (1.0f - ax) + fetch(vol, nx, ny, nz, i + 1, j + 1, k) * ax;
    float c01 = fetch(vol, nx, ny, nz, i, j, k + 1) * (1.0f - ax) + fetch(vol, nx, ny, nz, i + 1, j, k + 1) * ax;
    float c11 =
        fetch(vol, nx, ny, nz, i, j + 1, k + 1) * (1.0f - ax) + fetch(vol, nx, ny, nz, i + 1, j + 1, k + 1) * ax;
    float c0 = c00 * (1.0f - ay) + c10 * ay;
    float c1 = c01 * (1.0f - ay) + c11 * ay;
    return c0 * (1.0f - az) + c1 * az;
}

// BEV -> PVCS rotation of v (inverse of the couch/gantry/collimator rotation).
__device__ __forceinline__ float3 bev_to_pvcs(float3 v, float th, float ph, float co) {
    float s, c;
    sincosf(-(ph + co), &s, &c);
    // about y by -(phi+coll)
    float3 t = make_float3(c * v.x + s * v.z, v.y, -s * v.x + c * v.z);
    // about the couch axis r = (sin(-phi), 0, cos(-phi)) by theta (Rodrigues)
    float sr, cr;
    sincosf(-ph, &sr, &cr);
    float st, ct;
    sincosf(th, &st, &ct);
    float k = (1.0f - ct) * (t.x * sr + t.z * cr);
    return make_float3(k * sr + ct * t.x + st * (-cr * t.y), k * 0.0f + ct * t.y + st * (cr * t.x - sr * t.z),
                       k * cr + ct * t.z + st * (sr * t.y));
}

// 40 registers, 6 blocks per SM: the ray trace waits on density reads, and
// the extra warps hide more of that latency (measured 66.6 against 68.7 ms per
// 400-beam plan at 48 registers; 32 registers spilled and was slower).
template <bool kSkipDark>
__global__ void __launch_bounds__(256, 6) terma_kernel(const fd2_beam_t* __restrict__ beams,
                                                    const float* const* __restrict__ fluence,
                                                    float* const* __restrict__ terma, float* const* __restrict__ dens,
                                                    const float* __restrict__ density, int nx, int ny, int nz,
                                                    float vx, float vy, float vz, SpectrumParams spec) {
    const int bi = blockIdx.x;
    const fd2_beam_t& b = beams[bi];
    const int fx = b.fmap_size[0], fy = b.fmap_size[1];
    const int p = blockIdx.y * blockDim.x + threadIdx.x;
    if (p >= fx * fy) return;
    const int ix = p % fx, iy = p / fx;
    const float fl = fluence[bi][p];
    const float sad = b.sad, ls = b.long_spacing;
    float3 pc = bev_to_pvcs(make_float3((ix + 0.5f - fx * 0.5f) * b.beamlet_size[0], sad,
                                        (iy + 0.5f - fy * 0.5f) * b.beamlet_size[1]),
                            b.angles[0], b.angles[1], b.angles[2]);
    const float k = ls / (sad * kSubSteps);
    const float3 st = make_float3(pc.x * k, pc.y * k, pc.z * k);
    const float stn = sqrtf(st.x * st.x + st.y * st.y + st.z * st.z);
    float sxd = b.lim_min / sad;
    float3 cn = make_float3((b.source[0] + pc.x * sxd) / vx, (b.source[1] + pc.y * sxd) / vy,
                            (b.source[2] + pc.z * sxd) / vz);
    const float3 sn = make_float3(st.x / vx, st.y / vy, st.z / vz);
    const size_t pitch = b.TermaBEV_pitch / sizeof(float);
    float* __restrict__ to = terma[bi];
    float* __restrict__ ro = dens[bi];
    const bool dark = kSkipDark && fl == 0.0f;
    float rpl = 0.0f;
    const uint32_t L = b.long_dim;
    for (uint32_t i = 0; i < L; i++) {
        float tavg = 0.0f, davg = 0.0f;
#pragma unroll
        for (int j = 0; j < kSubSteps; j++) {
            cn.x += sn.x;
            cn.y += sn.y;
            cn.z += sn.z;
            float d = trilinear(density, nx, ny, nz, cn.x, cn.y, cn.z);
            rpl += d * stn;
            davg += d;
            sxd += k;
            if (!dark) {
                float tl = 0.0f;
                for (int e = 0; e < spec.n; e++) tl += spec.fluence_energy_mu[e] * fl * __expf(-spec.mu[e] * rpl);
                tavg += __fdividef(tl, sxd * sxd);
            }
        }
        to[p + pitch * i] = tavg * (1.0f / kSubSteps);
        ro[p + pitch * i] = davg * (1.0f / kSubSteps);
    }
}

}  // namespace

int launch_terma(fd2_context* ctx, size_t fmap_npixels, size_t n_beams, const fd2_beam_t* d_beams, const float* const* d_fluence,
                 float* const* d_terma, float* const* d_dens, const fd2_density* density,
                 const fd2_spectrum* spectrum, int fluence_skip, cudaStream_t stream) {
    (void)ctx;
    if (n_beams == 0) return FD2_OK;
    SpectrumParams sp;
    sp.n = spectrum->n;
    for (int e = 0; e < sp.n; e++) {
        sp.fluence_energy_mu[e] = spectrum->fluence[e] * spectrum->energy[e] * spectrum->mu[e];
        sp.mu[e] = spectrum->mu[e];
    }
    const fd2_volume_t& v = density->vol;
    // blocks per beam cover up to 1024 pixels (the reference's bound: one block per beam)
    dim3 grid((unsigned)n_beams, (unsigned)((fmap_npixels + 255) / 256)), block(256);
    if (fluence_skip)
        terma_kernel<true><<<grid, block, 0, stream>>>(d_beams, d_fluence, d_terma, d_dens, density->d_density,
                                                       v.dim[0], v.dim[1], v.dim[2], v.voxel_size[0],
                                                       v.voxel_size[1], v.voxel_size[2], sp);
    else
        terma_kernel<false><<<grid, block, 0, stream>>>(d_beams, d_fluence, d_terma, d_dens, density->d_density,
                                                        v.dim[0], v.dim[1], v.dim[2], v.voxel_size[0],
                                                        v.voxel_size[1], v.voxel_size[2], sp);
    FD2_CHECK_CUDA(cudaGetLastError());
    if (ctx) ctx->launches += 1;
    return FD2_OK;
}

}  // namespace fd2

extern "C" int fd2_terma_compute(fd2_context* ctx, size_t fmap_npixels, size_t n_beams, const fd2_beam_t* d_beams,
                                 float* const* d_fluence, float* const* d_terma, float* const* d_density_bev,
                                 const fd2_density* density, const fd2_spectrum* spectrum, void* stream) {
    FD2_REQUIRE(ctx && d_beams && d_fluence && d_terma && d_density_bev && density && spectrum,
                FD2_ERR_INVALID_ARGUMENT, "terma_compute: null argument");
    FD2_REQUIRE(fmap_npixels > 0 && fmap_npixels <= 1024, FD2_ERR_INVALID_ARGUMENT,
                "terma_compute: fmap_npixels %zu outside 1..1024", fmap_npixels);
    return fd2::launch_terma(ctx, fmap_npixels, n_beams, d_beams, (const float* const*)d_fluence, d_terma, d_density_bev,
                             density, spectrum, 1, (cudaStream_t)stream);
}
