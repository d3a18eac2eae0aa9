// cccs_dirs.cu -- cone directions of the CCCS march, one per (beamlet, zenith
// bin, azimuth), evaluated on the device exactly as the reference does at the
// start of every zenith bin (FastDoseLib/src/DoseComp.cu:280-290):
//     v = (sin t cos p, sin t sin p, cos t) / (beamlet_size.x, beamlet_size.y, long_spacing)
//     v = v * rsqrt(dot(v, v))
// This translation unit is compiled with the reference's math flags
// (-use_fast_math), so the sine/cosine, the three divisions and the reciprocal
// square root produce the reference's bits.  The march itself is chaotically
// sensitive to these bits (a one-ulp change of one azimuth moves a beamlet's
// dose by percent of its maximum at isolated voxels), so they are reproduced,
// not re-derived.
#include "fd2_internal.cuh"

namespace fd2 {

namespace {

__global__ void cone_dirs_kernel(const fd2_beam_t* __restrict__ beams, int n_beams, ConeAngles ang,
                                 float4* __restrict__ out) {
    const int n_per = ang.n_theta_fwd * ang.n_phi;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_beams * n_per) return;
    const int bi = i / n_per, t = (i % n_per) / ang.n_phi, f = i % ang.n_phi;
    const fd2_beam_t& b = beams[bi];
    float st, ct, sp, cp;
    __sincosf(ang.theta[t], &st, &ct);
    __sincosf(ang.phi[f], &sp, &cp);
    float vx = st * cp, vy = st * sp, vz = ct;
    vx = vx / b.beamlet_size[0];
    vy = vy / b.beamlet_size[1];
    vz = vz / b.long_spacing;
    const float inv = rsqrtf(vx * vx + vy * vy + vz * vz);
    out[i] = make_float4(vx * inv, vy * inv, vz * inv, 0.0f);
}

}  // namespace

int launch_cone_dirs(const fd2_beam_t* d_beams, size_t n_beams, const ConeAngles& ang, float4* d_out,
                     cudaStream_t stream) {
    const size_t n = n_beams * ang.n_theta_fwd * ang.n_phi;
    if (!n) return FD2_OK;
    cone_dirs_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(d_beams, (int)n_beams, ang, d_out);
    FD2_CHECK_CUDA(cudaGetLastError());
    return FD2_OK;
}

}  // namespace fd2
