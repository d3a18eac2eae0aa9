// flags.cu -- beamlet on/off flags from the PTV mask (IMRT::beamletFlagInit and
// d_beamletFlagInit, IMRTOpt/src/IMRTBeamBundle.cu:130-316).
//
// A fluence pixel of a bundle is on when any of ss x ss sub-rays, sampled at the
// depth of every BEV slice of the bundle, reads the linear-filtered PTV mask above
// zero.  The mask is sampled through the GPU texture unit with the same filtering
// and border mode as the reference, so the decision at the PTV margin (where the
// filter weight quantisation matters) is the same.  This is plan setup, not the
// hot path: one thread per (bundle, pixel).
#include <cstring>
#include <vector>

#include "fd2_internal.cuh"

namespace fd2 {
int calc_range(fd2_beam_t* b, const fd2_volume_t* vol);

namespace {

__device__ __forceinline__ float3 rot_axis(float3 p, float3 r, float t) {
    float s, c;
    __sincosf(t, &s, &c);
    float k = (1.0f - c) * (p.x * r.x + p.y * r.y + p.z * r.z);
    return make_float3(k * r.x + c * p.x + s * (r.y * p.z - r.z * p.y), k * r.y + c * p.y + s * (r.z * p.x - r.x * p.z),
                       k * r.z + c * p.z + s * (r.x * p.y - r.y * p.x));
}

__device__ __forceinline__ float3 bev_to_pvcs(float3 v, float th, float ph, float co) {
    float3 t = rot_axis(v, make_float3(0.f, 1.f, 0.f), -(ph + co));
    float s, c;
    __sincosf(-ph, &s, &c);
    return rot_axis(t, make_float3(s, 0.0f, c), th);
}

__global__ void flags_kernel(const fd2_beam_t* __restrict__ beams, uint8_t* __restrict__ out, cudaTextureObject_t tex,
                             float vx, float vy, float vz, int ss) {
    const fd2_beam_t& b = beams[blockIdx.x];
    const int fx = b.fmap_size[0], fy = b.fmap_size[1];
    const int p = blockIdx.y * blockDim.x + threadIdx.x;
    if (p >= fx * fy) return;
    const int bx = p % fx, by = p / fx;
    uint8_t on = 0;
    for (uint32_t i = 0; i < b.long_dim && !on; i++) {
        float sxd = b.lim_min + i * b.long_spacing;
        for (int j = 0; j < ss && !on; j++)
            for (int k = 0; k < ss && !on; k++) {
                float3 d = make_float3((bx + (j + 0.5f) / ss - fx * 0.5f) * b.beamlet_size[0], b.sad,
                                       (by + (k + 0.5f) / ss - fy * 0.5f) * b.beamlet_size[1]);
                float3 pv = bev_to_pvcs(d, b.angles[0], b.angles[1], b.angles[2]);
                float f = sxd / b.sad;
                float3 c = make_float3((b.source[0] + pv.x * f) / vx, (b.source[1] + pv.y * f) / vy,
                                       (b.source[2] + pv.z * f) / vz);
                if (tex3D<float>(tex, c.x, c.y, c.z) > 0) on = 1;
            }
    }
    out[(size_t)blockIdx.x * fx * fy + p] = on;
}

}  // namespace
}  // namespace fd2

extern "C" int fd2_beamlet_flags(fd2_context* ctx, size_t n, const fd2_bundle_t* bb, const uint8_t* mask,
                                 const fd2_volume_t* vol, int ss, uint8_t* flags_out) {
    FD2_REQUIRE(ctx && bb && mask && vol && flags_out, FD2_ERR_INVALID_ARGUMENT, "beamlet_flags: null argument");
    FD2_REQUIRE(ss > 0 && ss <= 16, FD2_ERR_INVALID_ARGUMENT, "beamlet_flags: super_sampling %d", ss);
    if (n == 0) return FD2_OK;
    const int fx = bb[0].fluence_dim[0], fy = bb[0].fluence_dim[1];
    std::vector<fd2_beam_t> beams(n);
    for (size_t i = 0; i < n; i++) {
        FD2_REQUIRE(bb[i].fluence_dim[0] == fx && bb[i].fluence_dim[1] == fy, FD2_ERR_INVALID_ARGUMENT,
                    "beamlet_flags: bundles must share one fluence dimension");
        fd2_beam_t& b = beams[i];
        std::memset(&b, 0, sizeof(b));
        for (int k = 0; k < 3; k++) { b.isocenter[k] = bb[i].isocenter[k]; b.angles[k] = bb[i].angles[k]; }
        b.beamlet_size[0] = bb[i].beamlet_size[0];
        b.beamlet_size[1] = bb[i].beamlet_size[1];
        b.fmap_size[0] = (uint32_t)fx;
        b.fmap_size[1] = (uint32_t)fy;
        b.sad = bb[i].sad;
        b.long_spacing = bb[i].long_spacing;
        FD2_TRY(fd2::calc_range(&b, vol));
    }
    const size_t nv = (size_t)vol->dim[0] * vol->dim[1] * vol->dim[2];
    std::vector<float> mf(nv);
    for (size_t i = 0; i < nv; i++) mf[i] = mask[i];
    cudaArray_t arr = nullptr;
    cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
    cudaExtent ext = make_cudaExtent(vol->dim[0], vol->dim[1], vol->dim[2]);
    FD2_CHECK_CUDA(cudaMalloc3DArray(&arr, &cd, ext));
    cudaMemcpy3DParms cp;
    std::memset(&cp, 0, sizeof(cp));
    cp.srcPtr = make_cudaPitchedPtr(mf.data(), vol->dim[0] * sizeof(float), vol->dim[0], vol->dim[1]);
    cp.dstArray = arr;
    cp.extent = ext;
    cp.kind = cudaMemcpyHostToDevice;
    cudaError_t err = cudaMemcpy3D(&cp);
    cudaResourceDesc rd;
    std::memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td;
    std::memset(&td, 0, sizeof(td));
    td.filterMode = cudaFilterModeLinear;
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
    td.readMode = cudaReadModeElementType;
    cudaTextureObject_t tex = 0;
    if (err == cudaSuccess) err = cudaCreateTextureObject(&tex, &rd, &td, nullptr);
    fd2_beam_t* d_beams = nullptr;
    uint8_t* d_out = nullptr;
    if (err == cudaSuccess) err = cudaMalloc(&d_beams, n * sizeof(fd2_beam_t));
    if (err == cudaSuccess) err = cudaMalloc(&d_out, n * fx * fy);
    if (err == cudaSuccess) err = cudaMemcpy(d_beams, beams.data(), n * sizeof(fd2_beam_t), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) {
        dim3 grid((unsigned)n, (unsigned)((fx * fy + 255) / 256));
        fd2::flags_kernel<<<grid, 256, 0, ctx->stream>>>(d_beams, d_out, tex, vol->voxel_size[0], vol->voxel_size[1],
                                                         vol->voxel_size[2], ss);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaStreamSynchronize(ctx->stream);
    if (err == cudaSuccess) err = cudaMemcpy(flags_out, d_out, n * fx * fy, cudaMemcpyDeviceToHost);
    if (tex) cudaDestroyTextureObject(tex);
    if (arr) cudaFreeArray(arr);
    if (d_beams) cudaFree(d_beams);
    if (d_out) cudaFree(d_out);
    FD2_CHECK_CUDA(err);
    return FD2_OK;
}
