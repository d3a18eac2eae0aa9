// ref_harness.cu -- extern "C" driver around the REFERENCE's own sources
// (FastDoseLib/src/*.cu, IMRTOpt/src/IMRTBeamBundle.cu, IMRTOpt/src/IMRTgeom.cu),
// compiled unmodified from the read-only reference checkout by oracle/build_ref.sh
// into oracle/_ref/libfdref.so.  TEST INFRASTRUCTURE: used to pin the oracle and
// the CUDA kernels (golden fixtures under tests/golden/) and as the
// "reference CUDA on the same B200" timing.  Never linked by the product.
//
// The harness follows the per-beam steps of IMRT::DoseMatConstruction
// (IMRTOpt/src/IMRTDoseMat.cu:183-259) but zeroes the BEV dose buffers before
// each call: the reference never clears them between beams (they accumulate),
// which this harness does not reproduce.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>

#include "fastdose.cuh"
#include "IMRTBeamBundle.cuh"
#include "IMRTgeom.cuh"
#include "IMRTDoseMat.cuh"
#include "IMRTDoseMatEns.cuh"
#include "IMRTArgs.h"
#include "../../include/fd2.h"

namespace fd = fastdose;

static_assert(sizeof(fd::d_BEAM_d) == sizeof(fd2_beam_t), "d_BEAM_d layout");
static_assert(offsetof(fd::d_BEAM_d, beamlet_size) == offsetof(fd2_beam_t, beamlet_size), "layout");
static_assert(offsetof(fd::d_BEAM_d, fmap_size) == offsetof(fd2_beam_t, fmap_size), "layout");
static_assert(offsetof(fd::d_BEAM_d, sad) == offsetof(fd2_beam_t, sad), "layout");
static_assert(offsetof(fd::d_BEAM_d, angles) == offsetof(fd2_beam_t, angles), "layout");
static_assert(offsetof(fd::d_BEAM_d, lim_min) == offsetof(fd2_beam_t, lim_min), "layout");
static_assert(offsetof(fd::d_BEAM_d, long_dim) == offsetof(fd2_beam_t, long_dim), "layout");
static_assert(offsetof(fd::d_BEAM_d, source) == offsetof(fd2_beam_t, source), "layout");
static_assert(offsetof(fd::d_BEAM_d, TermaBEV_pitch) == offsetof(fd2_beam_t, TermaBEV_pitch), "layout");
static_assert(offsetof(fd::d_BEAM_d, DensityBEV_pitch) == offsetof(fd2_beam_t, DensityBEV_pitch), "layout");

// MatCSREnsemble keeps its per-matrix nonzero counts private; the reference
// declares this validation routine a friend of the class (IMRTDoseMatEns.cuh)
// and defines it in a debug source the harness does not build, so the harness
// defines it to read the counts out.
static std::vector<size_t>* g_nnz_sink = nullptr;
bool IMRT::sparseValidation(const MatCSREnsemble* matEns) {
    if (g_nnz_sink) *g_nnz_sink = matEns->NonZeroElements;
    return 0;
}

std::map<std::string, std::any>& IMRT::harness_args() {
    static std::map<std::string, std::any> m;
    return m;
}

static void to_host_beam(const fd2_beam_t& s, fd::BEAM_h& b) {
    b.isocenter = make_float3(s.isocenter[0], s.isocenter[1], s.isocenter[2]);
    b.beamlet_size = make_float2(s.beamlet_size[0], s.beamlet_size[1]);
    b.fmap_size = make_uint2(s.fmap_size[0], s.fmap_size[1]);
    b.sad = s.sad;
    b.angles = make_float3(s.angles[0], s.angles[1], s.angles[2]);
    b.long_spacing = s.long_spacing;
    b.lim_min = s.lim_min;
    b.lim_max = s.lim_max;
    b.long_dim = s.long_dim;
    b.source = make_float3(s.source[0], s.source[1], s.source[2]);
}

static void from_host_beam(const fd::BEAM_h& b, fd2_beam_t& s) {
    std::memset(&s, 0, sizeof(s));
    s.isocenter[0] = b.isocenter.x; s.isocenter[1] = b.isocenter.y; s.isocenter[2] = b.isocenter.z;
    s.beamlet_size[0] = b.beamlet_size.x; s.beamlet_size[1] = b.beamlet_size.y;
    s.fmap_size[0] = b.fmap_size.x; s.fmap_size[1] = b.fmap_size.y;
    s.sad = b.sad;
    s.angles[0] = b.angles.x; s.angles[1] = b.angles.y; s.angles[2] = b.angles.z;
    s.long_spacing = b.long_spacing;
    s.lim_min = b.lim_min; s.lim_max = b.lim_max; s.long_dim = b.long_dim;
    s.source[0] = b.source.x; s.source[1] = b.source.y; s.source[2] = b.source.z;
    size_t pitch = (size_t)b.fmap_size.x * b.fmap_size.y * sizeof(float);
    s.TermaBEV_pitch = pitch;
    s.DensityBEV_pitch = pitch;
}

static void host_density(const fd2_volume_t* v, fd::DENSITY_h& d) {
    d.VoxelSize = make_float3(v->voxel_size[0], v->voxel_size[1], v->voxel_size[2]);
    d.VolumeDim = make_uint3(v->dim[0], v->dim[1], v->dim[2]);
    d.BBoxStart = make_uint3(v->bbox_start[0], v->bbox_start[1], v->bbox_start[2]);
    d.BBoxDim = make_uint3(v->bbox_dim[0], v->bbox_dim[1], v->bbox_dim[2]);
}

extern "C" {

// ---------------------------------------------------------------- host geometry
void ref_rotate_axis(const float* p, const float* r, float t, float* out) {
    float3 o = fd::rotateAroundAxisAtOriginRHS(make_float3(p[0], p[1], p[2]), make_float3(r[0], r[1], r[2]), t);
    out[0] = o.x; out[1] = o.y; out[2] = o.z;
}

void ref_rotate_beam(const float* v, float th, float ph, float co, int inverse, float* out) {
    float3 in = make_float3(v[0], v[1], v[2]);
    float3 o = inverse ? fd::inverseRotateBeamAtOriginRHS(in, th, ph, co) : fd::rotateBeamAtOriginRHS(in, th, ph, co);
    out[0] = o.x; out[1] = o.y; out[2] = o.z;
}

int ref_calc_range(fd2_beam_t* beam, const fd2_volume_t* vol) {
    fd::BEAM_h b;
    to_host_beam(*beam, b);
    fd::DENSITY_h d;
    host_density(vol, d);
    int st = b.calc_range(d) ? 1 : 0;
    fd2_beam_t out;
    from_host_beam(b, out);
    *beam = out;
    return st;
}

int ref_beamlet_init(const fd2_bundle_t* bb, int ix, int iy, const fd2_volume_t* vol, fd2_beam_t* out) {
    IMRT::BeamBundle bundle;
    bundle.isocenter = make_float3(bb->isocenter[0], bb->isocenter[1], bb->isocenter[2]);
    bundle.beamletSize = make_float2(bb->beamlet_size[0], bb->beamlet_size[1]);
    bundle.fluenceDim = make_int2(bb->fluence_dim[0], bb->fluence_dim[1]);
    bundle.SAD = bb->sad;
    bundle.angles = make_float3(bb->angles[0], bb->angles[1], bb->angles[2]);
    bundle.longSpacing = bb->long_spacing;
    bundle.subFluenceDim = make_int2(bb->sub_fluence_dim[0], bb->sub_fluence_dim[1]);
    bundle.subFluenceOn = make_int2(bb->sub_fluence_on[0], bb->sub_fluence_on[1]);
    fd::DENSITY_h d;
    host_density(vol, d);
    fd::BEAM_h b;
    int st = bundle.beamletInit(b, ix, iy, d) ? 1 : 0;
    from_host_beam(b, *out);
    return st;
}

// ---------------------------------------------------------------- GPU stages
// beamletFlagInit (IMRTBeamBundle.cu:130-266) for n bundles sharing one fluence dim.
int ref_beamlet_flags(int n, const fd2_bundle_t* bbs, const uint8_t* ptv, const fd2_volume_t* vol,
                      const float* density, uint8_t* flags_out) {
    std::vector<IMRT::BeamBundle> bundles(n);
    for (int i = 0; i < n; i++) {
        IMRT::BeamBundle& bundle = bundles[i];
        const fd2_bundle_t* bb = &bbs[i];
        bundle.isocenter = make_float3(bb->isocenter[0], bb->isocenter[1], bb->isocenter[2]);
        bundle.beamletSize = make_float2(bb->beamlet_size[0], bb->beamlet_size[1]);
        bundle.fluenceDim = make_int2(bb->fluence_dim[0], bb->fluence_dim[1]);
        bundle.SAD = bb->sad;
        bundle.angles = make_float3(bb->angles[0], bb->angles[1], bb->angles[2]);
        bundle.longSpacing = bb->long_spacing;
        bundle.subFluenceDim = make_int2(bb->sub_fluence_dim[0], bb->sub_fluence_dim[1]);
        bundle.subFluenceOn = make_int2(bb->sub_fluence_on[0], bb->sub_fluence_on[1]);
    }
    fd::DENSITY_h d;
    host_density(vol, d);
    size_t nv = (size_t)vol->dim[0] * vol->dim[1] * vol->dim[2];
    std::vector<uint8_t> mask(ptv, ptv + nv);
    if (IMRT::beamletFlagInit(bundles, mask, d)) return 1;
    cudaDeviceSynchronize();
    size_t P = (size_t)bbs[0].fluence_dim[0] * bbs[0].fluence_dim[1];
    for (int i = 0; i < n; i++)
        for (size_t j = 0; j < P; j++) flags_out[i * P + j] = bundles[i].beamletFlag[j];
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Terma + CCCS (+ optional batched interpolation into the dense matrix) for one
// batch of beamlets sharing fmap size, as one iteration of DoseMatConstruction.
// BEV outputs are [n][long_dim_max][P] (rows beyond a beamlet's long_dim are 0);
// dense_out is [n][nVoxels] or NULL.  times_ms[0..2] = Terma, CCCS, interp.
int ref_dose_batch(int n, const fd2_beam_t* beams, const float* fluence, const float* density,
                   const fd2_volume_t* vol, int nkern, const float* energy, const float* sfl,
                   const float* mu, const float* mu_en, int n_theta, const float* theta_mid,
                   const float* A, const float* a, const float* B, const float* b, int n_phi,
                   const float* phi, float extent, float* terma_out, float* dens_out,
                   float* dose_out, float* dense_out, float* times_ms, int repeats) {
    fd::DENSITY_h dh;
    host_density(vol, dh);
    size_t nv = (size_t)vol->dim[0] * vol->dim[1] * vol->dim[2];
    dh.density.assign(density, density + nv);
    fd::DENSITY_d dd;
    fd::density_h2d(dh, dd);

    fd::SPECTRUM_h sp;
    sp.nkernels = nkern;
    sp.energy.assign(energy, energy + nkern);
    sp.fluence.assign(sfl, sfl + nkern);
    sp.mu.assign(mu, mu + nkern);
    sp.mu_en.assign(mu_en, mu_en + nkern);
    if (sp.bind_spectrum()) return 3;

    fd::KERNEL_h kh;
    kh.nTheta = n_theta;
    kh.nPhi = n_phi;
    kh.thetaMiddle.assign(theta_mid, theta_mid + n_theta);
    kh.paramA.assign(A, A + n_theta);
    kh.parama.assign(a, a + n_theta);
    kh.paramB.assign(B, B + n_theta);
    kh.paramb.assign(b, b + n_theta);
    kh.phiAngles.assign(phi, phi + n_phi);
    if (kh.bind_kernel()) return 4;

    int fx = beams[0].fmap_size[0], fy = beams[0].fmap_size[1];
    size_t P = (size_t)fx * fy;
    int maxL = 0;
    for (int i = 0; i < n; i++) maxL = std::max(maxL, (int)beams[i].long_dim);
    size_t pitch = P * sizeof(float);
    std::vector<fd2_beam_t> hb(beams, beams + n);
    for (auto& x : hb) { x.TermaBEV_pitch = pitch; x.DensityBEV_pitch = pitch; }

    size_t per = P * maxL;
    float *dT, *dR, *dD, *dF;
    fd::d_BEAM_d* dB;
    cudaMalloc(&dT, per * n * sizeof(float));
    cudaMalloc(&dR, per * n * sizeof(float));
    cudaMalloc(&dD, per * n * sizeof(float));
    cudaMalloc(&dF, P * n * sizeof(float));
    cudaMalloc(&dB, n * sizeof(fd::d_BEAM_d));
    cudaMemcpy(dB, hb.data(), n * sizeof(fd2_beam_t), cudaMemcpyHostToDevice);
    for (int i = 0; i < n; i++) cudaMemcpy(dF + i * P, fluence, P * sizeof(float), cudaMemcpyHostToDevice);
    std::vector<float*> hT(n), hR(n), hD(n), hF(n);
    for (int i = 0; i < n; i++) {
        hT[i] = dT + per * i; hR[i] = dR + per * i; hD[i] = dD + per * i; hF[i] = dF + P * i;
    }
    float **aT, **aR, **aD, **aF;
    cudaMalloc(&aT, n * sizeof(float*)); cudaMalloc(&aR, n * sizeof(float*));
    cudaMalloc(&aD, n * sizeof(float*)); cudaMalloc(&aF, n * sizeof(float*));
    cudaMemcpy(aT, hT.data(), n * sizeof(float*), cudaMemcpyHostToDevice);
    cudaMemcpy(aR, hR.data(), n * sizeof(float*), cudaMemcpyHostToDevice);
    cudaMemcpy(aD, hD.data(), n * sizeof(float*), cudaMemcpyHostToDevice);
    cudaMemcpy(aF, hF.data(), n * sizeof(float*), cudaMemcpyHostToDevice);

    cudaEvent_t e0, e1, e2, e3;
    cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2); cudaEventCreate(&e3);
    float tt = 0, td = 0, ti = 0;
    float* d_dense = nullptr;
    size_t dense_size = (size_t)n * nv;
    if (dense_out) cudaMalloc(&d_dense, dense_size * sizeof(float));
    if (repeats < 1) repeats = 1;
    for (int rep = 0; rep < repeats; rep++) {
        cudaMemset(dT, 0, per * n * sizeof(float));
        cudaMemset(dR, 0, per * n * sizeof(float));
        cudaMemset(dD, 0, per * n * sizeof(float));
        cudaDeviceSynchronize();
        cudaEventRecord(e0);
        fd::TermaComputeCollective(P, n, dB, aF, aT, aR, dd, sp, 0);
        cudaEventRecord(e1);
        fd::DoseComputeCollective(P, n, dB, aT, aR, aD, n_theta, n_phi, 0);
        cudaEventRecord(e2);
        if (dense_out) {
            // the buffers DoseMatConstruction sets up (IMRTDoseMat.cu:143-175)
            int2 packDim;
            packDim.x = (int)ceilf(sqrtf((float)n));
            packDim.y = (int)ceilf((float)n / packDim.x);
            int3 packArrayDim{packDim.x * fx, packDim.y * fy, maxL};
            size_t packSize = (size_t)packArrayDim.x * packArrayDim.y * packArrayDim.z;
            float* packArray;
            cudaMalloc(&packArray, packSize * sizeof(float));
            cudaMemset(packArray, 0, packSize * sizeof(float));
            dim3 sbs{8, 8, 8};
            dim3 sgs{(vol->dim[0] - 1 + sbs.x) / sbs.x, (vol->dim[1] - 1 + sbs.y) / sbs.y,
                     (vol->dim[2] - 1 + sbs.z) / sbs.z};
            size_t preSize = (size_t)sgs.x * sgs.y * sgs.z * n;
            // d_superVoxelInterp runs a 4^3-block grid that can exceed the
            // supervoxel grid and then writes up to one padded grid past the
            // array; allocate that slack so those writes stay in bounds.
            size_t slack = (size_t)((sgs.x + 3) / 4 * 4) * ((sgs.y + 3) / 4 * 4) * ((sgs.z + 3) / 4 * 4);
            bool* pre;
            cudaMalloc(&pre, (preSize + slack) * sizeof(bool));
            int* longArr;
            cudaMalloc(&longArr, n * sizeof(int));
            std::vector<int> hl(n);
            for (int i = 0; i < n; i++) hl[i] = hb[i].long_dim;
            cudaMemcpy(longArr, hl.data(), n * sizeof(int), cudaMemcpyHostToDevice);
            cudaArray* arr;
            cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
            cudaMalloc3DArray(&arr, &cd, make_cudaExtent(packArrayDim.x, packArrayDim.y, packArrayDim.z));
            cudaStream_t ms;
            cudaStreamCreate(&ms);
            cudaDeviceSynchronize();
            cudaEventRecord(e2);
            IMRT::BEV2PVCSInterp(d_dense, dense_size, dB, n, dd, aD, P, pre, preSize, packArray, packDim,
                                 make_int2(fx, fy), packArrayDim, &arr, longArr, extent, 0, ms);
            cudaEventRecord(e3);
            cudaEventSynchronize(e3);
            cudaStreamDestroy(ms);
            cudaFreeArray(arr);
            cudaFree(longArr);
            cudaFree(pre);
            cudaFree(packArray);
        } else {
            cudaEventRecord(e3);
        }
        cudaEventSynchronize(e3);
        float a1, a2, a3;
        cudaEventElapsedTime(&a1, e0, e1);
        cudaEventElapsedTime(&a2, e1, e2);
        cudaEventElapsedTime(&a3, e2, e3);
        tt += a1; td += a2; ti += a3;
    }
    if (times_ms) { times_ms[0] = tt / repeats; times_ms[1] = td / repeats; times_ms[2] = ti / repeats; }
    if (terma_out) cudaMemcpy(terma_out, dT, per * n * sizeof(float), cudaMemcpyDeviceToHost);
    if (dens_out) cudaMemcpy(dens_out, dR, per * n * sizeof(float), cudaMemcpyDeviceToHost);
    if (dose_out) cudaMemcpy(dose_out, dD, per * n * sizeof(float), cudaMemcpyDeviceToHost);
    if (dense_out) {
        cudaMemcpy(dense_out, d_dense, dense_size * sizeof(float), cudaMemcpyDeviceToHost);
        cudaFree(d_dense);
    }
    cudaError_t err = cudaDeviceSynchronize();
    cudaFree(dT); cudaFree(dR); cudaFree(dD); cudaFree(dF); cudaFree(dB);
    cudaFree(aT); cudaFree(aR); cudaFree(aD); cudaFree(aF);
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2); cudaEventDestroy(e3);
    return err == cudaSuccess ? 0 : 5;
}

// fd::BEV2PVCS (TermaComp.cu:97-150), or with ssfactor > 0
// fd::BEV2PVCS_SuperSampling (geom.cu:343-474), of one beam's BEV array onto
// the volume through a linear-filter, border-addressed texture.  The output
// starts at zero (the supersampled form writes only voxels inside `extent`
// whose average reaches eps_fastdose).
static int bev2pvcs_common(const fd2_beam_t* beam, const float* bev, const fd2_volume_t* vol, int ssfactor,
                           float extent, float* out) {
    fd::DENSITY_d dd;
    dd.VoxelSize = make_float3(vol->voxel_size[0], vol->voxel_size[1], vol->voxel_size[2]);
    dd.VolumeDim = make_uint3(vol->dim[0], vol->dim[1], vol->dim[2]);
    int fx = beam->fmap_size[0], fy = beam->fmap_size[1], L = beam->long_dim;
    cudaArray* arr;
    cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
    cudaExtent ext = make_cudaExtent(fx, fy, L);
    cudaMalloc3DArray(&arr, &cd, ext);
    cudaMemcpy3DParms cp = {0};
    cp.srcPtr = make_cudaPitchedPtr((void*)bev, fx * sizeof(float), fx, fy);
    cp.dstArray = arr;
    cp.extent = ext;
    cp.kind = cudaMemcpyHostToDevice;
    cudaMemcpy3D(&cp);
    cudaResourceDesc rd;
    std::memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td;
    std::memset(&td, 0, sizeof(td));
    td.filterMode = cudaFilterModeLinear;
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
    td.readMode = cudaReadModeElementType;
    cudaTextureObject_t tex;
    cudaCreateTextureObject(&tex, &rd, &td, nullptr);
    cudaPitchedPtr outp;
    cudaMalloc3D(&outp, make_cudaExtent(vol->dim[0] * sizeof(float), vol->dim[1], vol->dim[2]));
    cudaMemset(outp.ptr, 0, outp.pitch * vol->dim[1] * vol->dim[2]);
    fd::BEAM_d bd;
    fd::BEAM_h bh;
    to_host_beam(*beam, bh);
    bd.isocenter = bh.isocenter; bd.beamlet_size = bh.beamlet_size; bd.fmap_size = bh.fmap_size;
    bd.sad = bh.sad; bd.angles = bh.angles; bd.long_spacing = bh.long_spacing; bd.lim_min = bh.lim_min;
    bd.lim_max = bh.lim_max; bd.long_dim = bh.long_dim; bd.source = bh.source;
    bd.fluence = nullptr; bd.TermaBEV = nullptr; bd.DensityBEV = nullptr; bd.DoseBEV = nullptr;
    if (ssfactor > 0)
        fd::BEV2PVCS_SuperSampling(bd, dd, outp, tex, ssfactor, extent, 0);
    else
        fd::BEV2PVCS(bd, dd, outp, tex, 0);
    cudaMemcpy2D(out, vol->dim[0] * sizeof(float), outp.ptr, outp.pitch, vol->dim[0] * sizeof(float),
                 (size_t)vol->dim[1] * vol->dim[2], cudaMemcpyDeviceToHost);
    cudaError_t err = cudaDeviceSynchronize();
    cudaDestroyTextureObject(tex);
    cudaFreeArray(arr);
    cudaFree(outp.ptr);
    dd.densityArray = nullptr;  // not owned
    return err == cudaSuccess ? 0 : 5;
}

int ref_bev2pvcs(const fd2_beam_t* beam, const float* bev, const fd2_volume_t* vol, float* out) {
    return bev2pvcs_common(beam, bev, vol, 0, 0.0f, out);
}

int ref_bev2pvcs_ss(const fd2_beam_t* beam, const float* bev, const fd2_volume_t* vol, int ssfactor, float extent,
                    float* out) {
    return bev2pvcs_common(beam, bev, vol, ssfactor < 1 ? 1 : ssfactor, extent, out);
}


// IMRT::DoseMatConstruction (IMRTDoseMat.cu:14-301) run step by step with the
// reference's own functions over n_bundles bundles that share one fluence
// grid: per beam (concurrency 1, :31) the descriptors go up, then
// fd::TermaComputeCollective, fd::DoseComputeCollective, IMRT::BEV2PVCSInterp
// into the dense [beamlets x voxels] matrix and MatCSREnsemble::addMat (cuSPARSE
// DenseToSparse), with the buffers DoseMatConstruction sets up (:37-175).
// Two departures, both for safety on this hardware:
// - the supervoxel flag array gets slack: d_superVoxelInterp (IMRTgeom.cu:
//   471-516) runs a grid of 4^3-thread blocks over the supervoxel grid with no
//   bounds check, so when that grid is not a multiple of 4 (a volume side that
//   is not a multiple of 32 voxels) it writes up to one padded grid past the
//   array; DoseMatConstruction allocates it exactly (:158-161);
// - the BEV dose buffer is zeroed before each beam: DoseComputeCollective
//   accumulates (+=) and the reference never clears it between beams.
// flags[b][i] marks bundle b's active beamlets (beamletFlagInit's output);
// each bundle's beamlets come from BeamBundle::beamletsInit.  Outputs:
// nnz_out[b], the matrix of bundle b; times_ms[0..4] = Terma, CCCS,
// interpolation, dense-to-CSR, and the whole loop (CUDA events on the default
// stream); n_beamlets_out = the beamlets computed.  est_nnz_per_mat is
// EstNonZeroElementsPerMat (IMRTArgs.cpp default 6e6).
int ref_dose_mat_steps(int n_bundles, const fd2_bundle_t* bbs, const uint8_t* flags, const float* density,
                       const fd2_volume_t* vol, int nkern, const float* energy, const float* sfl, const float* mu,
                       const float* mu_en, int n_theta, const float* theta_mid, const float* A, const float* a,
                       const float* B, const float* b, int n_phi, const float* phi, float extent,
                       uint64_t est_nnz_per_mat, uint64_t* nnz_out, float* times_ms, int64_t* n_beamlets_out) {
    fd::DENSITY_h dh;
    host_density(vol, dh);
    size_t nv = (size_t)vol->dim[0] * vol->dim[1] * vol->dim[2];
    dh.density.assign(density, density + nv);
    fd::DENSITY_d dd;
    fd::density_h2d(dh, dd);

    fd::SPECTRUM_h sp;
    sp.nkernels = nkern;
    sp.energy.assign(energy, energy + nkern);
    sp.fluence.assign(sfl, sfl + nkern);
    sp.mu.assign(mu, mu + nkern);
    sp.mu_en.assign(mu_en, mu_en + nkern);
    if (sp.bind_spectrum()) return 3;
    fd::KERNEL_h kh;
    kh.nTheta = n_theta;
    kh.nPhi = n_phi;
    kh.thetaMiddle.assign(theta_mid, theta_mid + n_theta);
    kh.paramA.assign(A, A + n_theta);
    kh.parama.assign(a, a + n_theta);
    kh.paramB.assign(B, B + n_theta);
    kh.paramb.assign(b, b + n_theta);
    kh.phiAngles.assign(phi, phi + n_phi);
    if (kh.bind_kernel()) return 4;

    // beam bundles and their beamlets, as BeamBundleInit leaves them
    const int sfd = bbs[0].sub_fluence_dim[0], son = bbs[0].sub_fluence_on[0];
    const size_t P = (size_t)bbs[0].fluence_dim[0] * bbs[0].fluence_dim[1];
    std::vector<IMRT::BeamBundle> bundles(n_bundles);
    for (int i = 0; i < n_bundles; i++) {
        IMRT::BeamBundle& bu = bundles[i];
        const fd2_bundle_t* bb = &bbs[i];
        bu.isocenter = make_float3(bb->isocenter[0], bb->isocenter[1], bb->isocenter[2]);
        bu.beamletSize = make_float2(bb->beamlet_size[0], bb->beamlet_size[1]);
        bu.fluenceDim = make_int2(bb->fluence_dim[0], bb->fluence_dim[1]);
        bu.SAD = bb->sad;
        bu.angles = make_float3(bb->angles[0], bb->angles[1], bb->angles[2]);
        bu.longSpacing = bb->long_spacing;
        bu.subFluenceDim = make_int2(bb->sub_fluence_dim[0], bb->sub_fluence_dim[1]);
        bu.subFluenceOn = make_int2(bb->sub_fluence_on[0], bb->sub_fluence_on[1]);
        bu.beamletFlag.assign(P, false);
        for (size_t j = 0; j < P; j++) bu.beamletFlag[j] = flags[i * P + j] != 0;
        bu.beamletsInit(dh);
    }
    // bundles without an active beamlet get no matrix (nnz 0): the ensemble's
    // offset table is laid out from the row counts it is given
    int maxNb = 0, maxL = 0;
    int64_t total = 0;
    std::vector<size_t> rowsPerMat;
    std::vector<int> used;
    for (int i = 0; i < n_bundles; i++) {
        nnz_out[i] = 0;
        const size_t r = bundles[i].beams_h.size();
        if (r == 0) continue;
        used.push_back(i);
        rowsPerMat.push_back(r);
        maxNb = std::max(maxNb, (int)r);
        total += (int64_t)r;
        for (auto& bh : bundles[i].beams_h) maxL = std::max(maxL, (int)bh.long_dim);
    }
    if (n_beamlets_out) *n_beamlets_out = total;
    if (maxNb == 0) return 0;

    cudaEvent_t ev[6];
    for (auto& e : ev) cudaEventCreate(&e);
    float acc[5] = {0, 0, 0, 0, 0};
    int rc = 0;
    {
        IMRT::MatCSREnsemble ens(rowsPerMat, nv, (size_t)est_nnz_per_mat * used.size());
        const size_t denseSize = (size_t)maxNb * nv;
        float* d_dense = nullptr;
        cudaMalloc(&d_dense, denseSize * sizeof(float));
        const size_t sP = (size_t)sfd * sfd;
        const size_t per = sP * maxL;
        fd::d_BEAM_d* d_beams = nullptr;
        float *dF, *dR, *dT, *dD;
        cudaMalloc(&d_beams, maxNb * sizeof(fd::d_BEAM_d));
        cudaMalloc(&dF, maxNb * sP * sizeof(float));
        cudaMalloc(&dR, per * maxNb * sizeof(float));
        cudaMalloc(&dT, per * maxNb * sizeof(float));
        cudaMalloc(&dD, per * maxNb * sizeof(float));
        // one centred subFluenceOn^2 open square per beamlet (:91-109)
        std::vector<float> single(sP, 0.0f), hF(maxNb * sP);
        const int lead = (int)((sfd - son) * 0.5f);
        for (int j = lead; j < lead + son; j++)
            for (int i = lead; i < lead + son; i++) single[i + j * sfd] = 1.0f;
        for (int k = 0; k < maxNb; k++) std::copy(single.begin(), single.end(), hF.begin() + k * sP);
        cudaMemcpy(dF, hF.data(), hF.size() * sizeof(float), cudaMemcpyHostToDevice);
        std::vector<float*> pF(maxNb), pR(maxNb), pT(maxNb), pD(maxNb);
        for (int k = 0; k < maxNb; k++) {
            pF[k] = dF + k * sP; pR[k] = dR + k * per; pT[k] = dT + k * per; pD[k] = dD + k * per;
        }
        float **aF, **aR, **aT, **aD;
        cudaMalloc(&aF, maxNb * sizeof(float*)); cudaMalloc(&aR, maxNb * sizeof(float*));
        cudaMalloc(&aT, maxNb * sizeof(float*)); cudaMalloc(&aD, maxNb * sizeof(float*));
        cudaMemcpy(aF, pF.data(), maxNb * sizeof(float*), cudaMemcpyHostToDevice);
        cudaMemcpy(aR, pR.data(), maxNb * sizeof(float*), cudaMemcpyHostToDevice);
        cudaMemcpy(aT, pT.data(), maxNb * sizeof(float*), cudaMemcpyHostToDevice);
        cudaMemcpy(aD, pD.data(), maxNb * sizeof(float*), cudaMemcpyHostToDevice);
        int2 packDim;
        packDim.x = (int)ceilf(sqrtf((float)maxNb));
        packDim.y = (int)ceilf((float)maxNb / packDim.x);
        int3 packArrayDim{packDim.x * sfd, packDim.y * sfd, maxL};
        float* packArray = nullptr;
        cudaMalloc(&packArray, (size_t)packArrayDim.x * packArrayDim.y * packArrayDim.z * sizeof(float));
        dim3 sbs{8, 8, 8};
        dim3 sgs{(vol->dim[0] - 1 + sbs.x) / sbs.x, (vol->dim[1] - 1 + sbs.y) / sbs.y,
                 (vol->dim[2] - 1 + sbs.z) / sbs.z};
        const size_t preSize = (size_t)sgs.x * sgs.y * sgs.z * maxNb;
        const size_t slack = (size_t)((sgs.x + 3) / 4 * 4) * ((sgs.y + 3) / 4 * 4) * ((sgs.z + 3) / 4 * 4);
        bool* pre = nullptr;
        cudaMalloc(&pre, (preSize + slack) * sizeof(bool));
        int* d_long = nullptr;
        cudaMalloc(&d_long, maxNb * sizeof(int));
        cudaArray* arr;
        cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
        cudaMalloc3DArray(&arr, &cd, make_cudaExtent(packArrayDim.x, packArrayDim.y, packArrayDim.z));
        cudaStream_t ms;
        cudaStreamCreate(&ms);
        const size_t pitch = sP * sizeof(float);
        cudaDeviceSynchronize();
        cudaEventRecord(ev[5]);
        for (int i : used) {
            const int n = (int)bundles[i].beams_h.size();
            std::vector<fd::d_BEAM_d> hb;
            std::vector<int> hl;
            for (auto& bh : bundles[i].beams_h) {
                hb.push_back(fd::d_BEAM_d(bh, pitch, pitch));
                hl.push_back(bh.long_dim);
            }
            cudaMemcpyAsync(d_beams, hb.data(), n * sizeof(fd::d_BEAM_d), cudaMemcpyHostToDevice, 0);
            cudaMemcpyAsync(d_long, hl.data(), n * sizeof(int), cudaMemcpyHostToDevice, 0);
            cudaMemsetAsync(dD, 0, per * n * sizeof(float), 0);
            cudaEventRecord(ev[0]);
            fd::TermaComputeCollective(sP, n, d_beams, aF, aT, aR, dd, sp, 0);
            cudaEventRecord(ev[1]);
            fd::DoseComputeCollective(sP, n, d_beams, aT, aR, aD, kh.nTheta, kh.nPhi, 0);
            cudaEventRecord(ev[2]);
            IMRT::BEV2PVCSInterp(d_dense, denseSize, d_beams, n, dd, aD, pitch / sizeof(float), pre, preSize,
                                 packArray, packDim, make_int2(sfd, sfd), packArrayDim, &arr, d_long, extent, 0, ms);
            cudaEventRecord(ev[3]);
            if (ens.addMat(d_dense, n, nv)) rc = 6;
            cudaEventRecord(ev[4]);
            cudaEventSynchronize(ev[4]);
            float t;
            for (int k = 0; k < 4; k++) {
                cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
                acc[k] += t;
            }
        }
        cudaEventSynchronize(ev[4]);
        cudaEventElapsedTime(&acc[4], ev[5], ev[4]);
        std::vector<size_t> nnz;
        g_nnz_sink = &nnz;
        IMRT::sparseValidation(&ens);
        g_nnz_sink = nullptr;
        for (size_t k = 0; k < used.size() && k < nnz.size(); k++) nnz_out[used[k]] = nnz[k];
        cudaStreamDestroy(ms);
        cudaFreeArray(arr);
        cudaFree(d_long); cudaFree(pre); cudaFree(packArray);
        cudaFree(aF); cudaFree(aR); cudaFree(aT); cudaFree(aD);
        cudaFree(dF); cudaFree(dR); cudaFree(dT); cudaFree(dD); cudaFree(d_beams); cudaFree(d_dense);
    }
    for (int k = 0; k < 5; k++) times_ms[k] = acc[k];
    for (auto& e : ev) cudaEventDestroy(e);
    cudaError_t err = cudaDeviceSynchronize();
    if (rc) return rc;
    return err == cudaSuccess ? 0 : 5;
}

}  // extern "C"
