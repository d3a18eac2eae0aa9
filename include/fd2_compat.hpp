// fd2_compat.hpp -- the reference's C++ call names over the fd2 C ABI.
//
// For C++ callers of FastDoseLib / IMRTOpt that switch to this library: the
// functions below keep the reference's namespaces, names, argument order and
// return convention (bool, true = failure), and take fd2 handles where the
// reference takes its classes (DENSITY_d, SPECTRUM_h and KERNEL_h become
// fd2_density / fd2_spectrum / fd2_cccs_kernel made on an fd2_context; the
// reference's __constant__ spectrum and kernel tables become those explicit
// handles).  Nothing here exits the process: on failure fd2_last_error()
// holds the message.  Header-only; link libfd2.so.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "fd2.h"
#include "fd2_imrt.h"
#include "fd2_opt.h"

namespace fastdose {

// TermaComputeCollective (FastDoseLib/include/TermaComp.cuh:7-17)
inline bool TermaComputeCollective(size_t fmap_npixels, size_t n_beams, const fd2_beam_t* d_beams,
                                   float* const* d_fluence_array, float* const* d_TermaBEV_array,
                                   float* const* d_DensityBEV_array, fd2_context* ctx, const fd2_density* density_d,
                                   const fd2_spectrum* spectrum_h, cudaStream_t stream = 0) {
    return fd2_terma_compute(ctx, fmap_npixels, n_beams, d_beams, d_fluence_array, d_TermaBEV_array,
                             d_DensityBEV_array, density_d, spectrum_h, stream) != FD2_OK;
}

// DoseComputeCollective (FastDoseLib/include/DoseComp.cuh:9-19); the reference's
// nTheta/nPhi arguments select from its global kernel table, here the handle.
inline bool DoseComputeCollective(size_t fmap_npixels, size_t n_beams, const fd2_beam_t* d_beams,
                                  float* const* TermaBEV_array, float* const* DensityBEV_array,
                                  float* const* DoseBEV_array, fd2_context* ctx, const fd2_cccs_kernel* kernel_h,
                                  cudaStream_t stream = 0) {
    return fd2_dose_compute(ctx, fmap_npixels, n_beams, d_beams, TermaBEV_array, DensityBEV_array, DoseBEV_array,
                            kernel_h, stream) != FD2_OK;
}

// BEV2PVCS (FastDoseLib/include/TermaComp.cuh:30-36) and
// BEV2PVCS_SuperSampling (FastDoseLib/include/geom.cuh:39-47): one beam's BEV
// array to a pitched PVCS volume.
inline bool BEV2PVCS(fd2_context* ctx, const fd2_beam_t& beam_d, const fd2_density* density_d, const float* d_bev,
                     float* d_pvcs, size_t pitch_bytes, cudaStream_t stream = 0) {
    return fd2_bev2pvcs(ctx, &beam_d, density_d, d_bev, d_pvcs, pitch_bytes, stream) != FD2_OK;
}

inline bool BEV2PVCS_SuperSampling(fd2_context* ctx, const fd2_beam_t& beam_d, const fd2_density* density_d,
                                   const float* d_bev, float* d_pvcs, size_t pitch_bytes, int ssfactor = 5,
                                   float extent = 2.0f, cudaStream_t stream = 0) {
    return fd2_bev2pvcs_supersampling(ctx, &beam_d, density_d, d_bev, d_pvcs, pitch_bytes, ssfactor, extent,
                                      stream) != FD2_OK;
}

}  // namespace fastdose

namespace IMRT {

// DoseMatConstruction (IMRTOpt/include/IMRTDoseMat.cuh:71-78): the beams'
// beamlets are concatenated in beam order; the getarg globals of the
// reference are the fields of params.
inline bool DoseMatConstruction(fd2_context* ctx, const std::vector<uint32_t>& beamlets_per_beam,
                                const std::vector<fd2_beam_t>& beamlets, const std::vector<float>& fluence,
                                const fd2_density* density_d, const fd2_spectrum* spectrum_h,
                                const fd2_cccs_kernel* kernel_h, const fd2_dosemat_params_t& params,
                                fd2_csr_ensemble** matEns, cudaStream_t stream = 0) {
    return fd2_dose_mat_construct(ctx, beamlets_per_beam.size(), beamlets_per_beam.data(), beamlets.data(),
                                  fluence.data(), density_d, spectrum_h, kernel_h, &params, matEns,
                                  stream) != FD2_OK;
}

// BOO_IMRT_L2OneHalf_gpu_QL (IMRTOpt/include/IMRTOptimize.cuh:53-70)
inline bool BOO_IMRT_L2OneHalf_gpu_QL(fd2_opt_problem* problem, const std::vector<int64_t>& beam_offsets,
                                      std::vector<float>& beamWeights, int showTrigger, int changeWeightsTrigger,
                                      int iters_global, const std::vector<int32_t>& pruneTrigger,
                                      int numBeamsWeWant, fd2_opt_state_t& state) {
    return fd2_boo_l2onehalf(problem, (int64_t)beamWeights.size(), beam_offsets.data(), beamWeights.data(),
                             showTrigger, changeWeightsTrigger, iters_global, pruneTrigger.data(),
                             (int)pruneTrigger.size(), numBeamsWeWant, &state) != FD2_OK;
}

// polish_BOO_IMRT_gpu (IMRTOpt/include/IMRTOptimize.cuh:87-100)
inline bool polish_BOO_IMRT_gpu(fd2_opt_problem* problem, int iters_global, int iters_local,
                                fd2_opt_state_t& state) {
    return fd2_polish(problem, iters_global, iters_local, &state) != FD2_OK;
}

}  // namespace IMRT
