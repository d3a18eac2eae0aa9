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

// BeamOrientationOptimization (IMRTOpt/src/IMRTOptimize.cu:197-388): the
// per-beam VOIMatricesT / SpFluenceGrad lists become the all-beam device
// matrices AT and D with their beam row blocks; the initial fluence is an
// argument (the reference draws it from rand() after srand(10086)).  Outputs as
// the reference's costs / activeBeams / activeNorms, plus the kept beams'
// fluence on the device.
inline bool BeamOrientationOptimization(fd2_context* ctx, const fd2_matrix* AT, const fd2_matrix* D,
                                        const std::vector<int64_t>& beam_rows, const std::vector<int64_t>& d_rows,
                                        int64_t n_ptv, int64_t n_oar, const std::vector<float>& maxDose,
                                        const std::vector<float>& maxWeightsLong,
                                        const std::vector<float>& minDoseTarget,
                                        const std::vector<float>& minDoseTargetWeights,
                                        const std::vector<float>& OARWeightsLong, const fd2_boo_params_t& params,
                                        const float* d_x0, std::vector<float>& costs, std::vector<int>& activeBeams,
                                        std::vector<float>& activeNorms, float* d_x) {
    const size_t n_beams = beam_rows.size() - 1;
    costs.assign(params.max_iter, 0.0f);
    std::vector<int32_t> active(n_beams);
    activeNorms.assign(n_beams, 0.0f);
    fd2_boo_result_t res{};
    if (fd2_beam_orientation_optimization(ctx, AT, D, (int64_t)n_beams, beam_rows.data(), d_rows.data(), n_ptv, n_oar,
                                          maxDose.data(), maxWeightsLong.data(), minDoseTarget.data(),
                                          minDoseTargetWeights.data(), OARWeightsLong.data(), &params, d_x0,
                                          costs.data(), active.data(), activeNorms.data(), d_x, &res) != FD2_OK)
        return true;
    activeBeams.assign(active.begin(), active.begin() + res.n_active);
    activeNorms.resize(res.n_active);
    return false;
}

}  // namespace IMRT
