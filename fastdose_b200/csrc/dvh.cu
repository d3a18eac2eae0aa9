// dvh.cu -- cumulative dose-volume histograms of a dose vector.
//
// The reference draws a structure's DVH from its sorted voxel doses
// (IMRTOpt/src/doseAnalyze.py:53-62: volume fraction receiving at least each
// dose).  Here the same curve is binned on the device: structure s lists its
// voxels (CSR offsets into one index array, so structures may overlap); voxel
// v falls in bin k = floor(dose[v] / width), clamped to [0, n_bins); each
// block counts into shared-memory bins and adds them to the structure's global
// counts; a second kernel turns the counts into the cumulative form
// cum[s][k] = voxels of s with bin >= k (the voxels receiving at least
// k * width).  Counts are integers: the result does not depend on scheduling.
#include <algorithm>

#include "../../include/fd2_opt.h"
#include "fd2_internal.cuh"

namespace fd2 {
namespace {

constexpr int kDvhThreads = 256;

// grid: (blocks per structure, structures); dynamic shared memory: n_bins counters
__global__ void dvh_count_kernel(const float* __restrict__ dose, int64_t n_voxels, const int64_t* __restrict__ off,
                                 const int32_t* __restrict__ voxels, int n_bins, float width,
                                 unsigned long long* __restrict__ counts, int* __restrict__ bad) {
    extern __shared__ unsigned int bins[];
    const int s = blockIdx.y;
    for (int k = threadIdx.x; k < n_bins; k += blockDim.x) bins[k] = 0;
    __syncthreads();
    const int64_t a = off[s], b = off[s + 1];
    for (int64_t i = a + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = voxels[i];
        if (v < 0 || v >= n_voxels) {  // not a voxel of the dose: counted, skipped
            atomicAdd(bad, 1);
            continue;
        }
        const float d = dose[v];
        const float q = floorf(__fdiv_rn(d, width));
        const int k = q < 0.0f ? 0 : (q >= (float)n_bins ? n_bins - 1 : (int)q);
        atomicAdd(&bins[k], 1u);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n_bins; k += blockDim.x)
        if (bins[k]) atomicAdd(&counts[(size_t)s * n_bins + k], (unsigned long long)bins[k]);
}

// one block per structure: suffix sums of its counts, in place
__global__ void dvh_cumulate_kernel(unsigned long long* __restrict__ counts, int n_bins) {
    if (threadIdx.x != 0) return;
    unsigned long long* c = counts + (size_t)blockIdx.x * n_bins;
    unsigned long long acc = 0;
    for (int k = n_bins - 1; k >= 0; k--) {
        acc += c[k];
        c[k] = acc;
    }
}

}  // namespace
}  // namespace fd2

extern "C" int fd2_dvh(fd2_context* ctx, const float* d_dose, int64_t n_voxels, int64_t n_structs,
                       const int64_t* h_struct_offsets, const int32_t* d_voxels, int n_bins, float bin_width,
                       unsigned long long* d_cumulative, void* stream) {
    FD2_REQUIRE(ctx && d_dose && (n_structs == 0 || (h_struct_offsets && d_voxels && d_cumulative)),
                FD2_ERR_INVALID_ARGUMENT, "dvh: null argument");
    FD2_REQUIRE(n_structs >= 0 && n_structs <= 65535 && n_bins > 0 && n_bins <= 12288 && bin_width > 0.0f,
                FD2_ERR_INVALID_ARGUMENT, "dvh: %lld structures (<= 65535), %d bins (1..12288), width %g (> 0)",
                (long long)n_structs, n_bins, (double)bin_width);
    if (n_structs == 0) return FD2_OK;
    FD2_REQUIRE(h_struct_offsets[0] == 0, FD2_ERR_INVALID_ARGUMENT, "dvh: structure offsets must start at 0");
    for (int64_t s = 0; s < n_structs; s++)
        FD2_REQUIRE(h_struct_offsets[s + 1] >= h_struct_offsets[s], FD2_ERR_INVALID_ARGUMENT,
                    "dvh: structure offsets decrease at %lld", (long long)s);
    cudaStream_t st = (cudaStream_t)stream;
    FD2_CHECK_CUDA(cudaMemsetAsync(d_cumulative, 0, (size_t)n_structs * n_bins * sizeof(unsigned long long), st));
    const size_t shm = (size_t)n_bins * sizeof(unsigned int);
    if (shm > 48 * 1024)
        FD2_CHECK_CUDA(cudaFuncSetAttribute(fd2::dvh_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)shm));
    const int per = std::max(1, (ctx->sm_count > 0 ? ctx->sm_count : 148) * 4 / (int)std::min<int64_t>(n_structs, 148));
    // [0]: out-of-range voxel count; then the structure offsets
    void* scratch = nullptr;
    const size_t off_bytes = (size_t)(n_structs + 1) * sizeof(int64_t);
    FD2_CHECK_CUDA(cudaMallocAsync(&scratch, 16 + off_bytes, st));
    int* d_bad = (int*)scratch;
    int64_t* d_off = (int64_t*)((char*)scratch + 16);
    int bad = 0;
    cudaError_t e = cudaMemsetAsync(d_bad, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_off, h_struct_offsets, off_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        fd2::dvh_count_kernel<<<dim3((unsigned)per, (unsigned)n_structs), fd2::kDvhThreads, shm, st>>>(
            d_dose, n_voxels, d_off, d_voxels, n_bins, bin_width, d_cumulative, d_bad);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        fd2::dvh_cumulate_kernel<<<(unsigned)n_structs, 32, 0, st>>>(d_cumulative, n_bins);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(scratch, st);
    FD2_CHECK_CUDA(e);
    ctx->launches += 2;
    FD2_REQUIRE(bad == 0, FD2_ERR_INVALID_ARGUMENT, "dvh: %d structure voxel indices outside [0, %lld)", bad,
                (long long)n_voxels);
    return FD2_OK;
}
