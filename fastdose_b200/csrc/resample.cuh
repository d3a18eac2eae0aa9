// resample.cuh -- per-beamlet resampling descriptors and launchers (internal).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "fd2_internal.cuh"

namespace fd2 {

// Everything the PVCS<->BEV mapping of one beamlet needs, precomputed on the host.
struct ColumnInfo {
    float R[9];        // PVCS -> BEV rotation (rotateBeamAtOriginRHS as a matrix, row-major)
    float src[3];      // source position (cm)
    float bsx, bsy;    // beamlet_size at the SAD plane
    float hx, hy;      // fmap_size / 2
    float inv_sad, lim_min, ls, inv_ls;
    int fx, fy, L;
    int box[6];        // voxel box [x0, y0, z0, x1, y1, z1) that can hold nonzeros
};

// Fills ci from a beam (rotation in double, rounded to float) and, when vol is
// given, the conservative voxel box of the beamlet's frustum.
void make_column_info(const fd2_beam_t& b, const fd2_volume_t* vol, ColumnInfo& ci);

int launch_bev2pvcs(const ColumnInfo& ci, const fd2_volume_t& v, const float* d_bev, float* d_out, size_t pitch,
                    int ss, float extent, cudaStream_t stream);
int launch_column_count(const ColumnInfo* d_infos, size_t n, uint32_t* d_counts, const fd2_volume_t& v, float extent,
                        cudaStream_t stream);
int launch_column_values(const ColumnInfo* d_infos, size_t n, const float* const* d_dose, const uint64_t* d_cap_off,
                         int32_t* d_tmp_col, float* d_tmp_val, uint32_t* d_row_nnz, float* d_row_max,
                         const fd2_volume_t& v, float extent, int ss, cudaStream_t stream);
int launch_column_rows(size_t n, const uint32_t* d_nnz, const float* d_max, int64_t* d_row_off, float* d_scale,
                       float* d_inv_scale, cudaStream_t stream);
int launch_column_gather(size_t n, const uint64_t* d_cap_off, const int64_t* d_row_off, const int32_t* d_tmp_col,
                         const float* d_tmp_val, const float* d_inv_scale, int32_t* d_col, void* d_val,
                         int value_type, cudaStream_t stream);

int launch_cccs_host(fd2_context* ctx, size_t n_beams, const fd2_beam_t* h_beams, const fd2_beam_t* d_beams,
                     const float* const* d_terma, const float* const* d_dens, float* const* d_dose,
                     const fd2_cccs_kernel* k, int schedule, cudaStream_t stream,
                     const int* d_order = nullptr);
// The march order of a batch: beamlet indices by decreasing depth (slices to
// march), ties in batch order, so a launch's last blocks are its short ones.
void cccs_longest_first(size_t n_beams, const fd2_beam_t* h_beams, int* order);
int cccs_auto_schedule(const fd2_context* ctx, size_t n_beams);

}  // namespace fd2
