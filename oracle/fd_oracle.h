/*
 * fd_oracle.h -- CPU restatement of the reference dose-calculation and
 * fluence-optimization path.  TEST INFRASTRUCTURE ONLY: the parity checker for
 * the CUDA kernels of fastdose_b200 and the timed CPU baseline.  Nothing in the
 * product links, loads or calls this code.
 *
 * Two builds come from the same source (oracle/Makefile):
 *   liboracle64.so  FD_REAL=double, single thread  -- the parity oracle;
 *   liboracle32.so  FD_REAL=float                  -- the timed CPU baseline
 *                   (callers run beamlets on parallel host threads).
 * Geometry on the host (calc_range, beamletInit) and the cone-march ray
 * stepping are single precision in both builds: the reference computes them in
 * float, and the boundary decisions of the march must be reproduced bit for bit.
 *
 * Every function cites the reference file:line it restates.
 */
#ifndef FD_ORACLE_H
#define FD_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#include "../include/fd2.h"

#ifdef __cplusplus
extern "C" {
#endif

/* geometry (float, reference host semantics) */
void or_rotate_axis_f(const float p[3], const float r[3], float t, float out[3]);
void or_rotate_beam_f(const float v[3], float theta, float phi, float coll, float out[3]);
void or_inv_rotate_beam_f(const float v[3], float theta, float phi, float coll, float out[3]);
int or_calc_range(fd2_beam_t* beam, const fd2_volume_t* vol);
int or_beamlet_init(const fd2_bundle_t* bundle, int ix, int iy, const fd2_volume_t* vol,
                    fd2_beam_t* out);
void or_beamlet_fluence(const fd2_bundle_t* bundle, float* out);
/* device-style line segment / coordinate helpers (double), DoseComp.cu:114-164 */
double or_calc_line_seg(const double s[3], const double e[3], const fd2_beam_t* beam);
void or_next_point(const double c[3], const double d[3], double out[3], int* flag);
void or_next_point_f(const float c[3], const float d[3], float out[3], int* flag);
/* normalised-BEV cone direction, DoseComp.cu:280-290 (double, rounded to float) */
void or_cone_direction(const fd2_beam_t* beam, float theta, float phi, float out[3]);

/* Beamlet on/off flags by PTV mask sampling, IMRTBeamBundle.cu:269-316.
 * tex_mode: 0 = exact trilinear weights, 1 = weights rounded to 1/256. */
void or_beamlet_flags(size_t n_beams, const fd2_beam_t* beams, const uint8_t* ptv_mask,
                      const fd2_volume_t* vol, int super_sampling, int tex_mode,
                      uint8_t* flags_out);

/* Terma ray trace of one beam, TermaComp.cu:179-253.  terma/dens are [L][P]. */
void or_terma(const fd2_beam_t* beam, const float* fluence, const float* density,
              const fd2_volume_t* vol, int nkern, const float* energy, const float* spec_fluence,
              const float* mu, int tex_mode, float* terma_out, float* dens_out);

/* CCCS of one beam in BEV, DoseComp.cu:217-392 (quirks Q1-Q4).  dose is
 * accumulated (+=) into dose_io, [L][P]. */
void or_cccs(const fd2_beam_t* beam, const float* terma, const float* dens, int n_theta,
             const float* theta, const float* A, const float* a, const float* B, const float* b,
             int n_phi, const float* phi, float* dose_io);
/* As or_cccs, marching with the given cone directions
 * ([forward zenith bin][azimuth][4], e.g. the library's device-evaluated table)
 * instead of the double-precision ones; NULL selects the latter. */
void or_cccs_dirs(const fd2_beam_t* beam, const float* terma, const float* dens, int n_theta,
                  const float* theta, const float* A, const float* a, const float* B, const float* b,
                  int n_phi, const float* phi, const float* dirs, float* dose_io);

/* Dense BEV->PVCS linear resampling, TermaComp.cu:124-150.  out is [z][y][x]. */
void or_bev2pvcs(const fd2_beam_t* beam, const float* bev, const fd2_volume_t* vol,
                 int tex_mode, float* out);

/* BEV->PVCS with supersampling, geom.cu:412-474.  Untouched voxels keep out's value. */
void or_bev2pvcs_ss(const fd2_beam_t* beam, const float* bev, const fd2_volume_t* vol,
                    int ssfactor, float extent, int tex_mode, float* out);

/* Beamlet column by 5^3 point sampling, IMRTgeom.cu:370-468 (voxel stage; the
 * supervoxel stage only skips work).  Writes the dense row (nVoxels floats). */
void or_beamlet_column(const fd2_beam_t* beam, const float* dose_bev, const fd2_volume_t* vol,
                       int ssfactor, float extent, float* row_out);

/* Whole single-beamlet pipeline into a dense row: Terma, CCCS, column. */
void or_beamlet_pipeline(const fd2_beam_t* beam, const float* fluence, const float* density,
                         const fd2_volume_t* vol, int nkern, const float* energy,
                         const float* spec_fluence, const float* mu, int n_theta,
                         const float* theta, const float* A, const float* a, const float* B,
                         const float* b, int n_phi, const float* phi, int ssfactor, float extent,
                         float* row_out);

/* ---- optimizer (IMRTOptUtils.cu, IMRTOptimize_var1.cu, IMRTOptimize.cu) ---- */
typedef struct or_csr {
    int64_t rows, cols, nnz;
    const int64_t* offsets;
    const int64_t* columns;
    const float* values;
} or_csr;

typedef struct or_problem {
    or_csr A, AT, D, DT;
    int64_t n_ptv, n_oar;
    const float* max_dose;       /* [n_ptv + n_oar] */
    const float* max_weights;    /* [n_ptv + n_oar] */
    const float* min_dose;       /* [n_ptv] */
    const float* min_weights;    /* [n_ptv] */
    const float* oar_weights;    /* [n_oar] */
    float gamma, eta;
} or_problem;

/* eval_g::evaluate, IMRTOptUtils.cu:74-156 (double accumulation) */
double or_eval_g(const or_problem* p, const float* x);
/* eval_grad::evaluate, IMRTOptUtils.cu:512-631 */
double or_eval_grad(const or_problem* p, const float* x, float* grad);
/* proxL2Onehalf_QL_gpu::evaluate + d_proxL2Onehalf_calc_tHat,
 * IMRTOptimize_var1.cu:502-570.  Groups are consecutive segments of x. */
void or_prox_l2onehalf(int64_t n_groups, const int64_t* group_offsets, const float* g0,
                       const float* tau, float* prox, float* nrmnew);
/* d_proxL2Onehalf_calc_tHat for one group, IMRTOptimize_var1.cu:544-570 */
double or_that(double nrm2, double tau);

/* Loop state shared by the two solvers (IMRTOptimize.cu:16-194, 391-476). */
typedef struct or_opt_state {
    int k_global;
    float theta_km1, tkm1;
    float* xkm1;        /* [n] in/out */
    float* vkm1;        /* [n] in/out */
    float* loss;        /* [iters_global] out */
    float* nrm;         /* [n_groups] out (BOO only) */
    float num_active;   /* out (BOO only) */
    int stop;           /* out (BOO only) */
    int trials;         /* out: total line-search trials */
} or_opt_state;

/* BOO_IMRT_L2OneHalf_gpu_QL, IMRTOptimize.cu:16-194 */
int or_boo_l2onehalf(const or_problem* p, int64_t n_groups, const int64_t* group_offsets,
                     float* beam_weights, int show_trigger, int change_weights_trigger,
                     int iters_global, const int* prune_trigger, int n_prune,
                     int num_beams_we_want, or_opt_state* st);
/* polish_BOO_IMRT_gpu, IMRTOptimize.cu:391-476 */
int or_polish(const or_problem* p, int iters_global, int iters_local, or_opt_state* st);

/* beamWeightsInit_func (Eigen version), IMRTOptimize_var1.cu:125-161.
 * A_beams[b] is the VOI x beamlets block of beam b (CSR). */
void or_beam_weights_init(int64_t n_beams, const or_csr* A_beams, int64_t n_ptv, float* out);

/* fluenceGradInit per beam, IMRTOptimize_var.cpp:59-180 with DxyInit/
 * KroneckerProduct (IMRTEigenLoad.cpp:307-407).  Writes the CSR of D_b into
 * caller buffers sized 2*n*n rows / 4*n*n nnz; returns rows, nnz via pointers. */
void or_fluence_grad(int fluence_dim, const uint8_t* active, int64_t* rows, int64_t* nnz,
                     int64_t* offsets, int64_t* columns, float* values);

#ifdef __cplusplus
}
#endif
#endif
