/*
 * fd2.h -- C ABI of the B200 (sm_100a) dose-calculation and fluence-optimization
 * library.  Every entry point takes plain pointers, sizes and POD structs; device
 * buffers are owned by the caller unless a handle says otherwise; streams are
 * passed as `void*` (a cudaStream_t, NULL = legacy default stream).
 *
 * Return convention: 0 = success, negative = fd2_status error.  Nothing here
 * calls exit().  The reference library returns bool with 1 = failure and exits
 * the process on CUDA errors (FastDoseLib/include/helper_cuda.h:583-595); the C++
 * compatibility shim (fd2_compat.hpp) maps status != 0 back to `return 1`.
 *
 * Thread safety: a context is used by one host thread at a time.  Handles made
 * from a context must not be shared between contexts.
 */
#ifndef FD2_H
#define FD2_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ------------------------------------------------------------------ status */
typedef enum fd2_status {
    FD2_OK = 0,
    FD2_ERR_INVALID_ARGUMENT = -1,
    FD2_ERR_CUDA = -2,
    FD2_ERR_OUT_OF_MEMORY = -3,
    FD2_ERR_IO = -4,
    FD2_ERR_GEOMETRY = -5,      /* beam misses the bounding box, canonical beamlet fit failed */
    FD2_ERR_CAPACITY = -6,      /* a caller-provided buffer is too small */
    FD2_ERR_WATCHDOG = -7,      /* a bounded device loop hit its iteration cap */
    FD2_ERR_NOT_SUPPORTED = -8,
    FD2_ERR_ADMISSION = -9      /* request does not fit the HBM admission budget */
} fd2_status;

/* Human-readable name of a status code (static storage). */
const char* fd2_status_string(int status);
/* ABI version: major*10000 + minor*100 + patch. */
int fd2_version(void);
/* Last error message recorded on this host thread (static per-thread storage). */
const char* fd2_last_error(void);

/* ------------------------------------------------------------------ beams */
/*
 * Beam / beamlet descriptor.  Byte-for-byte the layout of fastdose::d_BEAM_d
 * (FastDoseLib/include/beam.cuh:84-133: float3 isocenter, float2 beamlet_size,
 * uint2 fmap_size, float sad, float3 angles, float long_spacing, float lim_min,
 * float lim_max, uint long_dim, float3 source, size_t TermaBEV_pitch,
 * size_t DensityBEV_pitch), so an existing device array of d_BEAM_d can be
 * passed unchanged.  96 bytes; the two pad words are the alignment gaps the
 * CUDA vector types leave.
 *   angles = (gantry theta, couch phi, collimator) in radians.
 *   pitches are in bytes; this library requires Terma/Density/Dose pitches equal.
 */
typedef struct fd2_beam {
    float isocenter[3];
    uint32_t pad0;
    float beamlet_size[2];
    uint32_t fmap_size[2];
    float sad;
    float angles[3];
    float long_spacing;
    float lim_min;
    float lim_max;
    uint32_t long_dim;
    float source[3];
    uint32_t pad1;
    uint64_t TermaBEV_pitch;
    uint64_t DensityBEV_pitch;
} fd2_beam_t;

/* Volume geometry: density is float[z][y][x], x fastest (reference density.cuh:12). */
typedef struct fd2_volume {
    uint32_t dim[3];         /* VolumeDim (x, y, z) */
    float voxel_size[3];     /* cm */
    uint32_t bbox_start[3];  /* BBoxStart, voxels */
    uint32_t bbox_dim[3];    /* BBoxDim, voxels */
} fd2_volume_t;

/*
 * BEAM_h::calc_range (FastDoseLib/src/beam.cu:134-222): source position,
 * [lim_min, lim_max] and long_dim of one beam against the volume bounding box.
 * Host-only, single precision with the reference's operation order.
 * Reads isocenter, beamlet_size, fmap_size, sad, angles, long_spacing;
 * writes source, lim_min, lim_max, long_dim.
 */
int fd2_beam_calc_range(fd2_beam_t* beam, const fd2_volume_t* volume);

/* Beam-bundle parameters, the IMRT::BeamBundle fields (IMRTOpt/include/IMRTBeamBundle.cuh:9-31). */
typedef struct fd2_bundle {
    float isocenter[3];
    float beamlet_size[2];
    int32_t fluence_dim[2];
    float sad;
    float angles[3];
    float long_spacing;
    int32_t sub_fluence_dim[2];
    int32_t sub_fluence_on[2];
} fd2_bundle_t;

/*
 * IMRT::BeamBundle::beamletInit (IMRTOpt/src/IMRTBeamBundle.cu:341-569): the
 * canonical sub-beam of fluence pixel (ix, iy) of a bundle, with calc_range
 * applied.  Host-only, single precision.  Fluence of the sub-beam is the centred
 * sub_fluence_on^2 open square of a sub_fluence_dim^2 map (fd2_beamlet_fluence).
 */
int fd2_beamlet_init(const fd2_bundle_t* bundle, int ix, int iy,
                     const fd2_volume_t* volume, fd2_beam_t* out);

/*
 * BeamBundle::beamletsInit (IMRTBeamBundle.cu:319) for many bundles at once:
 * fd2_beamlet_init for every flagged pixel of every bundle (raster order, y
 * outer, x inner), spread over n_threads host threads (<= 0: one per core).
 * h_flags holds each bundle's fy x fx flags, bundle after bundle (bundles may
 * differ in fluence dimension).  out: room for cap beams, filled bundle after
 * bundle; counts[b] = beamlets of bundle b.  Host only; the same beams, bit for
 * bit, as one fd2_beamlet_init call per pixel.
 */
int fd2_bundles_beamlets(size_t n_bundles, const fd2_bundle_t* bundles, const uint8_t* h_flags,
                         const fd2_volume_t* volume, int n_threads, size_t cap, fd2_beam_t* out, uint32_t* counts);

/* Writes the sub-beam fluence map (float[fy][fx]) of a bundle into `out`. */
int fd2_beamlet_fluence(const fd2_bundle_t* bundle, float* out, size_t n);

/* ------------------------------------------------------------------ context */
typedef struct fd2_context fd2_context;
typedef struct fd2_density fd2_density;
typedef struct fd2_spectrum fd2_spectrum;
typedef struct fd2_cccs_kernel fd2_cccs_kernel;
typedef struct fd2_csr_ensemble fd2_csr_ensemble;

/* Creates a context on CUDA device `device` (makes it current on this thread). */
int fd2_context_create(int device, fd2_context** out);
int fd2_context_destroy(fd2_context* ctx);
/* Synchronises the context's internal streams. */
int fd2_context_synchronize(fd2_context* ctx);
/*
 * Returns the context's idle device memory: waits for the device, frees the
 * grow-only BEV, column and cone buffers, and trims the context's pool to the
 * allocations still alive (matrices not yet destroyed keep theirs).  The next
 * call regrows what it needs.  For a process that moves from one workload to
 * another on the same GPU (e.g. from building matrices to serving requests on
 * other contexts).
 */
int fd2_context_release(fd2_context* ctx);

/*
 * Instrumentation, the counterpart of the reference's per-kernel event timers
 * (FastDoseLib/src/TermaComp.cu:311-333, DoseComp.cu:450-472,
 * IMRTOpt/src/IMRTDoseMat.cu:261-274).  With timing on, the plan-level calls
 * bracket each stage with CUDA events and accumulate its device time.
 */
enum fd2_stage {
    FD2_STAGE_TERMA = 0,
    FD2_STAGE_CCCS = 1,
    FD2_STAGE_COLUMNS = 2,
    FD2_STAGE_OPT_SPMV = 3,
    FD2_STAGE_OPT_OTHER = 4,
    FD2_STAGE_COUNT = 5
};
int fd2_context_set_timing(fd2_context* ctx, int on);
/* Copies min(n, FD2_STAGE_COUNT) accumulated stage times (ms) and resets them. */
int fd2_context_stage_times(fd2_context* ctx, double* ms, int n);
/* Number of kernels this library launched through the context so far. */
uint64_t fd2_context_launch_count(const fd2_context* ctx);
/*
 * The context's tuned CCCS schedules (the construction's automatic choice,
 * measured once per batch shape): up to cap (shape key, schedule) pairs and
 * their number in *n; *runs = batches on which both schedules were timed.
 * Key bits: 0-7 log2 of the batch's beamlets, 8-23 map pixels, 24-39 azimuths,
 * 40- zenith bins.
 */
int fd2_context_tuned_schedules(const fd2_context* ctx, size_t cap, uint64_t* keys, int32_t* schedules, size_t* n,
                                uint64_t* runs);
/*
 * Graph-captured construction (fd2_dosemat_params_t.graph) on this context:
 * batches launched as one graph, executable graphs instantiated (one per
 * batch shape, or again when an in-place update is refused), and in-place
 * updates.  The reference has no counterpart (it launches kernel by kernel).
 * Any pointer may be NULL.
 */
int fd2_context_graph_counts(fd2_context* ctx, uint64_t* launches, uint64_t* instantiations, uint64_t* updates);

/*
 * fastdose::density_h2d (FastDoseLib/src/density.cu:23-58).  Copies a host
 * density volume to the device.  Sampling is trilinear on texel centres i+0.5
 * with zero outside the volume (the reference's linear/border texture).  The
 * device copy comes from a memory pool the library keeps per device for the
 * life of the process, and is complete on return; fd2_density_destroy waits
 * for the device (as cudaFree does) and returns it to that pool.  A density
 * may be destroyed after its context.
 */
int fd2_density_create(fd2_context* ctx, const float* host_density,
                       const fd2_volume_t* volume, fd2_density** out);
int fd2_density_destroy(fd2_density* d);
/* Device pointer of the density volume (float[z][y][x]). */
const float* fd2_density_device_ptr(const fd2_density* d);

/*
 * SPECTRUM_h::bind_spectrum (FastDoseLib/src/TermaComp.cu:67-78).  `fluence`
 * is the normalised bin weight as read_spectrum_file leaves it
 * (spectrum.cu:41-42).  n <= 24 (MAX_KERNEL_NUM).  The table lives in the handle,
 * not in process-global constant memory, so several spectra can coexist.
 */
int fd2_spectrum_create(fd2_context* ctx, int n, const float* energy, const float* fluence,
                        const float* mu, const float* mu_en, fd2_spectrum** out);
int fd2_spectrum_destroy(fd2_spectrum* s);

/*
 * KERNEL_h::bind_kernel (FastDoseLib/src/DoseComp.cu:25-38).  theta is the bin
 * middle angle; phi the azimuths.  nTheta, nPhi <= 24.
 */
int fd2_kernel_create(fd2_context* ctx, int n_theta, const float* theta,
                      const float* A, const float* a, const float* B, const float* b,
                      int n_phi, const float* phi, fd2_cccs_kernel** out);
int fd2_kernel_destroy(fd2_cccs_kernel* k);

/* ------------------------------------------------------------------ dose calc */
/*
 * fastdose::TermaComputeCollective (FastDoseLib/src/TermaComp.cu:153-176).
 * d_beams: device array of n_beams descriptors.  d_fluence / d_terma /
 * d_density_bev: device arrays of n_beams device pointers (the reference's
 * float** convention).  Outputs are [long_dim][pitch/4] per beam.
 */
int fd2_terma_compute(fd2_context* ctx, size_t fmap_npixels, size_t n_beams,
                      const fd2_beam_t* d_beams, float* const* d_fluence,
                      float* const* d_terma, float* const* d_density_bev,
                      const fd2_density* density, const fd2_spectrum* spectrum,
                      void* stream);

/*
 * fastdose::DoseComputeCollective (FastDoseLib/src/DoseComp.cu:179-214).
 * Accumulates (+=) into d_dose like the reference; zero it first for a fresh beam.
 */
int fd2_dose_compute(fd2_context* ctx, size_t fmap_npixels, size_t n_beams,
                     const fd2_beam_t* d_beams, float* const* d_terma,
                     float* const* d_density_bev, float* const* d_dose,
                     const fd2_cccs_kernel* kernel, void* stream);

/* Direction-table capacity of fd2_dose_compute_static, in bytes. */
#define FD2_DOSE_STATIC_DIR_BYTES (256u * 1024u)

/*
 * fd2_dose_compute without any device allocation.  No counterpart in the
 * reference: an addition for callers that may not allocate device memory
 * while they run (their device memory is carved from a pool fixed at
 * start-up, or owned by another runtime that forbids foreign allocations).
 * Same arguments and result as fd2_dose_compute, without a context: the
 * status word and the cone-direction table live in one fixed array in device
 * global memory (FD2_DOSE_STATIC_DIR_BYTES + 256 bytes, held by every GPU that
 * loads the library until exit), and nothing is allocated by cudaMalloc or
 * any library.
 *
 * - The array's address belongs to the CUDA context that loaded the
 *   library's device code.  The first call in each context (once per device
 *   under the runtime's primary context) looks it up, which may load that
 *   device code; make that first call during set-up, before any stream
 *   capture.  A second context on a device, or a context recreated after
 *   cudaDeviceReset, gets its own lookup.
 * - Limit: n_beams * n_forward_theta * n_phi * 16 <= FD2_DOSE_STATIC_DIR_BYTES
 *   (256 beams of an 8 x 8 cone kernel); larger batches return
 *   FD2_ERR_CAPACITY before any device work.
 * - Accumulates (+=) into d_dose like fd2_dose_compute: zero it first for a
 *   fresh dose.  The call clears its own status word; nothing else in the
 *   fixed array needs to start at zero.
 * - status_out (NULL, host or device int): receives the kernels' status code
 *   (0, or FD2_ERR_WATCHDOG) in stream order; read it after the stream
 *   synchronises.
 * - All calls on one device share the fixed array: calls whose device work
 *   overlaps (different streams, or unordered host threads) race and corrupt
 *   each other.  Serialise them.
 * The beam descriptors are read back to the host (synchronising the stream)
 * to size the launch.
 */
int fd2_dose_compute_static(size_t fmap_npixels, size_t n_beams, const fd2_beam_t* d_beams,
                            float* const* d_terma, float* const* d_density_bev, float* const* d_dose,
                            const fd2_cccs_kernel* kernel, int* status_out, void* stream);

/*
 * The cone directions the CCCS march uses: for every beam, forward zenith bin
 * (theta <= pi/2) and azimuth, the unit direction in normalised BEV units,
 * evaluated on the device with the reference's single-precision formula
 * (FastDoseLib/src/DoseComp.cu:280-290).  h_out: float[n_beams][n_fwd][n_phi][4]
 * (x, y, z, 0).  Diagnostic / test entry point.
 */
int fd2_cccs_cone_directions(fd2_context* ctx, const fd2_cccs_kernel* kernel, size_t n_beams,
                             const fd2_beam_t* h_beams, float* h_out, size_t n_out);

/*
 * fastdose::BEV2PVCS (FastDoseLib/src/TermaComp.cu:97-150): one beam's BEV array
 * d_bev ([long_dim][fmap_y][fmap_x], contiguous) resampled trilinearly onto the
 * whole volume.  d_out is float[z][y][pitch/4].
 */
int fd2_bev2pvcs(fd2_context* ctx, const fd2_beam_t* h_beam, const fd2_density* density,
                 const float* d_bev, float* d_out, size_t out_pitch_bytes, void* stream);

/*
 * fastdose::BEV2PVCS_SuperSampling (FastDoseLib/src/geom.cu:343-474).  Voxels
 * farther than `extent` from the beam axis, or whose supersampled sum is below
 * 1e-4, are left untouched, as in the reference.
 */
int fd2_bev2pvcs_supersampling(fd2_context* ctx, const fd2_beam_t* h_beam,
                               const fd2_density* density, const float* d_bev,
                               float* d_out, size_t out_pitch_bytes, int ssfactor,
                               float extent, void* stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* FD2_H */
