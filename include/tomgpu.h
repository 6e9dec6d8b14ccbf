/* tomgpu — B200-native (sm_100a) template matching for TOM.
 *
 * C ABI of libtomgpu.so.  Every entry point returns a tomgpu_status; nothing
 * longjmps or throws across this boundary.  Pointers ending in _dev are
 * device pointers owned by the caller; all other array pointers are host
 * pointers owned by the caller.  Volumes are single precision, x fastest
 * (MATLAB column-major order): element (x, y, z) sits at x + nx*(y + ny*z).
 *
 * Each entry point names the reference interface it replaces.  Reference
 * paths are relative to the TOM toolbox source tree.
 */
#ifndef TOMGPU_H
#define TOMGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    TOMGPU_OK = 0,
    TOMGPU_ERR_ARG = 1,         /* invalid argument: null pointer, size, mode */
    TOMGPU_ERR_UNSUPPORTED = 2, /* size beyond the FFT line limits or another fixed limit */
    TOMGPU_ERR_OOM = 3,         /* device allocation failed */
    TOMGPU_ERR_CUDA = 4,        /* CUDA runtime error (details: tomgpu_last_error) */
    TOMGPU_ERR_STATE = 5,       /* call order: e.g. run before a volume is set */
    TOMGPU_ERR_DEVICE = 6,      /* a kernel reported an internal error flag */
    TOMGPU_ERR_TIMEOUT = 7      /* a bounded device wait ran out */
} tomgpu_status;

typedef struct tomgpu_ctx tomgpu_ctx;
typedef struct tomgpu_match_plan tomgpu_match_plan;

/* ------------------------------------------------------------ context --- */
/* Library version string, e.g. "tomgpu 0.1 sm_100a". */
const char* tomgpu_version(void);
/* Human-readable name of a status code. */
const char* tomgpu_status_string(int status);
/* Message of the last failing call on this context (or of the last
 * tomgpu_ctx_create failure when ctx is NULL). */
const char* tomgpu_last_error(const tomgpu_ctx* ctx);

/* Create a context on a CUDA device.  The context owns a stream (replaceable
 * with tomgpu_ctx_set_stream) and its workspaces.  One context per host
 * thread; calls on one context are not thread-safe. */
int tomgpu_ctx_create(int device, tomgpu_ctx** out);
int tomgpu_ctx_destroy(tomgpu_ctx* ctx);
/* Issue all further work of this context on an existing cudaStream_t (passed
 * as void*); NULL selects the CUDA legacy default stream.  Work already
 * queued on the previous stream completes before the new stream's next work
 * (an event wait on the device; the call does not block the host). */
int tomgpu_ctx_set_stream(tomgpu_ctx* ctx, void* cuda_stream);
int tomgpu_ctx_synchronize(tomgpu_ctx* ctx);
/* Release the device memory that tomgpu_match and tomgpu_av3_align keep in
 * the context between calls (no counterpart in the reference: TOM plans
 * nothing across calls). */
int tomgpu_ctx_trim(tomgpu_ctx* ctx);
/* Device kernel launches issued by this context since creation. */
int64_t tomgpu_ctx_launch_count(const tomgpu_ctx* ctx);

/* Device time per kernel class of the matching loop, measured with CUDA
 * events recorded on the context stream around each launch while profiling
 * is enabled (no host synchronisation until the read). */
enum {
    TOMGPU_K_ROTATE = 0,   /* rotation * mask of the template batch */
    TOMGPU_K_FILTER = 1,   /* weight (psf) filter of the rotated templates */
    TOMGPU_K_SPEC_X = 2,   /* x-stage of the template spectrum */
    TOMGPU_K_SPEC_Z = 3,   /* z-stage of the template spectrum */
    TOMGPU_K_CORR_Y = 4,   /* y-DFT, product with the tomogram spectrum, inverse y-DFT */
    TOMGPU_K_INV_Z = 5,    /* inverse z-DFT */
    TOMGPU_K_C2R_FLCF = 6, /* inverse x (complex-to-real), FLCF, running max/arg-max */
    TOMGPU_K_COUNT = 7
};
/* enable != 0 starts (and resets) the timers, 0 stops recording. */
int tomgpu_ctx_profile(tomgpu_ctx* ctx, int enable);
/* Total milliseconds and launch count of one kernel class; synchronises the stream. */
int tomgpu_ctx_profile_read(tomgpu_ctx* ctx, int kernel, double* total_ms, int64_t* launches);

/* ----------------------------------------------------------- rotation --- */
enum { TOMGPU_EULER_DEG = 1, TOMGPU_MATRIX = 3 };

/* Replaces the tom_rotatec MEX: tom_rotatec(in, out, euler, 'linear', center)
 * (Sptrans/tom_rotatec.c:407-480, compute in rot3d :146-401; called from
 * Sptrans/tom_rotate.m:126).  mode TOMGPU_EULER_DEG: euler = [phi psi theta]
 * in degrees, ZXZ; TOMGPU_MATRIX: 9 floats in MATLAB column-major order of the
 * 3x3 matrix.  center is 0-based (tom_rotate passes ceil(size/2)).  Output
 * voxel x samples in at center + R^T (x - center), trilinear, 0 outside.
 * Bit-exact with rot3d.  Host buffers. */
int tomgpu_rotate3d(tomgpu_ctx* ctx, const float* in, float* out, const int dims[3],
                    const float* euler_or_matrix, int mode, const float center[3]);

/* Batched rot3d on device buffers: R rotations (eulers R x 3 degrees, host
 * array) of one volume into out_dev (R volumes back to back); optional
 * mask_dev multiplies every output voxel (tom_os3_findTemplate.m:264). */
int tomgpu_rotate3d_batch_dev(tomgpu_ctx* ctx, const float* in_dev, float* out_dev,
                              const int dims[3], const float* eulers, int R,
                              const float center[3], const float* mask_dev);

/* ZXZ rotation matrix of tom_rotatec for one Euler triplet (degrees), 9 floats
 * rm00, rm10, rm20, rm01, rm11, rm21, rm02, rm12, rm22 (Sptrans/tom_rotatec.c:164-288). */
int tomgpu_euler_matrix(const float euler[3], float m9[9]);

/* -------------------------------------------------------------- peaks --- */
/* Replaces the tom_peakinc MEX (Analysis/tom_peakinc.c:23-77, via
 * Analysis/tom_peakc.m:70): first strict maximum in x-fastest order starting
 * from -99999; pos1 is 1-based.  Host buffer. */
int tomgpu_peak(tomgpu_ctx* ctx, const float* v, const int dims[3], float* val, int pos1[3]);
int tomgpu_peak_dev(tomgpu_ctx* ctx, const float* v_dev, const int dims[3], float* val, int pos1[3]);

/* K peaks by repeated [c val M] = tom_peak(A, R) (Analysis/tom_peak.m:203-279):
 * each round takes the first maximum and zeroes the ball of radius R around
 * it.  The search zeroes balls in an internal scratch copy; v_dev is not modified.
 * vals: K floats, pos1: K x 3 ints (1-based). */
int tomgpu_topk_dev(tomgpu_ctx* ctx, const float* v_dev, const int dims[3], int K, double radius,
                    float* vals, int* pos1);

/* One round of [c val M] = tom_peak(A, R) in place: the first maximum of
 * v_dev, then the ball of radius R around it set to 0 (v_dev becomes M). */
int tomgpu_peak_radius_dev(tomgpu_ctx* ctx, float* v_dev, const int dims[3], double radius, float* val,
                           int pos1[3]);

/* Allocation-free variant of tomgpu_topk_dev, for callers that must not
 * allocate device memory at the time they search peaks (under a host
 * framework that owns the device memory, such as a MEX next to gpuArray data,
 * or in loops that may not risk an allocation failure).  No context: work is
 * issued on `stream` (NULL = legacy default stream); v_dev is the volume,
 * vals_dev (K floats) and pos1_dev (K x 3 ints, 1-based) are device outputs.
 * The scratch lives in file-scope device arrays: at most 16,777,216 voxels
 * (64 MiB, held on every GPU where the library's code is loaded until exit);
 * larger volumes return TOMGPU_ERR_UNSUPPORTED.  The first call on a device
 * sets the scratch up (looks up its device address) and should come before
 * any stream capture on that device; the address is kept for the life of the
 * process, so do not call this entry point again after cudaDeviceReset.
 * Calls share the scratch: calls that overlap on the GPU race.  Errors:
 * tomgpu_last_error(NULL).  This entry point has no counterpart in the
 * reference. */
int tomgpu_topk_noalloc_dev(void* stream, const float* v_dev, const int dims[3], int K, double radius,
                            float* vals_dev, int* pos1_dev);

/* tom_peak(A, 'spline') sub-voxel refinement at a given 1-based integer peak
 * (tom_intpeak, Analysis/tom_peak.m:437-525): per axis the parabola through
 * the 3 neighbours maximised on a 0.001 grid.  coord: 3 doubles, val: max. */
int tomgpu_peak_spline_dev(tomgpu_ctx* ctx, const float* v_dev, const int dims[3],
                           const int pos1[3], double coord[3], double* val);

/* ------------------------------------------------------ weights, masks --- */
/* Replaces tom_calc_weight_functioninc (Filtrans/tom_calc_weight_functioninc.c:152-289):
 * Radermacher exact weighting, angles 2 x n_tilt (phi, theta pairs, degrees),
 * output dims[0]*dims[1]*dims[2] floats (host). */
int tomgpu_weight3d(tomgpu_ctx* ctx, const int dims[3], const double* angles, int n_tilt,
                    double thickness, float* out);

/* Binary missing wedge on a centred grid (Filtrans/tom_wedge.m:62-77): 0 where
 * tan(angle) > |x|/|z|.  av3 form (av3/utils/av3_wedge.m:23-26) when
 * av3 != 0: 0 where tan(pi/2-max) > x/z and tan(-pi/2-min) < x/z.
 * Output on the device (dims product floats). */
int tomgpu_wedge_dev(tomgpu_ctx* ctx, const int dims[3], double angle_or_min, double max_angle,
                     int av3, float* out_dev);

/* ------------------------------------------------------- EM-format I/O --- */
/* Read an EM file (IOfun/tom_emread.m:153-176) into host memory as float
 * (byte, int16, int32, float and double data; either byte order).  With
 * out == NULL only dims is filled (size query); capacity is out's length in
 * floats.  Errors: tomgpu_last_error(NULL). */
int tomgpu_em_read(const char* path, int dims[3], float* out, size_t capacity);
/* Write a float volume as an EM file in PC byte order (magic 6 0 0 5,
 * IOfun/tom_emwrite.m:94-150); comment (may be NULL) fills the 80-char field. */
int tomgpu_em_write(const char* path, const float* data, const int dims[3], const char* comment);

/* out = real(ifftn(ifftshift(fftshift(fftn(in)) .* w))) in FP64 on the device
 * (Filtrans/tom_apply_weight_function.m:56-62); w is the centred weight. */
int tomgpu_apply_weight_dev(tomgpu_ctx* ctx, const float* in_dev, const float* w_dev, const int dims[3],
                            float* out_dev);

/* ------------------------------------------------------------- FFTs --- */
/* Replaces fftn / tom_fourier and ifftn / tom_ifourier (Filtrans/tom_fourier.m:44-50,
 * Filtrans/tom_ifourier.m:36-44) on device buffers.  Complex data are
 * interleaved (re, im) pairs, x fastest.  dir -1: forward, +1: inverse scaled
 * by 1/numel.  precision 32 or 64 (the buffer holds float or double pairs). */
int tomgpu_fft3d_c2c_dev(tomgpu_ctx* ctx, void* data_dev, const int dims[3], int dir, int precision);
/* Real-to-half-complex forward (nx/2+1 complex along x) and its inverse
 * (scaled by 1/numel); out-of-place for r2c, in-place spectrum for c2r. */
int tomgpu_fft3d_r2c_dev(tomgpu_ctx* ctx, const void* real_dev, void* half_dev, const int dims[3],
                         int precision);
int tomgpu_fft3d_c2r_dev(tomgpu_ctx* ctx, void* half_dev, void* real_dev, const int dims[3],
                         int precision);

/* ---------------------------------------------------- FLCF matching --- */
typedef struct {
    int batch;          /* rotations per batch; 0 = the largest of 64, 32, 16 whose
                           per-batch buffers fit in half the free device memory, else 8 */
    int wedge_fp64;     /* reserved, 0 */
    int path;           /* 0: fastest kernels for the sizes; 1: generic kernels only (they
                           compare the CC of every rotation, so of two rotations whose CC
                           rounds to the same float the first one is kept whatever the
                           batch: tom_os3_bestPeak's rule; the fast x-line kernels of path 0
                           compare out / (N M) + kappa within a batch, where such a tie can
                           go to the later rotation);
                           2: as 0, but the x-line kernels of the 512 / 928 x edges load their
                           tiles with per-thread cp.async instead of TMA and the y-column
                           kernel of the 512 y edge reads its constants from shared memory
                           instead of tensor memory (for comparison);
                           3: as 0, with the inverse z-DFT of the 256 z edge as tcgen05
                           tensor-core contractions (split TF32, FP32 accumulation) */
    int reserved[5];
} tomgpu_match_params;

/* A matching plan for one volume size and one template size.  It holds the
 * tomogram spectrum, the FP64 local statistics and per-batch workspaces.
 * Any volume and template edges (odd ones included) within the FFT line
 * limits: every edge up to 3528 voxels, and edges whose prime factors are all
 * in {2,3,5,7,11,13} up to 7150; the template no larger than the volume on any
 * axis.  Edges 128, 256, 464, 512, 928 (and others of the compiled list) run
 * dedicated kernels, every other edge the run-time line engine.  Outside
 * these limits: TOMGPU_ERR_UNSUPPORTED.  params may be NULL. */
int tomgpu_match_plan_create(tomgpu_ctx* ctx, const int vol_dims[3], const int tmpl_dims[3],
                             const tomgpu_match_params* params, tomgpu_match_plan** out);
int tomgpu_match_plan_destroy(tomgpu_match_plan* plan);
/* Bytes of device memory the plan holds. */
int64_t tomgpu_match_plan_bytes(const tomgpu_match_plan* plan);

/* Once per tomogram and template (tom_os3_findTemplate.m:243-245;
 * statistics/tom_os3_mean.m:49-62, statistics/tom_os3_std.m:48-67): the
 * tomogram spectrum and the local mean and standard deviation under the mask,
 * accumulated in FP64, and the FLCF denominators with the template's std.
 * The template and mask must be set first (tomgpu_match_set_template_dev or
 * _raw_dev).  A later template with the same mask keeps the volume (its
 * denominators follow the new template); one with another mask unsets it,
 * and runs return TOMGPU_ERR_STATE until the volume is set again. */
int tomgpu_match_set_volume_dev(tomgpu_match_plan* plan, const float* vol_dev);

/* Template, mask and optional weight (psf) volume, template-sized, device
 * buffers.  Applies findTemplate's preprocessing: tom_norm(1e5*(t+1),
 * 'mean0+1std') (tom_os3_findTemplate.m:157) and the unrotated, filtered
 * template statistics (tom_os3_normUnderMask on tom_os3_modifyImage,
 * :233-234).  psf_dev is the centred weight of tom_apply_weight_function
 * (NULL: no filter).  Must precede tomgpu_match_set_volume_dev; a volume set
 * before it stays set when the mask is the same and is unset otherwise. */
int tomgpu_match_set_template_dev(tomgpu_match_plan* plan, const float* tmpl_dev,
                                  const float* mask_dev, const float* psf_dev);

/* Template and mask taken as given, for tom_os3_corr(img, t) called without
 * cached statistics (search/tom_os3_corr.m:77-149 with calculationAvailable
 * false): the template statistics are tom_os3_normUnderMask(t, mask) of this
 * template, with no tom_norm and no filter.  Then tomgpu_match_corr_dev with
 * the same template gives tom_os3_corr's map. */
int tomgpu_match_set_template_raw_dev(tomgpu_match_plan* plan, const float* tmpl_dev,
                                      const float* mask_dev);

/* Rotation-batch autotuner: times R rotations of `eulers` (host, R x 3
 * degrees) for each of the n_cand candidate batch sizes (a candidate whose
 * work buffers do not fit is skipped), keeps the fastest per rotation for
 * the plan and returns it in *best (0 if none fitted: the plan keeps its
 * batch).  ms_per_rot (n_cand floats, or NULL) receives the measured times.
 * Uses scratch result buffers; needs the template and volume set. */
int tomgpu_match_autotune(tomgpu_match_plan* plan, const float* eulers, int R, const int* cands, int n_cand,
                          int* best, float* ms_per_rot);

/* Fill maxcc_dev with -1000 and angidx_dev with -1 (findTemplate's initial
 * ccc/angles, :215-218, with 0-based indices). */
int tomgpu_match_init_results_dev(tomgpu_match_plan* plan, float* maxcc_dev, int32_t* angidx_dev);

/* The hot loop (tom_os3_findTemplate.m:255-307): for each of R Euler triplets
 * (host array R x 3, degrees), rotate the template (rot3d), multiply the mask,
 * apply the weight (tom_os3_modifyImage), correlate with the tomogram
 * (tom_os3_corr FLCF, search/tom_os3_corr.m:151-176) and update the running
 * maximum where it strictly increases (tom_os3_bestPeak ccc mode,
 * search/tom_os3_bestPeak.m:42-47,94-96).  angidx receives index_offset + r
 * (0-based).  Results are device buffers of volume size. */
int tomgpu_match_run_dev(tomgpu_match_plan* plan, const float* eulers, int R, int index_offset,
                         float* maxcc_dev, int32_t* angidx_dev);

/* Single-rotation FLCF map (tom_os3_corr on an already rotated, masked and
 * filtered template, search/tom_os3_corr.m:151-176): the template statistics
 * are the plan's (set by tomgpu_match_set_template_dev).  t_dev: template-sized,
 * cc_dev: volume-sized. */
int tomgpu_match_corr_dev(tomgpu_match_plan* plan, const float* t_dev, float* cc_dev);

/* Local statistics computed by set_volume (volume-sized outputs, may be NULL). */
int tomgpu_match_stats_dev(tomgpu_match_plan* plan, float* mean_dev, float* std_dev);

/* FP64 rescoring of K candidate peaks (e.g. the top-K of a search): the FLCF
 * of the template at Euler eulers[k] (host, K x 3 degrees) centred on voxel
 * pos1[k] (host, K x 3, 1-based), evaluated by direct summation in double
 * precision over the template box — the correlation sum and the local mean and
 * variance under the mask of search/tom_os3_corr.m:151-176 at that voxel, with
 * no FFT.  vol_dev: the tomogram (device, volume-sized); cc: K doubles (host).
 * Uses the plan's template, mask and weight. */
int tomgpu_match_rescore_fp64_dev(tomgpu_match_plan* plan, const float* vol_dev, const float* eulers,
                                  const int* pos1, int K, double* cc);

/* One-shot, host buffers (what a MEX gateway calls): plan, upload, set
 * template and volume, run all R angles, download.  maxcc/angidx: volume-sized
 * host arrays; angidx is 0-based (-1 where never updated).  The plan and the
 * device copies of the arguments stay in the context for the next call with
 * the same sizes, psf presence and params (a search split over several calls,
 * or one template after another), so such a call allocates nothing;
 * tomgpu_ctx_trim releases them. */
int tomgpu_match(tomgpu_ctx* ctx, const float* tomo, const int vol_dims[3], const float* tmpl,
                 const int tmpl_dims[3], const float* mask, const float* psf, const float* eulers,
                 int R, const tomgpu_match_params* params, float* maxcc, int32_t* angidx);

/* ccf = tom_corr(a, b [, 'norm', mask [, psf1, psf2]]) (Analysis/tom_corr.m:51-121)
 * on device buffers of size dims: mask == NULL gives the plain form
 * real(fftshift(ifftn(F(b) conj F(a))))/numel; with a mask, a and b are first
 * normalised inside it (norm_inside_mask: mean over the mask, std with n - 1)
 * and the result is divided by the mask size; with psfs, a is convolved with
 * psf2 and b with psf1 before normalising (cross-wedging). */
int tomgpu_corr_dev(tomgpu_ctx* ctx, const float* a_dev, const float* b_dev, const int dims[3],
                    const float* mask_dev, const float* psf1_dev, const float* psf2_dev, float* ccf_dev);

/* ------------------------------------------------- subtomogram alignment --- */
/* One alignment job of tom_av3_align (av3_new/tom_av3_align.m:1-189) with
 * filter.Apply = 0.  All volumes are device buffers of size n (x fastest).
 * wedge_ref == NULL: the 5-7 argument form without wedges; wedge_part == NULL
 * with wedge_ref set: the 8 argument form (wedge_part = wedge_ref).  mask is
 * required (pass tom_spheremask(ones) for the reference's default);
 * mask_ccf == NULL means ones.  Angle ranges are [start increment end] in
 * degrees, scanned phi outer, psi, theta inner; indices follow
 * tom_av3_angle2index (phi fastest). */
typedef struct {
    int n[3];
    const float* ref;
    const float* part;
    const float* mask;
    const float* mask_ccf;
    const float* wedge_ref;
    const float* wedge_part;
    float phi[3];
    float psi[3];
    float theta[3];
} tomgpu_align_job;

/* Run n_jobs alignment jobs (any mix of box sizes); per job the outputs of
 * [angles, shifts, ccf_peak] = tom_av3_align(...): angles (3 floats, degrees),
 * shifts (3 floats, spline sub-voxel peak minus floor(n/2)+1), ccf_peak
 * (1 float).  Host output arrays of n_jobs*3, n_jobs*3 and n_jobs floats. */
int tomgpu_av3_align_dev(tomgpu_ctx* ctx, const tomgpu_align_job* jobs, int n_jobs, float* angles,
                         float* shifts, float* ccf_peak);

/* Engine choice for tomgpu_av3_align_ex_dev (NULL params: the defaults). */
typedef struct {
    int path;           /* 0 (default): the jobs with a cubic box of edge 24, 32, 40, 48, 56, 64, 72,
                           80, 96, 100, 112, 120 or 128 run batched, one stream of (particle, rotation) entries per edge
                           and wedge form, the others one job at a time; 1: every job one at a
                           time; 2: as 0 but the scan's last inverse DFT always over the whole
                           box (0 evaluates it only where mask_ccf is non-zero, when every job
                           of the edge has a mask_ccf with a small support) */
    size_t batch_bytes; /* batched engine: device bytes of a batch's two half-spectrum sets
                           (0: 1 GB) */
} tomgpu_align_params;

/* tomgpu_av3_align_dev with an engine choice; the same outputs. */
int tomgpu_av3_align_ex_dev(tomgpu_ctx* ctx, const tomgpu_align_job* jobs, int n_jobs,
                            const tomgpu_align_params* params, float* angles, float* shifts,
                            float* ccf_peak);

/* tomgpu_av3_align_ex_dev on host volumes (what a MEX gateway of
 * tom_av3_align calls): the job's volume pointers are host arrays of its box
 * size (x fastest).  Each distinct array is uploaded once, so jobs that share
 * a reference, mask or wedge by pointer share one device copy; a pointer
 * shared by jobs of different box sizes is an error.  params may be NULL. */
int tomgpu_av3_align(tomgpu_ctx* ctx, const tomgpu_align_job* jobs, int n_jobs,
                     const tomgpu_align_params* params, float* angles, float* shifts, float* ccf_peak);

/* One aligned particle for the averaging step of av3_tomomatch. */
typedef struct {
    const float* particle;  /* box n, device (after av3_tomomatch's tom_limit(p, -3, 4, 'z')) */
    const float* wedge;     /* centred wedge weight of its tomogram (av3_wedge), box n, device */
    float shift[3];         /* tshift, motl rows 11-13 (voxels) */
    float angles[3];        /* phi, psi, theta, motl rows 17-19 (degrees) */
} tomgpu_avg_item;

/* The averaging step after alignment (av3/alignment/av3_tomomatch.m:239-249):
 * for each item in order, average += tom_rotate(tom_shift(particle, -shift),
 * [-psi -phi -theta]) and wei += 1 where tom_rotate(wedge, [-psi -phi
 * -theta]) >= 0.5 (the nested tom_limit).  average_dev and wei_dev are device
 * doubles of box size that accumulate across calls (zero them first). */
int tomgpu_av3_average_add_dev(tomgpu_ctx* ctx, const int n[3], const tomgpu_avg_item* items, int K,
                               double* average_dev, double* wei_dev);

/* The weighting that ends an iteration (av3_tomomatch.m:263-265): w = 1./wei
 * with values above 1e5 set to 0, then real(ifftn(ifftshift(
 * tom_spheremask(fftshift(fftn(average)).*w, floor(n(1)/2)-3)))).  FP64. */
int tomgpu_av3_average_final_dev(tomgpu_ctx* ctx, const int n[3], const double* average_dev,
                                 const double* wei_dev, double* out_dev);

/* Wedge of one volume for tomgpu_corr3d_peaks_dev (the WEDGE_REF / WEDGE_PART
 * forms of tom_mex_corr3d): none ([]), a simple wedge of half-angle
 * angle_deg (a scalar: tom::SimpleWedge with the cutoff radius
 * (min(size)-1)/2), or a weight volume (fftshifted, box-sized, device). */
enum { TOMGPU_WEDGE_NONE = 0, TOMGPU_WEDGE_SIMPLE = 1, TOMGPU_WEDGE_VOLUME = 2 };
typedef struct {
    int kind;
    float angle_deg;
    const float* volume;
} tomgpu_wedge_spec;

/* The C++ picker's batched aligner: [out] = tom_mex_corr3d(size, templates,
 * particles, angles, mask, wedge_ref, wedge_part, 'peak', mask_cc)
 * (Oscar3/c++Picker/src/mex/tom_mex_corr3d.cpp:53-806 ->
 * tom::corr3d_batch, src/tom/corr/corr.cpp:1217-1470, with
 * CorrelationHandlerPeaks, src/tom/corr/correlation_handler.cpp:96-120).
 * templates / particles: host arrays of nt / np device pointers to box-sized
 * volumes (n, each axis an FFT length); angles_deg: nang x 3 [phi psi theta]
 * (host, degrees); mask (device, box) or NULL; wedge_t (nt) / wedge_p (np)
 * host arrays or NULL; mask_cc: fftshifted peak mask (device) or NULL.
 * Outputs, host, [particle][template] order (template fastest) like the
 * MEX's nt x np struct array: peak (3 doubles, 0-based x y z), val (ncc_val,
 * NaN when no angle gave a peak) and angle_idx (1-based, 0 when none). */
int tomgpu_corr3d_peaks_dev(tomgpu_ctx* ctx, const int n[3], const float* const* templates, int nt,
                            const float* const* particles, int np, const double* angles_deg, int nang,
                            const float* mask, const tomgpu_wedge_spec* wedge_t,
                            const tomgpu_wedge_spec* wedge_p, const float* mask_cc, double* peak,
                            double* val, int32_t* angle_idx);

/* tomgpu_corr3d_peaks_dev with every volume (templates, particles, mask,
 * wedge volumes, mask_cc) in host memory: the form the tom_mex_corr3d
 * gateway calls (Oscar3/c++Picker/src/mex/tom_mex_corr3d.cpp:53-806, whose
 * volumes are MATLAB arrays or EM files read on the host).  The volumes are
 * copied to the device for the call; outputs as tomgpu_corr3d_peaks_dev. */
int tomgpu_corr3d_peaks(tomgpu_ctx* ctx, const int n[3], const float* const* templates, int nt,
                        const float* const* particles, int np, const double* angles_deg, int nang,
                        const float* mask, const tomgpu_wedge_spec* wedge_t, const tomgpu_wedge_spec* wedge_p,
                        const float* mask_cc, double* peak, double* val, int32_t* angle_idx);

/* ---------------------------------------------------- learned proposer
 * Training and inference kernels of the candidate proposer (a dilated 3-D
 * convolutional network, tom_b200/proposer.py); no counterpart in the
 * reference.  Volumes are [C][Z][Y][X] FP32 device buffers of one sample;
 * weights [Cout][Cin][27] (taps x fastest), bias [Cout].  Gradient outputs
 * accumulate (zero them first); loss_dev is one device double that
 * accumulates. */
int tomgpu_cnn_conv3d_fwd_dev(tomgpu_ctx* ctx, const float* in, int ci, const int dims[3], const float* w,
                              const float* b, int co, int dil, int relu, float* out);
int tomgpu_cnn_conv3d_bwd_data_dev(tomgpu_ctx* ctx, const float* gout, int co, const int dims[3], const float* w,
                                   int ci, int dil, float* gin);
int tomgpu_cnn_conv3d_bwd_weight_dev(tomgpu_ctx* ctx, const float* in, int ci, const int dims[3], const float* gout,
                                     int co, int dil, float* gw, float* gb);
/* Dense layer over P samples: out[k][p] = b[k] + sum_c W[k][c] F[c][p]. */
int tomgpu_cnn_dense_fwd_dev(tomgpu_ctx* ctx, const float* W, const float* b, const float* F, int K, int C,
                             int64_t P, int relu, float* out);
int tomgpu_cnn_dense_bwd_dev(tomgpu_ctx* ctx, const float* W, const float* F, const float* g, int K, int C,
                             int64_t P, float* gF, float* gW, float* gb);
int tomgpu_cnn_relu_bwd_dev(tomgpu_ctx* ctx, float* g, const float* act, int64_t n);
int tomgpu_cnn_bce_dev(tomgpu_ctx* ctx, const float* logit, const float* target, int64_t n, float pos_weight,
                       float* grad, double* loss_dev);
int tomgpu_cnn_softmax_ce_dev(tomgpu_ctx* ctx, const float* logits, const int32_t* labels, int K, int P,
                              float* grad, double* loss_dev);
int tomgpu_cnn_adam_dev(tomgpu_ctx* ctx, float* p, const float* g, float* m, float* v, int64_t n, float lr,
                        float beta1, float beta2, float eps, int step);
int tomgpu_cnn_gather_dev(tomgpu_ctx* ctx, const float* f, int C, int64_t nv, const int64_t* idx, int P,
                          float* out);
int tomgpu_cnn_scatter_add_dev(tomgpu_ctx* ctx, const float* g, int C, int64_t nv, const int64_t* idx, int P,
                               float* gf);

/* U-Net candidate proposer (tom_b200/unet.py; no counterpart in the
 * reference): BF16 3x3x3 convolutions on the tensor cores with FP32
 * accumulation and the layers around them.  Activations are channels-last
 * BF16 (uint16_t bit patterns), act[z][y][x][c] with channel stride cs; a
 * call reads or writes the channel slice [off, off + C) (cs and off multiples
 * of 8, buffers 16-byte aligned).  dims = {X, Y, Z}.  Master weights are FP32
 * [Cout][Cin][27] (taps x fastest, t = 9 dz + 3 dy + dx, offset t - 13 in
 * the order (dx, dy, dz) - 1).  Gradient outputs accumulate (zero them
 * first).  Errors: TOMGPU_ERR_ARG for bad pointers / slices,
 * TOMGPU_ERR_UNSUPPORTED for channel counts outside the built kernels,
 * TOMGPU_ERR_TIMEOUT (from the next synchronising call) if a bounded device
 * wait ran out. */
/* The packed BF16 weights of one convolution (27 Cout Cin values): flip = 0
 * the forward form, flip = 1 the input-gradient form (taps mirrored, channel
 * roles swapped).  Cout, Cin multiples of 16, at most 96. */
int tomgpu_unet_pack_weights_dev(tomgpu_ctx* ctx, const float* w, int cout, int cin, int flip, uint16_t* packed);
/* out = act(conv3(in) + bias) on the tensor cores.  relu != 0 applies a
 * ReLU; mask != null multiplies by (mask > 0) (the derivative of a ReLU whose
 * output is mask; the input-gradient form).  Cin a multiple of 16 (<= 96),
 * Cout one of 16, 32, 48, 64, 96. */
int tomgpu_unet_conv3_dev(tomgpu_ctx* ctx, const uint16_t* in, int in_cs, int in_off, int cin, const int dims[3],
                          const uint16_t* packed, int cout, const float* bias, int relu, const uint16_t* mask,
                          int mask_cs, int mask_off, uint16_t* out, int out_cs, int out_off);
/* gw[co][ci][t] += sum_v gout[v][co] in[v + off(t)][ci] on the tensor cores
 * (Cin <= 96, Cout <= 64, multiples of 16). */
int tomgpu_unet_conv3_wgrad_dev(tomgpu_ctx* ctx, const uint16_t* in, int in_cs, int in_off, int cin,
                                const int dims[3], const uint16_t* gout, int g_cs, int g_off, int cout, float* gw);
/* First layer: one FP32 input channel -> 16 BF16 channels (bias, ReLU), and
 * its weight / bias gradients. */
int tomgpu_unet_conv_first_dev(tomgpu_ctx* ctx, const float* vol, const int dims[3], const float* w, const float* b,
                               uint16_t* out);
int tomgpu_unet_conv_first_wgrad_dev(tomgpu_ctx* ctx, const float* vol, const int dims[3], const uint16_t* gout,
                                     float* gw, float* gb);
/* Candidate head over n voxels of 16 channels, w = 16 weights and the bias
 * (17 floats): logit = w[16] + w[0..15] . f (prob != 0: its logistic
 * sigmoid, the centre probability); backward: gf = g w (f > 0) (written),
 * gw[0..15] += sum g f, gw[16] += sum g. */
int tomgpu_unet_head_dev(tomgpu_ctx* ctx, const uint16_t* f, int64_t n, const float* w, int prob, float* logit);
int tomgpu_unet_head_bwd_dev(tomgpu_ctx* ctx, const uint16_t* f, int64_t n, const float* w, const float* g,
                             uint16_t* gf, float* gw);
/* 2x2x2 average pool of a slice into a dense [C] volume (dims: the fine
 * volume, even), and its backward: gin[v][off + c] (+)= gout[v / 2][c] / 8,
 * times (mask > 0) when mask is given (mask shares gin's cs / off). */
int tomgpu_unet_pool_dev(tomgpu_ctx* ctx, const uint16_t* in, int cs, int off, int C, const int dims[3],
                         uint16_t* out);
int tomgpu_unet_pool_bwd_dev(tomgpu_ctx* ctx, const uint16_t* gout, int C, const int dims[3], const uint16_t* mask,
                             int cs, int off, uint16_t* gin, int accumulate);
/* Nearest 2x upsample of a dense [C] volume into a slice of the fine volume
 * (dims: fine), and its backward (sum of the 8 fine gradients). */
int tomgpu_unet_upsample_dev(tomgpu_ctx* ctx, const uint16_t* in, int C, const int dims[3], uint16_t* out, int cs,
                             int off);
int tomgpu_unet_upsample_bwd_dev(tomgpu_ctx* ctx, const uint16_t* gout, int cs, int off, int C, const int dims[3],
                                 uint16_t* gin);
/* out[c] += sum over n voxels of g[v][off + c] (bias gradients; C <= 96). */
int tomgpu_unet_channel_sum_dev(tomgpu_ctx* ctx, const uint16_t* g, int cs, int off, int C, int64_t n, float* out);
/* out = (vol - mean) / std over n values (moments in FP64 on the device;
 * out may be vol). */
int tomgpu_unet_normalise_dev(tomgpu_ctx* ctx, const float* vol, int64_t n, float* out);
/* 2x2x2 mean of an FP32 volume (dims even) into the half-size volume out. */
int tomgpu_unet_bin2_dev(tomgpu_ctx* ctx, const float* vol, const int dims[3], float* out);
/* Features at P voxels (flat indices) as FP32 F[c][p], and the scatter-add
 * of a gradient G[c][p] back into distinct voxels of a BF16 gradient, where
 * the ReLU features f are positive. */
int tomgpu_unet_gather_dev(tomgpu_ctx* ctx, const uint16_t* f, int C, const int64_t* idx, int P, float* out);
int tomgpu_unet_scatter_add_dev(tomgpu_ctx* ctx, const float* g, int C, const int64_t* idx, int P, const uint16_t* f,
                                uint16_t* gf);

/* ---------------------------------------------------------- peak analysis */

/* tom_os3_analyzePeak(img, peakMap, template, 'PSR')
 * (Oscar3/matlabPicker/analyze/tom_os3_analyzePeak.m:61-101): the peak map's
 * local mean and std under tom_os3_sphereMask(template) with a centred
 * floor(T/4) box zeroed, then (peak - mean)/std where std > 1000 eps(max std),
 * else 0.  peak_dev/out_dev: map-sized (map_dims, x edge even); tmpl_dims: the
 * template's size (only its size enters).  FP64 inside. */
int tomgpu_analyze_psr_dev(tomgpu_ctx* ctx, const float* peak_dev, const int map_dims[3],
                           const int tmpl_dims[3], float* out_dev);

/* A = tom_os3_corr(t, t) (search/tom_os3_corr.m:77-176, same-size inputs, no
 * options): the template's autocorrelation FLCF with the default sphere mask,
 * divided at every voxel.  Template-sized device buffers.  FP64 inside. */
int tomgpu_template_autocorr_dev(tomgpu_ctx* ctx, const float* t_dev, const int tmpl_dims[3], float* out_dev);

/* tom_os3_analyzePeak(0, peakMap, template, 'Autocorrelation')
 * (tom_os3_analyzePeak.m:174-190): the FLCF of the peak map with A =
 * tom_os3_corr(t, t) under mask_dev (options.correlation.mask; NULL =
 * tom_os3_sphereMask), with A's own statistics. */
int tomgpu_analyze_autocorr_dev(tomgpu_ctx* ctx, const float* peak_dev, const int map_dims[3],
                                const float* t_dev, const int tmpl_dims[3], const float* mask_dev,
                                float* out_dev);

/* tom_os3_bestPeak criteria (options.analysis.ccc / .psr / .autocorr). */
enum { TOMGPU_ANALYSIS_CCC = 1, TOMGPU_ANALYSIS_PSR = 2, TOMGPU_ANALYSIS_AUTOCORR = 4 };

/* Fill maxcc, psr and autoc with -1000 and angidx with -1. */
int tomgpu_match_init_analysis_dev(tomgpu_match_plan* plan, float* maxcc_dev, int32_t* angidx_dev,
                                   float* psr_dev, float* autoc_dev);

/* The search loop of tom_os3_findTemplate.m:255-307 as the reference runs it:
 * for every rotation the FLCF map, its PSR map and its autocorrelation map
 * (tom_os3_analyzePeak on the rotated, masked, filtered template), then
 * tom_os3_bestPeak (search/tom_os3_bestPeak.m:12-47): a voxel takes the
 * rotation's cc, psr, autocorrelation and index where every criterion in
 * `flags` (TOMGPU_ANALYSIS_*, at least one) strictly improves.  Several
 * N-sized FFTs per rotation: the analysis search, not the fast one. */
int tomgpu_match_run_analysis_dev(tomgpu_match_plan* plan, const float* eulers, int R, int index_offset,
                                  int flags, float* maxcc_dev, int32_t* angidx_dev, float* psr_dev,
                                  float* autoc_dev);

#ifdef __cplusplus
}
#endif
#endif /* TOMGPU_H */
