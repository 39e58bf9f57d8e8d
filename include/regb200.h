/* regb200 -- C ABI of the B200 (sm_100a) registration hot path.
 *
 * Drop-in boundary for the reference's registration calls.  Each entry point below
 * names the reference interface it replaces (file:line within the reference
 * project).  Conventions:
 *   - volumes are x-fastest, index = (z*h + y)*w + x (utility/basic_image.hpp:160);
 *   - a displacement field is AoS float xyz per voxel (tipl::vector<3>);
 *   - a transform T[12] is the reference's transformation_matrix storage:
 *     T[0..8] = sr row-major, T[9..11] = shift; it maps a voxel of the fixed
 *     ("from") grid to a voxel of the sampled ("to") volume
 *     (numerical/transformation.hpp:589-605, 834-839);
 *   - an affine parameter vector is affine_param<float,3> order:
 *     translocation[3], rotation[3], scaling[3], affine[3]
 *     (numerical/transformation.hpp:428-438);
 *   - every call returns a regb_status; nothing throws across the ABI.
 * Pointers in a regb_volume / regb_field with location REGB_DEVICE are CUDA device
 * pointers on the current device; REGB_HOST pointers are ordinary host memory, and
 * the call copies in and out itself.  `stream` arguments are cudaStream_t values
 * (NULL = the legacy default stream); calls on host memory synchronise before they
 * return.
 */
#ifndef REGB200_H
#define REGB200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int regb_status;
#define REGB_OK 0
#define REGB_FALSE 1            /* the reference's `false` (cdm: zero cost / no result) */
#define REGB_ERR_ARG (-1)       /* bad argument (null pointer, size, dtype, limit) */
#define REGB_ERR_CUDA (-2)      /* a CUDA runtime error; see regb_last_error() */
#define REGB_ERR_NOMEM (-3)     /* device allocation failed */
#define REGB_CANCELLED (-4)     /* the caller's terminated flag was set */
#define REGB_ERR_NOTFOUND (-5)  /* unknown job id */
#define REGB_PENDING (-6)       /* job not finished yet (regb_poll) */
#define REGB_ERR_BUDGET (-7)    /* job larger than the engine's device-memory budget */

typedef enum { REGB_U8 = 0, REGB_F32 = 1, REGB_U16 = 2, REGB_BF16 = 3 } regb_dtype;
typedef enum { REGB_HOST = 0, REGB_DEVICE = 1 } regb_location;

typedef struct {
    void* ptr;
    int dim[3]; /* w, h, d */
    int dtype;  /* regb_dtype */
    int location;
} regb_volume;

typedef struct {
    float* ptr; /* 3 floats per voxel */
    int dim[3];
    int location;
} regb_field;

/* reg/linear.hpp:255-256 */
typedef enum { REGB_REG_TRANSLOCATION = 1, REGB_REG_ROTATION = 2, REGB_REG_RIGID_BODY = 3,
               REGB_REG_SCALING = 4, REGB_REG_TRANSLOCATION_SCALING = 5, REGB_REG_RIGID_SCALING = 7,
               REGB_REG_TILT = 8, REGB_REG_AFFINE = 15 } regb_reg_type;
/* REGB_COST_MI32: mutual information on a 32 x 32 joint histogram -- the reference's
 * mutual_information with mi_band_width 5 (reg/linear.hpp:81-82, 174-203), both volumes
 * quantised at every pyramid level by normalize_upper_lower2(v, 31.99) as it does for
 * non-uint8 images.  The reference builds only the 256-bin form; this is a variant. */
typedef enum { REGB_COST_CORR = 0, REGB_COST_MI = 1, REGB_COST_MI32 = 2 } regb_cost_type;
typedef enum { REGB_BOUND_REG = 0, REGB_BOUND_NARROW = 1, REGB_BOUND_LARGE = 2 } regb_bound;

/* linear_reg_param (reg/linear.hpp:268-288); bound selects reg_bound / narrow_bound /
 * large_bound (reg/linear.hpp:258-266). */
typedef struct {
    int reg_type;          /* regb_reg_type, default AFFINE */
    int cost_type;         /* regb_cost_type, default MI */
    int bound;             /* regb_bound, default REGB_BOUND_REG */
    unsigned int search_count; /* default 16 */
    int absolute_bound;    /* default 1 */
} regb_linear_param;

/* cdm_param (reg/cdm.hpp:36-44); gradient_type 'r' (local correlation) or 'd'. */
typedef struct {
    float resolution;      /* default 2.0 */
    float speed;           /* default 0.3 */
    float smoothing;       /* default 0.05 */
    unsigned int min_dimension; /* default 16 */
    int gradient_type;     /* default 'r' */
} regb_cdm_param;

void regb_linear_param_default(regb_linear_param* p);
void regb_cdm_param_default(regb_cdm_param* p);

/* Library status. */
const char* regb_version(void);
const char* regb_last_error(void);   /* thread-local text of the last failure */
regb_status regb_device_info(int* device, int* sm_count, size_t* free_bytes, size_t* total_bytes);
/* Release every cached device buffer of this thread's context and every cached page-locked host block. */
regb_status regb_release(void);
/* Testing hook (no counterpart in the reference, which reports a failed CUDA call in
 * cdm_cuda as `false`, reg/cdm.hpp:518-523): the next `count` device allocations of
 * exactly `bytes` bytes made by this library fail as if the device were out of memory,
 * so the call or engine job making them reports REGB_ERR_NOMEM; count 0 clears it.
 * Lets a test fail one job of a running engine on the host, without touching the GPU. */
regb_status regb_debug_fail_allocations(size_t bytes, int count);

/* Launch accounting (no reference counterpart: instrumentation of this library).
 * launches counts every kernel this library launched since the last reset; with
 * timing on, each MI / correlation cost launch is bracketed by CUDA events on its
 * stream and its algorithmic bytes (fixed voxels + sampled voxels + 2*256 KB of
 * histogram for MI) are accumulated. */
typedef struct {
    long long launches;
    long long mi_launches, mi_tasks;
    double mi_voxels, mi_bytes, mi_ms;
    long long corr_launches, corr_tasks;
    double corr_voxels, corr_bytes, corr_ms;
    double mi_busy_ms;   /* union of the MI launches' device intervals (launches on two
                            streams may overlap, so it can be below mi_ms) */
    long long cdm_iterations;  /* CDM iterations run (every level, every job) */
    double cdm_voxel_iterations;  /* sum over CDM levels of iterations x voxels of the level */
    double cdm_model_bytes;  /* the CDM pass model's bytes: voxel iterations x (596 + 4 x
                                bytes per pixel) -- compose, gradient, cost mean, Poisson
                                init and 12 sweeps, scale, accumulate, smooth, each pass
                                reading its inputs and writing its outputs once */
} regb_stats;
regb_status regb_stats_reset(int timing);
regb_status regb_stats_get(regb_stats* out);

/* ---- launch-shape autotuner (no counterpart in the reference) ---------------------- */
/* Times the batched affine cost kernels (correlation, MI, 32-bin MI) with 96 candidate
 * transforms a launch (the size of the serving engine's gathered launches) for a few
 * block sizes (minimum voxels per block) on the current device, on one pair per size
 * bucket (regb_autotune_buckets), and keeps the fastest of each for the rest of the
 * process.  Outside the serving engine, a launch that fills less than half of one wave
 * of resident blocks at the chosen size has its chunks split to fill it.  The choice only decides how voxels are
 * split across blocks, so costs are identical under every choice.  tuned (optional, indexed by regb_cost_type)
 * receives the choices for a 182x218x182 grid, seconds (optional) the time the tuning took. */
regb_status regb_autotune(int tuned[3], double* seconds);
/* The block sizes in use for a 182x218x182 grid (the defaults until a tuner runs). */
regb_status regb_tuning_get(int tuned[3]);
/* The tuner per size bucket of the fixed grid: buckets 0..3 hold grids of up to
 * 741,455 voxels, up to 3,890,000, up to 11,000,000, and more (around the 64^3, 128^3,
 * 182x218x182 and 256^3 grids); each bucket is timed on a pair of its representative
 * grid.  tuned (optional) receives the table, tuned[bucket * 3 + regb_cost_type].
 * cache_path: NULL = no file; "" = the default file ($REGB_AUTOTUNE_CACHE, else
 * $XDG_CACHE_HOME/tipl_b200/autotune.txt, else ~/.cache/tipl_b200/autotune.txt); a file
 * that holds this device's table (keyed by device name and compute capability) is loaded
 * instead of timing (*from_cache = 1), and a timed table is written to it.  regb_autotune
 * is this call without a file. */
regb_status regb_autotune_buckets(const char* cache_path, int tuned[12], double* seconds, int* from_cache);
/* The block sizes in use, tuned[bucket * 3 + regb_cost_type]. */
regb_status regb_tuning_get_buckets(int tuned[12]);

/* ---- transform algebra (host) -------------------------------------------------- */
/* transformation_matrix(affine_param, from, from_vs, to, to_vs)
 * (numerical/transformation.hpp:636-701), in float as the reference computes it. */
regb_status regb_affine_to_matrix(const float param[12], const int from_dim[3], const float from_vs[3],
                                  const int to_dim[3], const float to_vs[3], float T[12]);
/* The same composition in double (the FP64 affine path). */
regb_status regb_affine_to_matrix_f64(const double param[12], const int from_dim[3], const double from_vs[3],
                                      const int to_dim[3], const double to_vs[3], double T[12]);
/* transformation_matrix::inverse (numerical/transformation.hpp:820-832); REGB_FALSE if singular. */
regb_status regb_matrix_inverse(float T[12]);
/* transformation_matrix::to_affine_param(from, from_vs, to, to_vs)
 * (numerical/transformation.hpp:703-741): the 12 parameters (translocation, rotation,
 * scaling, affine) of a from-voxel -> to-voxel matrix. */
regb_status regb_matrix_to_affine_param(const float T[12], const int from_dim[3], const float from_vs[3],
                                        const int to_dim[3], const float to_vs[3], float param[12]);

/* ---- storage conversions ------------------------------------------------------------ */
/* normalize_upper_lower2(in, out, upper) (numerical/numerical.hpp:909-927) on the device:
 * out = uint8((in - min) * (upper / (max - min))) for a U8, F32, U16 or BF16 volume, in
 * the reference's float arithmetic.  The reference's callers quantise this way, with
 * upper = 255.999, before tipl::reg::linear.  REGB_FALSE (out untouched) when the volume
 * is constant, as the reference then returns without writing. */
regb_status regb_normalize_to_u8(const regb_volume* in, regb_volume* out, float upper, void* stream);
/* Exact widening of a U8, U16 or BF16 volume to F32 (BF16 = the upper 16 bits of an IEEE
 * float); the FP32 nonlinear path runs on volumes stored this way. */
regb_status regb_widen_to_f32(const regb_volume* in, regb_volume* out, void* stream);

/* ---- subject preprocessing of the mm_reg pipeline (reg/mm_reg.hpp:14-20) ----------- */
/* filter::gaussian(I, bandwidth) (filter/gaussian.hpp:18-96) of an F32 volume: bandwidth
 * rounds of the separable [1 2 1] x, y, z passes with the edge sample repeated, then the
 * scale 2^-(6 * bandwidth).  in and out are distinct F32 volumes of one shape. */
regb_status regb_gaussian(const regb_volume* in, regb_volume* out, int bandwidth, void* stream);
/* reg::subject_image_pre (reg/mm_reg.hpp:14-20): gaussian (bandwidth 1), then
 * segmentation::normalize_otsu_median(I, 255.99) (numerical/otsu.hpp:110-136), then the
 * float -> uint8 conversion.  in: F32, or U8 / U16 / BF16 widened exactly to float
 * first; out: U8 of the same shape.  Synchronises the stream (the Otsu threshold and
 * median are decided on the host). */
regb_status regb_subject_image_pre(const regb_volume* in, regb_volume* out, void* stream);

/* ---- mask-moment initialisation of linear() (reg/linear.hpp:658-684) --------------- */
/* has_mask(img) (numerical/basic_op.hpp:811-830) of a uint8 volume: *out = 1 when more
 * than a fifth of its voxels are 0 or its non-zero voxels' bounding box lies inside the
 * volume on some axis. */
regb_status regb_has_mask(const regb_volume* img, int* out);
/* estimate_affine_param(source, source_vs, target, target_vs, arg)
 * (numerical/transformation.hpp:933-1021) on uint8 volumes: parameters that map the
 * centroid and principal axes of source's voxels > 0 onto target's.  REGB_FALSE (param =
 * identity) when either volume has no voxel > 0.  The moments are formed from exact
 * per-line voxel counts made on the device; regb_linear runs this step itself. */
regb_status regb_estimate_affine_param(const regb_volume* source, const float source_vs[3],
                                       const regb_volume* target, const float target_vs[3], float param[12]);

/* ---- resample ------------------------------------------------------------------- */
/* tipl::resample<linear>(from, to, trans) (numerical/resampling.hpp:1239-1298):
 * to(x) = trilinear(from, T x), 0 outside; uint8 results truncate like the
 * reference.  allow_shift_copy != 0 takes the CPU path's integer-shift copy
 * (resampling.hpp:1243-1262) when T qualifies. from/to must share dtype (U8 or F32)
 * and location. */
regb_status regb_resample(const regb_volume* from, regb_volume* to, const float T[12], int allow_shift_copy,
                          void* stream);

/* ---- affine costs ---------------------------------------------------------------- */
/* mutual_information<3>::operator() (reg/linear.hpp:173-203, GPU 207-252) for K
 * candidate transforms at once: cost[k] = -MI of the 256x256 joint histogram of the
 * uint8 fixed volume and the trilinear uint8 sample of the moving volume.
 * hist_out (optional, host, K*65536 int32) receives the joint histograms. */
regb_status regb_mi_cost(const regb_volume* fixed, const regb_volume* moving, const float* T, int K,
                         double* cost, int32_t* hist_out, void* stream);
/* No counterpart in the reference: the same MI on a 32x32 joint histogram
 * (REGB_COST_MI32).  Both volumes are first quantised to 0..31 by
 * normalize_upper_lower2(v, 31.99) (the reference's step for non-uint8 inputs,
 * reg/linear.hpp:195-196); bin = (fixed << 5) + moving sample; the cost is
 * -sum(mu log(mu / row / col)) / 1024 (reg/linear.hpp:87-104 with 32 bins).
 * hist_out (optional, host, K*1024 int32) receives the joint histograms. */
regb_status regb_mi32_cost(const regb_volume* fixed, const regb_volume* moving, const float* T, int K,
                           double* cost, int32_t* hist_out, void* stream);
/* No counterpart in the reference.  The MI cost of regb_mi_cost for callers that
 * cannot allocate device memory -- a processing callback inside a host application
 * that owns all device memory through its own pool, or a latency-critical loop that
 * must not take the device-wide synchronisation cudaMalloc/cudaFree can cause.
 * fixed/moving are uint8 DEVICE pointers (dims w,h,d), T is K host transforms, cost
 * is a DEVICE array of K doubles.  Nothing is allocated: all scratch lives in one
 * file-scope device array (4 MiB of joint histograms plus about 25 KiB), so K <= 16 and
 * larger K is rejected with REGB_ERR_ARG, as is a fixed width above 65535.  The first
 * call on a device looks up that array's device address and fills the MI reduction's
 * n*ln(n) table (another static device array, 512 KiB); it is also the call on which
 * the CUDA runtime, which loads device code lazily, brings this library's kernels and
 * both arrays (about 4.5 MiB, plus code) into device memory, so make it during
 * initialisation, where allocation is still allowed.  Every call shares the array:
 * calls that overlap on the GPU (different streams or host threads without ordering)
 * race and give wrong costs.  The call is synchronous: it synchronises the stream
 * before it returns, so the costs are written when it returns, and it cannot be part
 * of a CUDA graph -- a call while the stream is being captured returns REGB_ERR_ARG. */
regb_status regb_mi_cost_noalloc(const uint8_t* fixed, const int fixed_dim[3], const uint8_t* moving,
                                 const int moving_dim[3], const float* T, int K, double* cost, void* stream);
/* correlation::operator() (reg/linear.hpp:23-78) for K transforms: 1 - r^2 with the
 * smaller volume as the grid (transform inverted when the roles swap). */
regb_status regb_corr_cost(const regb_volume* fixed, const regb_volume* moving, const float* T, int K,
                           double* cost, void* stream);

/* ---- displacement algebra -------------------------------------------------------- */
/* tipl::compose_displacement(from, dis, to) (numerical/dif.hpp:90-115, 260-285). */
regb_status regb_compose_displacement(const regb_volume* from, const regb_field* dis, regb_volume* to,
                                      void* stream);
/* tipl::accumulate_displacement(dis, new_dis) (numerical/dif.hpp:166-186, 311-329):
 * new_dis <- dis composed with new_dis, in place. */
regb_status regb_accumulate_displacement(const regb_field* dis, regb_field* new_dis, void* stream);
/* displacement_to_mapping(dis, mapping, T) (numerical/dif.hpp:42-51): mapping(x) =
 * T(x + dis(x)), the template-grid -> subject-voxel mapping of the mm_reg pipeline
 * (reg/mm_reg.hpp:279-283).  dis and mapping share a shape. */
regb_status regb_displacement_to_mapping(const regb_field* dis, const float T[12], regb_field* mapping, void* stream);
/* inv_displacement_to_mapping(inv_dis, inv_mapping, T) (numerical/dif.hpp:53-66): over the
 * inv_mapping grid, p = T^-1(x), inv_mapping(x) = p + trilinear(inv_dis, p) (zero off the
 * field); the subject-grid -> template-voxel mapping (reg/mm_reg.hpp:274-278).
 * REGB_FALSE when T is singular. */
regb_status regb_inv_displacement_to_mapping(const regb_field* inv_dis, const float T[12], regb_field* inv_mapping,
                                             void* stream);
/* compose_mapping(from, mapping) (numerical/dif.hpp:70-90) of a uint8 volume: to(x) =
 * trilinear(from, mapping(x)), 0 where the 2x2x2 cell leaves from; to has the mapping's shape. */
regb_status regb_compose_mapping(const regb_volume* from, const regb_field* mapping, regb_volume* to, void* stream);
/* It_match_fov (reg/mm_reg.hpp:313-329): a copy of the uint8 template It with 0 wherever
 * T (template voxel -> subject voxel) lands outside a subject volume of moving_dim. */
regb_status regb_match_fov(const regb_volume* It, const float T[12], const int moving_dim[3], regb_volume* out,
                           void* stream);
/* correlation(x, y) (numerical/statistics.hpp:585-598) of two uint8 volumes of one shape:
 * Pearson r from exact integer moments, 0 when either is constant; masked != 0 gives
 * correlation_ygz (:600-619), over the voxels with y > 0 only (mm_reg's default r). */
regb_status regb_correlation(const regb_volume* x, const regb_volume* y, int masked, double* r);
/* ---- NIfTI volumes (io/nifti.hpp) ------------------------------------------------- */
/* Geometry of a NIfTI file as tipl::io::gz_nifti reports it after its LPS
 * reorientation (toLPS, io/nifti.hpp:129-160, 1293-1298; handle_qform :1223-1260). */
typedef struct {
    int dim[3];            /* LPS dims (width, height, depth) */
    float vs[3];           /* voxel size, reordered with the axes (nii >> vs) */
    float srow[12];        /* voxel -> space rows srow_x, srow_y, srow_z (nii >> T) */
    int file_dim[8];       /* dim[] as stored */
    int datatype;          /* NIfTI datatype code, bitpix */
    int bitpix;
    int nvolumes;          /* volumes in the file (product of dim[4..dim[0]]) */
    float scl_slope, scl_inter;
    int sform_code;        /* after handle_qform */
    int is_mni;            /* gz_nifti::is_mni (io/nifti.hpp:856-864) */
    int big_endian;
    int nifti2;            /* 1: a NIfTI-2 (540-byte) header */
    int n_steps;           /* the reorientation: steps[0..n_steps) of 0..2 flip x/y/z, */
    int steps[8];          /* 3 swap xy, 4 swap yz, 5 swap xz, in the order applied */
    char descrip[81];
} regb_nifti_info;
/* Reads the header of a .nii, .nii.gz or .hdr/.img file (the gz_nifti open path,
 * io/nifti.hpp:624-754, with gz_stream's gzip handling); no device work. */
regb_status regb_nifti_info_read(const char* path, regb_nifti_info* info);
/* nii >> image<3,float> (io/nifti.hpp:1134-1172, 1193-1205) for volume `volume`:
 * the stored bytes go to the device as they are, and one kernel converts them
 * (byte order, datatype, scl_slope/scl_inter) into out in LPS orientation.  out:
 * REGB_F32, dims info->dim, host or device.  info (optional) receives the geometry.
 * Datatypes 2, 4, 8, 16, 64, 256, 512, 768, 1024, 1280 (RGB and complex are not
 * read). */
regb_status regb_nifti_load(const char* path, int volume, regb_volume* out, regb_nifti_info* info, void* stream);
/* nii << vs << T << is_mni << image (io/nifti.hpp:969-1030): writes vol (U8, U16 or F32,
 * host or device) as a NIfTI-1 file with its voxels as they are, pixdim vs, srow rows
 * and sform code 4 (is_mni) or 1.  Like the reference's writer, the file is always
 * gzip-compressed (io/gz_stream.hpp:535-580), whatever the extension, and a U16 volume
 * carries the int16 datatype code (its type table, io/nifti.hpp:286-290). */
regb_status regb_nifti_save(const char* path, const regb_volume* vol, const float vs[3], const float srow[12],
                            int is_mni, const char* descrip);
/* The displacement file of mm_reg::export_nonlinear (reg/mm_reg.hpp:418-441): a 4-D float
 * NIfTI of dims (w, h, d, 6) -- volumes 0..2 the x, y, z components of f2t (the reverse
 * field), volumes 3..5 those of t2f (the forward field) -- with the template's voxel
 * size and srow rows (sform code 1), written as the reference's writer writes it (gzip).
 * The export's volumes (I, It, J, JJ) are regb_nifti_save calls. */
regb_status regb_mm_reg_export_fields(const char* path, const regb_field* f2t, const regb_field* t2f, const float vs[3],
                                      const float srow[12]);

/* downsample_with_padding (numerical/resampling.hpp:575-671); out dims (d+1)/2. */
regb_status regb_downsample(const regb_volume* in, regb_volume* out, void* stream);
/* best_d *= 2; upsample_with_padding(best_d, shape) (reg/cdm.hpp:402-403,
 * numerical/resampling.hpp:849-891). */
regb_status regb_upsample_field_x2(const regb_field* in, regb_field* out, void* stream);

/* ---- CDM passes (reg/cdm.hpp) ----------------------------------------------------- */
/* cdm_get_gradient (reg/cdm.hpp:84-151): new_d = gradient, *cost = mean cost. */
regb_status regb_cdm_gradient(const regb_volume* Js, const regb_volume* It, regb_field* new_d, int gradient_type,
                              float* cost, void* stream);
/* cdm_solve_poisson (reg/cdm.hpp:158-253), 12 Jacobi sweeps, in place. */
regb_status regb_cdm_poisson(regb_field* new_d, void* stream);
/* cdm_max_displacement_length (reg/cdm.hpp:260-295). */
regb_status regb_cdm_max_length(const regb_field* d, float* out, void* stream);
/* cdm_smooth (reg/cdm.hpp:302-366): dd = blend(d, smoothing). */
regb_status regb_cdm_smooth(const regb_field* d, regb_field* dd, float smoothing, void* stream);

/* ---- whole registrations ---------------------------------------------------------- */
/* tipl::reg::cdm_common<out,T,3>(It, Is, dis, terminated, param) (reg/cdm.hpp:534-558,
 * the GPU path cdm_cuda 492-524) for one modality pair; It/Is uint8 or float, same dims and
 * dtype; dis_out receives the field.  Returns REGB_FALSE where the reference
 * returns false.  terminated (may be NULL) is polled between iterations. */
regb_status regb_cdm(const regb_volume* It, const regb_volume* Is, regb_field* dis_out, const regb_cdm_param* param,
                     volatile const int* terminated);
/* cdm_common over lists of modality pairs (reg/cdm.hpp:373-474, 534-558): It[i] / Is[i]
 * for i < nmod (1..12), all of one dims and dtype (uint8 or float).  Each iteration
 * composes and differentiates every modality, sums the gradients in modality order and
 * takes the mean of their costs (reg/cdm.hpp:419-435); a partial cost sum of exactly
 * zero returns REGB_FALSE.  gradient_types is cdm_param::gradient_type: modality i
 * uses its i-th char ('r' or 'd'), 'r' past its end; NULL = param->gradient_type for
 * modality 0 and 'r' for the others.  regb_cdm is this call with nmod = 1. */
regb_status regb_cdm_multi(const regb_volume* It, const regb_volume* Is, int nmod, regb_field* dis_out,
                           const regb_cdm_param* param, const char* gradient_types, volatile const int* terminated);
/* cdm_common<out, unsigned char, 2> over lists of 2-D modality pairs (reg/cdm.hpp:373-474,
 * 534-558 at dimension 2; the GPU instantiation it replaces is cdm_cuda<tipl::out,
 * unsigned char, 2> of reg/cdm_cu.hpp:12-17): It[i] / Is[i] uint8 images of dims
 * (w, h, 1), all alike.  dis_out has dims (w, h, 1) and receives the field as
 * interleaved x, y floats (tipl::vector<2>), 2*w*h of them.  The 2-D stencils are the
 * reference's: bilinear samples, a 5x5 regression window, Poisson and smoothing over
 * the four flat-index neighbours +-1, +-w with weights -1/4 and smoothing/4, and a
 * pyramid that recurses while min(w, h) > min_dimension.  Otherwise as regb_cdm_multi. */
regb_status regb_cdm2d_multi(const regb_volume* It, const regb_volume* Is, int nmod, regb_field* dis_out,
                             const regb_cdm_param* param, const char* gradient_types, volatile const int* terminated);
/* tipl::reg::linear<out,3>(from, from_vs, to, to_vs, arg, param, terminated)
 * (reg/linear.hpp:622-700): uint8 volumes (one image pair), arg in/out, final cost
 * out.  cost_evals (may be NULL) receives the number of cost evaluations. */
regb_status regb_linear(const regb_volume* from, const float from_vs[3], const regb_volume* to,
                        const float to_vs[3], float arg[12], const regb_linear_param* param,
                        volatile const int* terminated, float* cost_out, long long* cost_evals);
/* tipl::reg::linear over lists of image pairs (reg/linear.hpp:421-440, 517-525;
 * mm_reg's mm_linear): from[i] / to[i] for i < npairs (1..12), uint8, every from of one
 * dims and every to of one dims.  A candidate's cost is the sum of the pairs' costs
 * (0 + c0 + c1 + ..., in double) divided by 2 * npairs; the mask start looks at the
 * first pair.  regb_linear is this call with npairs = 1. */
regb_status regb_linear_multi(const regb_volume* from, const float from_vs[3], const regb_volume* to,
                              const float to_vs[3], int npairs, float arg[12], const regb_linear_param* param,
                              volatile const int* terminated, float* cost_out, long long* cost_evals);

/* The state of the reference's linear_reg_runner when its GPU implementation is
 * entered: linear_reg_imp<out,mr,uint8,3>(std::true_type, runner, cost_type,
 * terminated) (reg/linear.hpp:597-604, instantiated by reg/linear_cu.hpp:1-19).
 * Bounds and stage list are the runner's fields (linear_reg_runner, reg/linear.hpp:
 * 298-306); multi_resolution is the template flag mr. */
typedef struct {
    float arg_upper[12];
    float arg_lower[12];
    int reg_list[8];       /* DOF stages, e.g. {1, 5, 7, 15} */
    int n_reg;
    unsigned int search_count;
    int multi_resolution;  /* 1 = optimize<cost, true> (pyramid above 96^3) */
    int cost_type;         /* regb_cost_type */
    double precision;      /* default 0.001 */
    int max_iterations;    /* default 128 */
} regb_runner_state;
/* Fills the runner state tipl::reg::linear would set up for param (no mask-based
 * initialisation; that stays with the caller). */
regb_status regb_runner_state_from_param(const int from_dim[3], const float from_vs[3], const int to_dim[3],
                                         const float to_vs[3], const float arg[12], const regb_linear_param* param,
                                         regb_runner_state* out);
/* Runs the runner from that state on one image pair: arg in/out, final cost out. */
regb_status regb_linear_run(const regb_volume* from, const float from_vs[3], const regb_volume* to,
                            const float to_vs[3], float arg[12], const regb_runner_state* state,
                            volatile const int* terminated, float* cost_out, long long* cost_evals);
/* The same over npairs image pairs (as regb_linear_multi): the GPU branch of a
 * linear_reg_runner whose from / to lists hold several images. */
regb_status regb_linear_run_multi(const regb_volume* from, const float from_vs[3], const regb_volume* to,
                                  const float to_vs[3], int npairs, float arg[12], const regb_runner_state* state,
                                  volatile const int* terminated, float* cost_out, long long* cost_evals);

/* ---- serving engine ---------------------------------------------------------------
 * No counterpart in the reference (which registers one pair per call): registration
 * jobs submitted as they arrive run concurrently on one GPU.  Their affine probe sets
 * are evaluated together in shared launches and their CDM levels iterate together,
 * with continuous batching (jobs join and leave between launches).  A job starts
 * when a slot is free and its estimated device memory fits the budget.  Each job's
 * result equals what regb_linear / regb_cdm give for it alone. */
typedef struct regb_engine regb_engine;

typedef struct {
    size_t hbm_budget_bytes;   /* admission budget for running jobs; 0 = 80% of free memory */
    int max_active;            /* concurrent jobs; 0 = 64 */
    int gather_us;             /* once the device is free, how long a cost batch waits for
                                  more jobs to join; 0 = 10 us */
    int cdm_iters_per_round;   /* CDM iterations launched between two reads of the done
                                  flags; 0 = 4 */
    int affine_workers;        /* affine cost launches in flight at once (each worker its own
                                  stream and scratch), 1..4 (larger values are clamped); 0 = 3 */
} regb_engine_config;

/* One registration: affine (tipl::reg::linear) of moving to the template, then
 * optionally CDM (tipl::reg::cdm_common) of the template against the affine-
 * resampled moving volume (the reg/mm_reg.hpp:348-416 pipeline).  Host buffers must
 * stay valid until the job has finished. */
typedef struct {
    int template_id;           /* resident template (regb_engine_add_template), or -1 */
    regb_volume fixed;         /* used when template_id < 0 */
    float fixed_vs[3];
    regb_volume moving;
    float moving_vs[3];
    int run_linear;            /* 1 = run the affine stage (uint8 volumes) */
    regb_linear_param linear;
    float arg[12];             /* initial affine parameters */
    int run_cdm;               /* 1 = run CDM after the affine stage */
    regb_cdm_param cdm;
    float* field_out;          /* optional: receives the CDM field (template dims x 3 floats) */
    int field_location;        /* REGB_HOST or REGB_DEVICE for field_out */
    int subject_pre;           /* 0: subject quantised like a template (normalize_upper_lower2,
                                  255.999) unless already uint8; 1: subject_image_pre (gaussian +
                                  Otsu-median normalisation, reg/mm_reg.hpp:14-20) -- then the whole
                                  job runs on uint8 like the mm_reg pipeline */
    int mm_reg;                /* 1: the rest of the mm_reg pipeline (reg/mm_reg.hpp:286-416) after a
                                  uint8 CDM: the reverse CDM (subject on the template grid against the
                                  template), the mappings, and the linear / nonlinear correlations
                                  (correlation_ygz) in the result.  The reference's mm_reg
                                  registers with correlation (reg/mm_reg.hpp:53): set
                                  linear.cost_type = REGB_COST_CORR to match it (the Python
                                  Engine.submit does so when mm_reg is set) */
    float* field_rev_out;      /* optional: the reverse displacement (template dims x 3 floats) */
    float* mapping_out;        /* optional: template grid -> subject voxel mapping (template dims x 3) */
    float* inv_mapping_out;    /* optional: subject grid -> template voxel mapping (moving dims x 3) */
    const float* prev_field;   /* mm_reg, optional, with prev_field_rev: the forward and reverse */
    const float* prev_field_rev; /* fields of an earlier registration of this pair (template dims
                                  x 3 floats, at field_location).  The new fields are accumulated
                                  onto them (accumulate_displacement(previous_t2f, t2f_dis) and
                                  (previous_f2t, f2t_dis), reg/mm_reg.hpp:408-412) before the
                                  mappings and the nonlinear r; field_out / field_rev_out receive
                                  the accumulated fields */
} regb_job;

typedef struct {
    int status;                /* REGB_OK, REGB_CANCELLED or an error code */
    float linear_cost;
    float arg[12];
    long long cost_evals;
    int cdm_ok;                /* 1 when CDM ran and returned true */
    int cdm_iterations;
    double queued_ms;          /* submit -> start */
    double run_ms;             /* start -> done */
    int cdm_rev_ok;            /* mm_reg: 1 when the reverse CDM returned true */
    double r_linear;           /* mm_reg: correlation_ygz(affine-resampled subject, template) */
    double r_nonlinear;        /* mm_reg: correlation_ygz(subject through the mapping, template) */
} regb_result;

typedef struct {
    int queued, running;
    size_t used_bytes, budget_bytes;
    long long affine_launches, affine_tasks, cdm_rounds;
    long long cdm_round_segments;  /* CDM levels summed over rounds: / cdm_rounds = the
                                      levels that share one round's launches */
    double cdm_round_ms;           /* device time of the CDM rounds, summed (CUDA events on
                                      the scheduler's stream, from the segment upload to the
                                      status read-back) */
    int cdm_max_round_segments;    /* the most CDM levels one round has carried */
} regb_engine_stats;

void regb_engine_config_default(regb_engine_config* c);
void regb_job_default(regb_job* j);
regb_status regb_engine_create(const regb_engine_config* cfg, regb_engine** out);
/* Cancels queued and running jobs, waits for the running ones, frees everything. */
regb_status regb_engine_destroy(regb_engine* e);
/* Copies a template volume to the device once; jobs then refer to it by id. */
regb_status regb_engine_add_template(regb_engine* e, const regb_volume* vol, const float vs[3], int* template_id);
/* Queues a job; REGB_ERR_BUDGET when it can never fit the budget. */
regb_status regb_engine_submit(regb_engine* e, const regb_job* job, uint64_t* id);
/* REGB_OK with the result when the job has finished, REGB_PENDING otherwise. */
regb_status regb_engine_poll(regb_engine* e, uint64_t id, regb_result* out);
regb_status regb_engine_wait(regb_engine* e, uint64_t id, regb_result* out);
/* Sets the job's terminated flag (polled between iterations); a queued job ends at once. */
regb_status regb_engine_cancel(regb_engine* e, uint64_t id);
/* Drops a finished job's record. */
regb_status regb_engine_release_job(regb_engine* e, uint64_t id);
regb_status regb_engine_get_stats(regb_engine* e, regb_engine_stats* out);

#ifdef __cplusplus
}
#endif
#endif
