// Internal (C++) interface between the host drivers and the CUDA kernels.
// Nothing here is part of the C ABI (include/regb200.h).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#ifdef __CUDACC__
#define REGB_HD __host__ __device__
#else
#define REGB_HD
#endif

namespace regb {

struct Dim3 {
    int w, h, d;
    REGB_HD long long n() const { return (long long)w * h * d; }
    REGB_HD int wh() const { return w * h; }
};

// One affine cost evaluation: a (job, candidate transform) pair.  All pointers are
// device pointers.  hist/moments/ticket are per-task scratch that must be zero on
// entry; the kernel's last block re-zeroes them.
struct AffineTask {
    const uint8_t* fixed;   // the grid the cost is summed over (template)
    const uint8_t* moving;  // the sampled volume
    Dim3 fd;                // fixed extent
    Dim3 md;                // moving extent
    float T[12];            // fixed voxel -> moving voxel (sr row-major, shift)
    int mode;               // 0 trilinear, 1 integer-shift copy (correlation only)
    unsigned long long tex; // 0, or the moving volume as a (w, h*d) texture of halves
                            // (cudaTextureObject_t) read by the cost kernels' gathers
    int keep;               // MI: 1 = leave the counts in hist (no reduction, no clearing)
    int shift[3];
    int nchunk;             // chunks of this task
    int chunk;              // rows (y, z) of the fixed grid per chunk
    uint32_t* hist;                // MI: 65536 counters
    uint32_t* col;                 // MI (256 bins): the 256 column sums of hist
    double* part;                  // MI (256 bins): kMiReduceBlocks partial sums
    const int32_t* row_hist;       // MI: template value histogram (256)
    unsigned long long* moments;   // correlation: sum y, sum y^2, sum x*y
    long long sx, sxx;             // correlation: template sum x, sum x^2
    unsigned int* ticket;          // blocks finished
    double* cost;                  // output
};

// Modality pairs one CDM level takes (the reference's mm_reg holds at most 12).
constexpr int kCdmMaxModalities = 12;

// Device control block of one CDM level of one job (the reference's host-side
// loop state, reg/cdm.hpp:408-470, kept on the device so iterations need no host
// round trip).
struct CdmCtl {
    float cost[8];
    int ncost;
    float best_cost;
    float cur_smoothing;
    float theta;
    float scale;           // speed / theta
    float speed;
    float smoothing;       // cdm_param::smoothing (the stop threshold)
    int index;             // iteration of this level
    int max_iter;          // 200
    int done;              // 1 = loop left (break / iteration cap / theta 0), 2 = zero cost (failure)
    int save_best;         // this iteration: best_d <- cur_d
    int restore;           // this iteration: cur_d <- best_d
    unsigned int theta_bits;  // max |new_d| of the first iteration (float bits)
    unsigned int ticket;
    float last_cost;
    int iters_run;
    float mod_cost[kCdmMaxModalities];  // this iteration's mean cost of each modality
};

// One CDM job level as seen by the iteration kernels (blockIdx.y = segment).
struct CdmSeg {
    int w, h, d;
    int nblk;         // blocks this segment uses (a function of its size only, so a
                      // job's reduction order does not depend on what it is batched with)
    int nmod;         // modality pairs (1 when 0)
    int ndim;         // 2: a 2-D level (d == 1; tipl::image<2> and vector<2> math: bilinear
                      // samples, the Poisson and smoothing weights of 4 neighbours; the
                      // field's z stays 0); anything else: 3-D
    const void* It[kCdmMaxModalities];  // template (fixed) image of each modality at this level
    const void* Is[kCdmMaxModalities];  // subject (moving) image of each modality at this level
    void* Js;         // composed subject (scratch, pixel type)
    float* cur_d;     // current field
    float* best_d;    // best field
    float* new_d;     // gradient -> Poisson result (scratch)
    float* aux_d;     // Poisson iterate A / Poisson result (scratch)
    float* tmp_d;     // Poisson iterate B / accumulated field (scratch)
    double* cost_part;  // per-block partial cost sums (nblk entries)
    CdmCtl* ctl;
    // A launch over several segments (their entries back to back) has sum(nblk) blocks:
    // this segment owns blocks [blk0, blk0 + nblk), blk0 ascending along the entries
    // (0 for a launch of this segment alone).
    int blk0;
};

template <typename T>
cudaError_t launch_resample(const T* from, Dim3 fd, T* to, Dim3 td, const float* Tm, const int* shift,
                            cudaStream_t st);
// Blocks per task of the 256x256 MI reduction (each reduces 65536 / 32 bins).
constexpr int kMiReduceBlocks = 32;
// The 256-bin MI: the histogram launch, then the reduction launch (which leaves
// hist, col and ticket zeroed again).  A task with keep = 1 keeps its counts and
// column sums and gets no cost.
cudaError_t launch_mi(const AffineTask* d_tasks, int ntask, int max_chunks, cudaStream_t st);
// The same with every task's moving volume read through its texture (tex != 0).
cudaError_t launch_mi_tex(const AffineTask* d_tasks, int ntask, int max_chunks, cudaStream_t st);
// Writes a uint8 volume of n voxels as halves (a texture's backing store, rows of w
// voxels at a pitch of `pitch` halves).
cudaError_t launch_u8_to_half_pitched(const uint8_t* in, int w, long long rows, void* out, size_t pitch,
                                      cudaStream_t st);
cudaError_t launch_corr(const AffineTask* d_tasks, int ntask, int max_chunks, cudaStream_t st);
// 32 x 32-bin MI (volumes quantised to 0..31); hist: 1024 counters per task, zero on entry
cudaError_t launch_mi32(const AffineTask* d_tasks, int ntask, int max_chunks, cudaStream_t st);
// The MI32 and correlation kernels with every task's moving volume read through its
// texture (tex != 0; correlation tasks in integer-shift mode still read bytes).
cudaError_t launch_mi32_tex(const AffineTask* d_tasks, int ntask, int max_chunks, cudaStream_t st);
cudaError_t launch_corr_tex(const AffineTask* d_tasks, int ntask, int max_chunks, cudaStream_t st);
// Blocks of a cost kernel resident on one SM (is_corr: the correlation kernel, else
// either MI kernel, which launch one 768-thread block per SM).
int cost_blocks_per_sm(bool is_corr);
cudaError_t launch_fixed_stats(const uint8_t* f, long long n, int32_t* hist, unsigned long long* sums,
                               cudaStream_t st);

// CDM passes.  pix: 0 = uint8, 1 = float.  segs is a device array of nseg segments;
// blocks is gridDim.x per segment.
// mod selects the modality pair: compose reads Is[mod]; the gradient reads It[mod],
// writes new_d for modality 0 and adds to it for the others, and its last block keeps
// the modality's mean cost; after the last modality that block also runs the loop
// decisions.
cudaError_t launch_cdm_compose(const CdmSeg* segs, int nseg, int blocks, int pix, cudaStream_t st, int mod = 0);
cudaError_t launch_cdm_gradient(const CdmSeg* segs, int nseg, int blocks, int pix, int gradient_type,
                                cudaStream_t st, int mod = 0);
// 12 sweeps; the first also applies best_d save/restore, the last forms theta.
cudaError_t launch_cdm_poisson(const CdmSeg* segs, int nseg, int blocks, int sweeps, cudaStream_t st);
cudaError_t launch_cdm_theta(const CdmSeg* segs, int nseg, int blocks, cudaStream_t st);
cudaError_t launch_cdm_accumulate(const CdmSeg* segs, int nseg, int blocks, cudaStream_t st);
cudaError_t launch_cdm_smooth(const CdmSeg* segs, int nseg, int blocks, cudaStream_t st);

// Pyramid passes (single volume, device pointers).
cudaError_t launch_downsample(const void* in, void* out, int w, int h, int d, int pix, cudaStream_t st);
cudaError_t launch_upsample_field_x2(const float* in, int iw, int ih, int id, float* out, int ow, int oh, int od,
                                     cudaStream_t st, int ndim = 3);
// The x, y components of an xyz field (n voxels) as interleaved pairs (tipl::vector<2>).
cudaError_t launch_field_xy(const float* xyz, long long n, float* xy, cudaStream_t st);
// Sum of a segment's cost partials -> float mean (the reference's mean(cost_map)).
cudaError_t launch_cost_mean(const CdmSeg* segs, int nseg, float* out, cudaStream_t st);
int cdm_blocks_for(long long nvox);
// out[i] = segs[i].ctl->done
cudaError_t launch_cdm_status(const CdmSeg* segs, int nseg, int* out, cudaStream_t st);

// normalize_upper_lower2 to uint8 of a U8 / F32 / U16 / BF16 volume (dtype codes of
// regb_dtype); mm is 2 words of device scratch; out is untouched when max == min
// (then mm[0] == mm[1] afterwards).
cudaError_t launch_normalize_to_u8(const void* in, int dtype, long long n, float upper, uint8_t* out, unsigned* mm,
                                   cudaStream_t st);
// Exact min / max of a U8 / F32 / U16 / BF16 volume as order-preserving float keys:
// mm[0] = key(min), mm[1] = key(max), key(f) = f >= 0 ? bits | 2^31 : ~bits.
cudaError_t launch_minmax(const void* in, int dtype, long long n, unsigned* mm, cudaStream_t st);
// Exact widening of a U8 / F32 / U16 / BF16 volume to float.
cudaError_t launch_widen_to_f32(const void* in, int dtype, long long n, float* out, cudaStream_t st);

// Subject preprocessing (preprocess_kernels.cu).  One round of the separable [1 2 1]
// Gaussian (x, y, z passes), optionally times scale.
cudaError_t launch_gaussian_round(const float* in, float* out, int w, int h, int d, float scale, int apply_scale,
                                  cudaStream_t st);
// 256-bin histogram of floor((v - mn) * range), clamped to [0, 255] (zeroes hist first).
cudaError_t launch_otsu_hist(const float* v, long long n, float mn, float range, unsigned* hist, cudaStream_t st);
// The values > ot in voxel order into out; counts holds compact_tiles(n) + 1 words and
// receives the total in its last word.
long long compact_tiles(long long n);
cudaError_t launch_compact_above(const float* v, long long n, float ot, unsigned* counts, float* out, cudaStream_t st);
// The 256 chunk middles of median() over m >= 2048 values.
cudaError_t launch_chunk_medians(const float* v, long long m, float* med, cudaStream_t st);
// count of v * s > 0 (zeroes cnt first)
cudaError_t launch_positive_count(const float* v, long long n, float s, unsigned long long* cnt, cudaStream_t st);
// out = uint8(clamp(v * s - (shift ? c : 0), 0, upper))
cudaError_t launch_otsu_normalize(const float* v, long long n, float s, int shift, float c, float upper, uint8_t* out,
                                  cudaStream_t st);

// Mapping steps of the mm_reg pipeline (mapping_kernels.cu).  Fields are AoS float xyz.
// mapping = T(dis + index); out = iT(index) + trilinear(inv_dis, iT(index)) over MD;
// to = uint8 trilinear(from, mapping) (0 off from); m[6] = exact sums x, y, x^2, y^2, xy and
// the count, over all voxels or (masked) those with y > 0.
cudaError_t launch_displacement_to_mapping(const float* dis, Dim3 D, const float* T, float* mapping, cudaStream_t st);
cudaError_t launch_inv_displacement_to_mapping(const float* inv_dis, Dim3 DD, const float* iT, Dim3 MD, float* out,
                                               cudaStream_t st);
cudaError_t launch_compose_mapping_u8(const uint8_t* from, Dim3 FD, const float* mapping, Dim3 MD, uint8_t* to,
                                      cudaStream_t st);
cudaError_t launch_moments_u8(const uint8_t* x, const uint8_t* y, long long n, int masked, unsigned long long* m,
                              cudaStream_t st);
// out = It where T(x) lies inside a volume of shape MD, else 0 (mm_reg's It_match_fov)
cudaError_t launch_match_fov_u8(const uint8_t* It, Dim3 FD, const float* T, Dim3 MD, uint8_t* out, cudaStream_t st);

// One NIfTI volume from its stored bytes to the float32 LPS volume (nifti_kernels.cu):
// out voxel v reads file voxel M v + o; datatype is the NIfTI code.
struct NiftiMap {
    Dim3 file;  // dims as stored
    Dim3 out;   // dims after the reorientation
    int M[9];
    long long o[3];
    int datatype;
    int big_endian;
    float scl_slope, scl_inter;
};
cudaError_t launch_nifti_convert(const uint8_t* raw, const NiftiMap& m, float* out, cudaStream_t st);

// Voxels > 0 per (x, y), (x, z), (y, z) line of a uint8 volume (zeroes the tables first).
cudaError_t launch_mask_counts(const uint8_t* v, Dim3 dim, uint32_t* xy, uint32_t* xz, uint32_t* yz,
                               cudaStream_t st);

}  // namespace regb
