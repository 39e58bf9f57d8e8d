// Batched affine cost evaluation: K candidate transforms of one image pair (at one
// pyramid level) in a single launch.  Also the task-level entry used by the
// serving engine to put candidates of many jobs into one launch.
#pragma once
#include <string>
#include <vector>
#include "host.h"

namespace regb {

// Device scratch for up to `cap` tasks: MI histograms, correlation moments,
// completion tickets, costs.  Kept zeroed between launches by the kernels.
struct TaskScratch {
    int cap = 0;
    DevBuf<uint32_t> hist;
    DevBuf<uint32_t> col;    // 256-bin MI: 256 column sums per task
    DevBuf<double> part;     // 256-bin MI: kMiReduceBlocks partial sums per task
    DevBuf<unsigned long long> moments;
    DevBuf<unsigned int> ticket;
    DevBuf<double> cost;
    DevBuf<AffineTask> tasks;
    PinBuf<AffineTask> h_tasks;
    PinBuf<double> h_cost;
    void ensure(int k, bool need_hist, cudaStream_t st);
    void release();
};

class AffineBatcher;

// A uint8 volume held as a (w, h*d) 2-D texture of halves for the MI kernel's
// gathers (empty when the volume exceeds the pitch-linear texture limits).
struct TexVol {
    cudaTextureObject_t t = 0;
    DevBuf<uint16_t> mem;
    TexVol() = default;
    TexVol(const TexVol&) = delete;
    TexVol& operator=(const TexVol&) = delete;
    TexVol(TexVol&& o) noexcept : t(o.t), mem(std::move(o.mem)) { o.t = 0; }
    TexVol& operator=(TexVol&& o) noexcept
    {
        if (this != &o) {
            reset();
            t = o.t;
            mem = std::move(o.mem);
            o.t = 0;
        }
        return *this;
    }
    ~TexVol() { reset(); }
    void reset();
    // Builds the texture of v (device, dims d); leaves t = 0 when d does not fit.
    void build(const uint8_t* v, Dim3 d, cudaStream_t st);
};

// normalize_upper_lower2 bound of the 32-bin MI: float(32) - 0.01f (reg/linear.hpp:195-196)
constexpr float kMi32Upper = 32.0f - 0.01f;
// The 256-bin MI kernel counts in 16-bit shared-memory counters and a block holds at
// least one whole row of the fixed grid, so a row may hold at most 65535 voxels.
constexpr int kMiMaxWidth = 65535;
// Throws REGB_ERR_ARG when a 256-bin MI grid's rows are wider than kMiMaxWidth.
void check_mi_width(int fixed_width, const char* who);

// Fills the scratch pointers of h_tasks[0..K), launches the MI or correlation
// kernel for all of them, and copies the costs back (synchronises st).  fill: split
// the chunks of a launch below half a wave (fill_wave); the serving engine's batcher
// passes false.
void run_affine_tasks(TaskScratch& s, int K, int cost_type, cudaStream_t st, double* out, bool fill = true);

// Chunking of one task over its fixed-grid voxels.
void set_task_chunks(AffineTask& t, int cost_type);
// Splits the chunks of a launch of K tasks that fills less than half of one wave of
// resident blocks (costs unchanged: chunking only decides which block counts which voxels).
void fill_wave(AffineTask* t, int K, int cost_type);
// The chunking parameter (minimum voxels per block) per size bucket of the fixed grid
// and cost type, and its autotuner: for each bucket it times each cost kernel on a pair
// of the bucket's representative grid (64^3, 128^3, 182x218x182, 256^3) with 96
// candidates a launch for a few block sizes on the current device and keeps the fastest
// (results do not depend on the choice).  chosen (optional) receives the table
// [bucket * 3 + cost type]; cache_path names a table file (NULL: none, "": the default
// file), which is read instead of timing when it holds this device's table and written
// after timing; from_cache (optional) tells which happened.  Returns the seconds taken.
constexpr int kTuneBuckets = 4;
int tune_bucket(long long voxels);
int min_block_voxels(int bucket, int cost_type);
void set_min_block_voxels(int bucket, int cost_type, int v);
std::string default_tune_cache();
double autotune_cost_kernels(cudaStream_t st, int* chosen, const char* cache_path, int* from_cache);

class AffineEvaluator {
public:
    struct Pair {
        const uint8_t* from;
        Dim3 fd;
        const uint8_t* to;
        Dim3 td;
    };
    AffineEvaluator(const std::vector<Pair>& levels, int cost_type, cudaStream_t st);
    // T: K transforms (12 floats each) mapping the level's from-grid to its to-volume.
    std::vector<double> eval(int level, const float* T, int K);
    // Builds the task of one candidate (used by the engine to batch across jobs).
    void make_task(int level, const float* T, AffineTask& out) const;
    int cost_type() const { return cost_type_; }
    // Route evaluations through a cross-job batcher instead of launching directly.
    void set_batcher(AffineBatcher* b) { batcher_ = b; }

private:
    struct Lvl {
        Pair p;
        bool swap = false;  // correlation: the to-volume is the smaller one and becomes the grid
        DevBuf<uint8_t> qf, qt;  // 32-bin MI: the level's volumes quantised to 0..31
        TexVol tex;              // the sampled volume as a texture (t = 0: byte loads)
        DevBuf<int32_t> row_hist;
        DevBuf<unsigned long long> sums;
        long long sx = 0, sxx = 0;
    };
    std::vector<Lvl> lv_;
    int cost_type_;
    cudaStream_t st_;
    TaskScratch s_;
    AffineBatcher* batcher_ = nullptr;
};

}  // namespace regb
