#include "affine_eval.h"
#include "batcher.h"
#include "stats.h"
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <sys/stat.h>
#include <cstring>
#include <string>
#include <vector>

namespace regb {

void TaskScratch::ensure(int k, bool need_hist, cudaStream_t st)
{
    if (k <= cap && (!need_hist || hist.n >= (size_t)cap * 65536))
        return;
    const int c = std::max(k, std::max(16, cap * 2));
    if (need_hist) {
        hist.alloc((size_t)c * 65536, st);
        hist.zero();
        col.alloc((size_t)c * 256, st);
        col.zero();
        part.alloc((size_t)c * kMiReduceBlocks, st);
    }
    moments.alloc((size_t)c * 3, st);
    moments.zero();
    ticket.alloc((size_t)c, st);
    ticket.zero();
    cost.alloc((size_t)c, st);
    tasks.alloc((size_t)c, st);
    h_tasks.alloc((size_t)c);
    h_cost.alloc((size_t)c);
    cap = c;
}

void TaskScratch::release()
{
    hist.reset();
    col.reset();
    part.reset();
    moments.reset();
    ticket.reset();
    cost.reset();
    tasks.reset();
    h_tasks.reset();
    h_cost.reset();
    cap = 0;
}

static bool tex_enabled()
{
    static const bool on = [] {
        const char* e = std::getenv("REGB_TEXTURE");
        return !(e && e[0] == '0');
    }();
    return on;
}

void TexVol::reset()
{
    if (t)
        cudaDestroyTextureObject(t);
    t = 0;
    mem.reset();
}

void TexVol::build(const uint8_t* v, Dim3 d, cudaStream_t st)
{
    reset();
    // pitch-linear 2-D texture limits of sm_100 (131072 x 65000 texels), pitch in
    // multiples of 32 bytes
    const long long rows = (long long)d.h * d.d;
    if (!tex_enabled() || d.w < 2 || rows < 2 || d.w > 131072 || rows > 65000)
        return;
    const size_t pitch = (((size_t)d.w * 2 + 31) / 32) * 32 / 2;  // in halves
    mem.alloc(pitch * (size_t)rows, st);
    REGB_CK(launch_u8_to_half_pitched(v, d.w, rows, mem.p, pitch, st));
    cudaResourceDesc rd;
    std::memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypePitch2D;
    rd.res.pitch2D.devPtr = mem.p;
    rd.res.pitch2D.desc = cudaCreateChannelDesc(16, 0, 0, 0, cudaChannelFormatKindFloat);
    rd.res.pitch2D.width = (size_t)d.w;
    rd.res.pitch2D.height = (size_t)rows;
    rd.res.pitch2D.pitchInBytes = pitch * 2;
    cudaTextureDesc td;
    std::memset(&td, 0, sizeof(td));
    td.addressMode[0] = td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    if (cudaCreateTextureObject(&t, &rd, &td, nullptr) != cudaSuccess) {
        // no texture (e.g. the device's texture objects are used up): the byte-load
        // kernels read the volume instead, with the same results
        (void)cudaGetLastError();
        t = 0;
        mem.reset();
    }
}

// Minimum voxels per block of each cost kernel, per size bucket of the fixed grid
// (index [bucket][cost type]); the autotuner replaces the defaults with the fastest
// measured choice.  Chunking only decides which block counts which voxels, so every
// choice gives the same costs.
static std::atomic<int> g_min_block_voxels[kTuneBuckets][3] = {{{32768}, {60000}, {60000}},
                                                                {{32768}, {60000}, {60000}},
                                                                {{32768}, {60000}, {60000}},
                                                                {{32768}, {60000}, {60000}}};

int tune_bucket(long long voxels)
{
    // between the geometric means of the representative grids 64^3, 128^3,
    // 182x218x182 and 256^3
    return voxels <= 741455LL ? 0 : voxels <= 3890000LL ? 1 : voxels <= 11000000LL ? 2 : 3;
}

void check_mi_width(int fixed_width, const char* who)
{
    if (fixed_width > kMiMaxWidth)
        throw Failure(REGB_ERR_ARG, std::string(who) + ": the 256-bin MI takes fixed volumes at most 65535 voxels "
                                                       "wide (16-bit per-block counters)");
}

int min_block_voxels(int bucket, int cost_type) { return g_min_block_voxels[bucket][cost_type].load(); }
void set_min_block_voxels(int bucket, int cost_type, int v) { g_min_block_voxels[bucket][cost_type].store(v); }

void set_task_chunks(AffineTask& t, int cost_type)
{
    // a chunk is a run of whole rows of the fixed grid
    const long long w = t.fd.w, rows = (long long)t.fd.h * t.fd.d;
    const long long mv = g_min_block_voxels[tune_bucket(t.fd.n())][cost_type].load();
    long long rpc;
    if (cost_type == REGB_COST_MI) {
        // 16-bit per-block counters: at most 65535 voxels per block.  Blocks are made
        // large because each one ends with a flush of its whole shared histogram: fewer,
        // fuller blocks flush less often.
        const long long hi = std::max<long long>(1, 65535 / w);
        rpc = (rows + 147) / 148;
        rpc = std::max<long long>(rpc, (mv + w - 1) / w);
        rpc = std::min<long long>(rpc, hi);
    } else if (cost_type == REGB_COST_MI32)
        // 32-bit counters (no per-block voxel bound); about one block per SM for a large
        // grid, at least mv voxels per block for a small one
        rpc = std::max<long long>((rows + 147) / 148, (mv + w - 1) / w);
    else
        rpc = std::max<long long>(1, (mv + w - 1) / w);
    t.chunk = (int)rpc;
    t.nchunk = (int)std::max<long long>(1, (rows + rpc - 1) / rpc);
}

constexpr int kTuneTasks = 96;  // candidates per timed launch

// Candidate minimum voxels per block, by cost type (MI: at most 65535, its 16-bit counters).
static const int kTuneCand[3][5] = {{8192, 16384, 32768, 65536, 131072},  // correlation
                                    {16384, 32768, 49152, 60000, 65535},  // MI
                                    {8192, 16384, 32768, 60000, 131072}}; // MI32

static bool tune_candidate(int cost_type, int v)
{
    for (int c : kTuneCand[cost_type])
        if (c == v)
            return true;
    return false;
}

// The on-disk table: one line "<device name>|<bucket>|<cost type>|<voxels>" per choice.
static std::string tune_key()
{
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return "";
    }
    std::string k = prop.name;
    for (char& c : k)
        if (c == '|' || c == '\n')
            c = ' ';
    return k + " sm" + std::to_string(prop.major) + std::to_string(prop.minor);
}

static bool tune_load(const std::string& path, int* table)
{
    std::FILE* f = std::fopen(path.c_str(), "r");
    if (!f)
        return false;
    const std::string key = tune_key();
    int got = 0;
    int tmp[kTuneBuckets * 3];
    char line[512];
    while (std::fgets(line, sizeof(line), f)) {
        std::string l(line);
        const size_t p1 = l.find('|');
        if (p1 == std::string::npos || l.substr(0, p1) != key)
            continue;
        int b = -1, c = -1, v = 0;
        if (std::sscanf(l.c_str() + p1 + 1, "%d|%d|%d", &b, &c, &v) == 3 && b >= 0 && b < kTuneBuckets && c >= 0 &&
            c < 3 && tune_candidate(c, v)) {
            tmp[b * 3 + c] = v;
            got |= 1 << (b * 3 + c);
        }
    }
    std::fclose(f);
    if (got != (1 << (kTuneBuckets * 3)) - 1)
        return false;  // not this device's complete table
    std::memcpy(table, tmp, sizeof(tmp));
    return true;
}

static void tune_store(const std::string& path, const int* table)
{
    // create the directories on the way (an existing one is fine)
    for (size_t pos = path.find('/', 1); pos != std::string::npos; pos = path.find('/', pos + 1))
        ::mkdir(path.substr(0, pos).c_str(), 0755);
    // keep other devices' lines, replace this device's
    const std::string key = tune_key();
    std::vector<std::string> keep;
    if (std::FILE* f = std::fopen(path.c_str(), "r")) {
        char line[512];
        while (std::fgets(line, sizeof(line), f)) {
            std::string l(line);
            if (l.compare(0, key.size() + 1, key + "|") != 0)
                keep.push_back(l);
        }
        std::fclose(f);
    }
    const std::string tmp = path + ".tmp";
    std::FILE* f = std::fopen(tmp.c_str(), "w");
    if (!f)
        return;  // an unwritable cache only costs the next process a tuning run
    for (const auto& l : keep)
        std::fputs(l.c_str(), f);
    for (int b = 0; b < kTuneBuckets; ++b)
        for (int c = 0; c < 3; ++c)
            std::fprintf(f, "%s|%d|%d|%d\n", key.c_str(), b, c, table[b * 3 + c]);
    std::fclose(f);
    std::rename(tmp.c_str(), path.c_str());
}

std::string default_tune_cache()
{
    if (const char* e = std::getenv("REGB_AUTOTUNE_CACHE"))
        return e;
    if (const char* x = std::getenv("XDG_CACHE_HOME"))
        return std::string(x) + "/tipl_b200/autotune.txt";
    if (const char* h = std::getenv("HOME"))
        return std::string(h) + "/.cache/tipl_b200/autotune.txt";
    return "";
}

double autotune_cost_kernels(cudaStream_t st, int* chosen, const char* cache_path, int* from_cache)
{
    const auto t_start = std::chrono::steady_clock::now();
    const std::string path = cache_path ? (cache_path[0] ? std::string(cache_path) : default_tune_cache()) : "";
    int table[kTuneBuckets * 3];
    if (from_cache)
        *from_cache = 0;
    if (!path.empty() && tune_load(path, table)) {
        for (int b = 0; b < kTuneBuckets; ++b)
            for (int c = 0; c < 3; ++c)
                g_min_block_voxels[b][c].store(table[b * 3 + c]);
        if (chosen)
            std::memcpy(chosen, table, sizeof(table));
        if (from_cache)
            *from_cache = 1;
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    }
    // one smooth, many-valued pair per bucket, of the bucket's representative grid, and
    // kTuneTasks small rigid candidates: a launch of the order of the serving engine's
    // (its launches gather about 50 to 160 candidates; smaller launches outside the
    // engine get their chunks split to fill one wave)
    static const Dim3 kRep[kTuneBuckets] = {{64, 64, 64}, {128, 128, 128}, {182, 218, 182}, {256, 256, 256}};
    cudaEvent_t a, b;
    REGB_CK(cudaEventCreate(&a));
    REGB_CK(cudaEventCreate(&b));
    for (int bk = 0; bk < kTuneBuckets; ++bk) {
        const Dim3 d = kRep[bk];
        const size_t n = (size_t)d.n();
        std::vector<uint8_t> hf(n), hm(n);
        for (size_t i = 0; i < n; ++i) {
            const int x = (int)(i % d.w), y = (int)((i / d.w) % d.h), z = (int)(i / d.wh());
            hf[i] = (uint8_t)((x * 3 + y * 5 + z * 7) / 4 + ((x * y) >> 7));
            hm[i] = (uint8_t)((x * 2 + y * 3 + z * 5) / 3 + ((y * z) >> 7));
        }
        DevBuf<uint8_t> f(n, st), m(n, st);
        REGB_CK(cudaMemcpyAsync(f.p, hf.data(), n, cudaMemcpyHostToDevice, st));
        REGB_CK(cudaMemcpyAsync(m.p, hm.data(), n, cudaMemcpyHostToDevice, st));
        std::vector<float> T(12 * kTuneTasks);
        for (int k = 0; k < kTuneTasks; ++k) {
            const float ang = 0.01f * (float)(k % 12 - 6) + 0.002f * (float)(k / 12), ca = std::cos(ang),
                        sa = std::sin(ang);
            const float R[9] = {ca, -sa, 0.0f, sa, ca, 0.0f, 0.0f, 0.0f, 1.0f};
            const float c[3] = {d.w / 2.0f, d.h / 2.0f, d.d / 2.0f};
            for (int r = 0; r < 3; ++r) {
                float sh = c[r] + 0.3f * (float)(k % 3);
                for (int j = 0; j < 3; ++j) {
                    T[12 * k + 3 * r + j] = R[3 * r + j];
                    sh -= R[3 * r + j] * c[j];
                }
                T[12 * k + 9 + r] = sh;
            }
        }
        for (int ct = 0; ct < 3; ++ct) {
            AffineEvaluator ev({AffineEvaluator::Pair{f.p, d, m.p, d}}, ct, st);
            int best = g_min_block_voxels[bk][ct].load();
            float best_ms = 1e30f;
            for (int v : kTuneCand[ct]) {
                g_min_block_voxels[bk][ct].store(v);
                ev.eval(0, T.data(), kTuneTasks);  // warm-up
                float ms_min = 1e30f;
                for (int rep = 0; rep < 3; ++rep) {
                    REGB_CK(cudaEventRecord(a, st));
                    ev.eval(0, T.data(), kTuneTasks);
                    REGB_CK(cudaEventRecord(b, st));
                    REGB_CK(cudaEventSynchronize(b));
                    float ms = 0.0f;
                    REGB_CK(cudaEventElapsedTime(&ms, a, b));
                    ms_min = std::min(ms_min, ms);
                }
                if (ms_min < best_ms) {
                    best_ms = ms_min;
                    best = v;
                }
            }
            g_min_block_voxels[bk][ct].store(best);
            table[bk * 3 + ct] = best;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (chosen)
        std::memcpy(chosen, table, sizeof(table));
    if (!path.empty())
        tune_store(path, table);
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
}

// A launch of few tasks on small grids fills less than half of one wave of resident
// blocks at the tuned chunk size, and then one block's serial share of voxels sets
// its time.  Such a launch cuts every chunk into f pieces (never below
// kFillMinVoxels voxels a block), f the largest factor that still fits one wave:
// ceil(rows / ceil(rpc / f)) <= f * ceil(rows / rpc), so the launch stays within
// f times its blocks.  Chunking only decides which block counts which voxels, so
// the costs do not change.  The serving engine's gathered launches are left whole: its
// CDM rounds run on another stream at the same time and use the SMs such a launch
// leaves free (splitting them measured 2.5 % fewer jobs/s on the open-loop workload).
constexpr long long kFillMinVoxels = 2048;

void fill_wave(AffineTask* t, int K, int cost_type)
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return;
    }
    long long blocks = 0;
    for (int k = 0; k < K; ++k)
        blocks += t[k].nchunk;
    const long long slots = (long long)sms * cost_blocks_per_sm(cost_type == REGB_COST_CORR);
    const long long f = slots / std::max<long long>(1, blocks);
    if (f < 2)
        return;
    for (int k = 0; k < K; ++k) {
        const long long w = t[k].fd.w, rows = (long long)t[k].fd.h * t[k].fd.d;
        const long long floor_rows = std::max<long long>(1, (kFillMinVoxels + w - 1) / w);
        const long long rpc = std::min<long long>(t[k].chunk, std::max(floor_rows, (t[k].chunk + f - 1) / f));
        t[k].chunk = (int)rpc;
        t[k].nchunk = (int)std::max<long long>(1, (rows + rpc - 1) / rpc);
    }
}

void run_affine_tasks(TaskScratch& s, int K, int cost_type, cudaStream_t st, double* out, bool fill)
{
    if (fill)
        fill_wave(s.h_tasks.p, K, cost_type);
    int max_chunks = 1, max_chunks_tex = 1, ntex = 0;
    for (int k = 0; k < K; ++k) {
        AffineTask& t = s.h_tasks.p[k];
        t.ticket = s.ticket.p + k;
        t.cost = s.cost.p + k;
        t.moments = s.moments.p + 3 * k;
        t.hist = (cost_type != REGB_COST_CORR) ? s.hist.p + (size_t)k * 65536 : nullptr;
        t.col = (cost_type != REGB_COST_CORR) ? s.col.p + (size_t)k * 256 : nullptr;
        t.part = (cost_type != REGB_COST_CORR) ? s.part.p + (size_t)k * kMiReduceBlocks : nullptr;
        if (t.tex) {
            ++ntex;
            max_chunks_tex = std::max(max_chunks_tex, t.nchunk);
        } else
            max_chunks = std::max(max_chunks, t.nchunk);
    }
    if (ntex && ntex < K)  // texture tasks first (each task's outputs stay at its own index)
        std::stable_partition(s.h_tasks.p, s.h_tasks.p + K, [](const AffineTask& t) { return t.tex != 0; });
    REGB_CK(cudaMemcpyAsync(s.tasks.p, s.h_tasks.p, sizeof(AffineTask) * K, cudaMemcpyHostToDevice, st));
    double vox = 0.0, bytes = 0.0;
    for (int k = 0; k < K; ++k) {
        const AffineTask& t = s.h_tasks.p[k];
        vox += (double)t.fd.n();
        // algorithmic bytes of one evaluation: the fixed grid and the sampled volume
        // once each, plus the int32 joint histogram written and read (MI: 256x256, MI32: 32x32)
        bytes += (double)t.fd.n() + (double)t.md.n() +
                 (cost_type == REGB_COST_MI ? 524288.0 : (cost_type == REGB_COST_MI32 ? 8192.0 : 0.0));
    }
    KernelTimer tm;
    tm.begin(st, cost_type == REGB_COST_CORR ? 1 : 0);  // both MI forms count as MI
    // texture tasks (the first ntex) and byte-load tasks run as separate launches
    if (cost_type == REGB_COST_MI) {
        if (ntex)
            REGB_CK(launch_mi_tex(s.tasks.p, ntex, max_chunks_tex, st));
        if (ntex < K)
            REGB_CK(launch_mi(s.tasks.p + ntex, K - ntex, max_chunks, st));
    } else if (cost_type == REGB_COST_MI32) {
        if (ntex)
            REGB_CK(launch_mi32_tex(s.tasks.p, ntex, max_chunks_tex, st));
        if (ntex < K)
            REGB_CK(launch_mi32(s.tasks.p + ntex, K - ntex, max_chunks, st));
    } else {
        if (ntex)
            REGB_CK(launch_corr_tex(s.tasks.p, ntex, max_chunks_tex, st));
        if (ntex < K)
            REGB_CK(launch_corr(s.tasks.p + ntex, K - ntex, max_chunks, st));
    }
    tm.end(st, K, vox, bytes);
    // the 256-bin MI is a histogram launch plus a reduction launch per kernel variant
    count_launch((cost_type == REGB_COST_MI ? 2 : 1) * ((ntex ? 1 : 0) + (ntex < K ? 1 : 0)));
    REGB_CK(cudaMemcpyAsync(s.h_cost.p, s.cost.p, sizeof(double) * K, cudaMemcpyDeviceToHost, st));
    REGB_CK(cudaStreamSynchronize(st));
    std::memcpy(out, s.h_cost.p, sizeof(double) * K);
}

AffineEvaluator::AffineEvaluator(const std::vector<Pair>& levels, int cost_type, cudaStream_t st)
    : cost_type_(cost_type), st_(st)
{
    lv_.resize(levels.size());
    PinBuf<unsigned long long> h(2);
    for (size_t i = 0; i < levels.size(); ++i) {
        Lvl& L = lv_[i];
        L.p = levels[i];
        if (cost_type == REGB_COST_MI32) {
            // per level, normalize_upper_lower2(v, 31.99): values 0..31 (a constant volume stays 0)
            DevBuf<unsigned> mm(2, st);
            L.qf.alloc((size_t)L.p.fd.n(), st);
            L.qt.alloc((size_t)L.p.td.n(), st);
            L.qf.zero();
            L.qt.zero();
            REGB_CK(launch_normalize_to_u8(L.p.from, REGB_U8, L.p.fd.n(), kMi32Upper, L.qf.p, mm.p, st));
            REGB_CK(launch_normalize_to_u8(L.p.to, REGB_U8, L.p.td.n(), kMi32Upper, L.qt.p, mm.p, st));
            count_launch(4);
            L.p.from = L.qf.p;
            L.p.to = L.qt.p;
        }
        if (cost_type == REGB_COST_MI)
            check_mi_width(L.p.fd.w, "MI cost");
        const uint8_t* grid = L.p.from;
        long long n = L.p.fd.n();
        if (cost_type == REGB_COST_CORR && L.p.fd.n() > L.p.td.n()) {  // reg/linear.hpp:28-33
            L.swap = true;
            grid = L.p.to;
            n = L.p.td.n();
        }
        // the sampled volume as a texture (the to-volume, or the from-volume when the
        // correlation swaps the roles)
        if (L.swap)
            L.tex.build(L.p.from, L.p.fd, st);
        else
            L.tex.build(L.p.to, L.p.td, st);
        L.row_hist.alloc(256, st);
        L.sums.alloc(2, st);
        REGB_CK(launch_fixed_stats(grid, n, L.row_hist.p, L.sums.p, st));
        REGB_CK(cudaMemcpyAsync(h.p, L.sums.p, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        REGB_CK(cudaStreamSynchronize(st));
        L.sx = (long long)h.p[0];
        L.sxx = (long long)h.p[1];
    }
}

void AffineEvaluator::make_task(int level, const float* T, AffineTask& t) const
{
    const Lvl& L = lv_[level];
    std::memset(&t, 0, sizeof(t));
    float M[12];
    std::memcpy(M, T, sizeof(M));
    if (L.swap) {
        matrix_inverse(M);  // a singular matrix is left unchanged, as the reference does
        t.fixed = L.p.to;
        t.fd = L.p.td;
        t.moving = L.p.from;
        t.md = L.p.fd;
    } else {
        t.fixed = L.p.from;
        t.fd = L.p.fd;
        t.moving = L.p.to;
        t.md = L.p.td;
    }
    std::memcpy(t.T, M, sizeof(M));
    t.mode = 0;
    if (cost_type_ == REGB_COST_CORR && integer_shift(M, t.shift))
        t.mode = 1;  // the CPU resample's integer-shift copy
    t.tex = (unsigned long long)L.tex.t;  // the texture of the volume this task samples
    t.row_hist = L.row_hist.p;
    t.sx = L.sx;
    t.sxx = L.sxx;
    set_task_chunks(t, cost_type_);
}

std::vector<double> AffineEvaluator::eval(int level, const float* T, int K)
{
    std::vector<double> out(K);
    if (K == 0)
        return out;
    if (batcher_) {
        std::vector<AffineTask> t(K);
        for (int k = 0; k < K; ++k)
            make_task(level, T + 12 * k, t[k]);
        batcher_->eval(t.data(), K, cost_type_, out.data());
        return out;
    }
    s_.ensure(K, cost_type_ != REGB_COST_CORR, st_);
    for (int k = 0; k < K; ++k)
        make_task(level, T + 12 * k, s_.h_tasks.p[k]);
    run_affine_tasks(s_, K, cost_type_, st_, out.data());
    return out;
}

}  // namespace regb
