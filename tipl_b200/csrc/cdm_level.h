// Device state of one CDM level of one job (fields, scratch, control block).
#pragma once
#include <functional>
#include <string>
#include "host.h"

namespace regb {

// An instantiated CUDA graph of work captured from a stream.
struct GraphExec {
    cudaGraphExec_t exec = nullptr;
    long long nodes = 0;  // kernels per replay
    GraphExec() = default;
    GraphExec(const GraphExec&) = delete;
    GraphExec& operator=(const GraphExec&) = delete;
    ~GraphExec() { reset(); }
    void capture(const std::function<void(cudaStream_t)>& body);
    void launch(cudaStream_t st);
    void reset();
};

struct CdmLevel {
    int pix = 0;
    std::string gtypes;  // gradient type of each modality ('r' / 'd'), one char per pair
    CdmSeg seg{};
    CdmCtl h_ctl{};
    DevBuf<uint8_t> js;
    DevBuf<float> cur, nd, aux, tmp;
    DevBuf<double> part;
    DevBuf<CdmCtl> ctl;
    DevBuf<CdmSeg> d_seg;
    // It / Is: gtypes.size() modality pairs of one shape.  best is the level's in/out
    // field (starts as the upsampled coarser result).
    // ndim 2: a level of a 2-D registration (d == 1).
    void init(const void* const* It, const void* const* Is, const std::string& gtypes, int w, int h, int d, int pix,
              const regb_cdm_param& p, float* best, cudaStream_t st, int ndim = 3);
};

// One iteration of every segment in d_segs (reg/cdm.hpp:418-470); the segments
// share pix and the gradient types of their modalities (gtypes, one char each).
// blocks: sum(nblk) over the nseg entries, whose blk0 number them (one entry
// alone: its nblk, blk0 0).
void launch_iteration(const CdmSeg* d_segs, int nseg, int blocks, int pix, const std::string& gtypes,
                      cudaStream_t st);

}  // namespace regb
