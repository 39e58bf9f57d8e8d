// Mask-moment initialisation of an affine registration (reg/linear.hpp:658-684).
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

namespace regb {

// Voxels > 0 per (x, y) column, (x, z) and (y, z) line of a uint8 volume.
struct MaskCounts {
    int w = 0, h = 0, d = 0;
    std::vector<uint32_t> xy, xz, yz;  // [y*w + x], [z*w + x], [z*h + y]
};

// One device pass (mask_count_kernel) and a copy of the tables to the host; syncs st.
void mask_counts(const uint8_t* d_vol, const int* dim, MaskCounts& out, cudaStream_t st);
bool has_mask(const MaskCounts& c);
void eigen_sym3(const double* A, double* V, double* d);
bool estimate_affine_param(const MaskCounts& src, const float* svs, const MaskCounts& tgt, const float* tvs,
                           float* arg);
void matrix_to_affine_param(const float* T, const int* from_dim, const float* from_vs, const int* to_dim,
                            const float* to_vs, float* arg);

}  // namespace regb
