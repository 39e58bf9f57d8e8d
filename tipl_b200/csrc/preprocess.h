// Subject preprocessing of the mm_reg pipeline (reg/mm_reg.hpp:14-20) on the device.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace regb {

// filter::gaussian(I, bandwidth) (filter/gaussian.hpp:18-96): d_out may equal d_in
// only for bandwidth 0.
void gaussian(const float* d_in, const int* dim, int bandwidth, float* d_out, cudaStream_t st);
// segmentation::otsu_median (numerical/otsu.hpp:86-100); syncs st.
float otsu_median(const float* d_img, long long n, cudaStream_t st);
// correlation(x, y) of two uint8 device volumes (numerical/statistics.hpp:569-598), or
// correlation_ygz (masked: voxels with y > 0 only); syncs st.
double correlation_u8(const uint8_t* d_x, const uint8_t* d_y, long long n, bool masked, cudaStream_t st);
// reg::subject_image_pre: gaussian, normalize_otsu_median(I, 255.99), uint8; syncs st.
void subject_image_pre(const float* d_in, const int* dim, uint8_t* d_out, cudaStream_t st);

}  // namespace regb
