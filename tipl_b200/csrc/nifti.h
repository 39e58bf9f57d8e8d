// NIfTI-1 / NIfTI-2 volumes in and out of the registration path (io/nifti.hpp of the
// reference): the header is parsed and the LPS reorientation worked out on the host;
// the voxel bytes go to the device as they are in the file, and one kernel converts
// them (byte order, data type, scl_slope / scl_inter) and reorients them.
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include "host.h"

namespace regb {

// The header fields the reader uses, in the NIfTI-1 types (a NIfTI-2 header is
// narrowed to them as the reference does, io/nifti.hpp:682-719).
struct NiftiHeader {
    int16_t datatype = 0, bitpix = 0;
    int16_t dim[8] = {0};
    float pixdim[8] = {0};
    float vox_offset = 352.0f;
    float scl_slope = 1.0f, scl_inter = 0.0f;
    int16_t qform_code = 0, sform_code = 0;
    float quatern_b = 0, quatern_c = 0, quatern_d = 0;
    float qoffset_x = 0, qoffset_y = 0, qoffset_z = 0;
    float srow[12] = {0};  // srow_x, srow_y, srow_z
    char descrip[80] = {0};
    bool big_endian = false;
    bool nifti2 = false;
    bool pair = false;  // header and voxels in separate .hdr / .img files
};

// A parsed file, reoriented to LPS (io/nifti.hpp:1293-1298, :129-160).
struct NiftiFile {
    NiftiHeader h;                // after handle_qform and the LPS steps
    int16_t file_dim[8] = {0};    // dims as stored in the file
    std::vector<char> seq;        // 0..2 flip x/y/z, 3 swap xy, 4 swap yz, 5 swap xz
    // file voxel (x, y, z) = M * (LPS voxel) + o, with the LPS volume of dims h.dim[1..3]
    int M[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    long long o[3] = {0, 0, 0};
};

// Reads and parses the header of path (.nii, .nii.gz, .hdr/.img); throws Failure.
NiftiFile nifti_open(const std::string& path);
// Bytes of volume `vol` (the first three dims) exactly as stored; throws Failure.
std::vector<uint8_t> nifti_read_voxels(const std::string& path, const NiftiFile& f, int vol);
int nifti_bytes_per_voxel(int datatype, int bitpix);
// Writes a NIfTI-1 file the way the reference's writer does (io/nifti.hpp:969-1020,
// io/gz_stream.hpp:535-580): the 348-byte header, four zero bytes and the voxels, not
// reoriented, through a gzip stream whatever the file name's extension.
void nifti_write(const std::string& path, const void* data, int datatype, int bitpix, const int dim[3],
                 const float vs[3], const float srow[12], int sform_code, const char* descrip, int nvol = 1);

}  // namespace regb
