// NIfTI-1 images for the dualgpmf command line: single-file (.nii, .nii.gz)
// and two-file (.hdr/.img, optionally gzipped) datasets, both byte orders.
//
// Written from the NIfTI-1 format definition: the 348-byte header, the
// voxel order (x fastest), and the two ways of mapping voxel indices to
// scanner coordinates (qform_code > 0: quaternion rotation, pixel sizes,
// qfac and offsets; qform_code = 0: a diagonal of the pixel sizes).  Voxel
// values are converted to float for the sampler; the raw header is kept so
// outputs carry the input's geometry, as the reference writes its outputs
// through the output-mask image (src/dualgpm.cpp:304-351).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace drb {
namespace nifti {

enum DataType : int16_t {
  DT_UINT8 = 2,
  DT_INT16 = 4,
  DT_INT32 = 8,
  DT_FLOAT32 = 16,
  DT_FLOAT64 = 64,
  DT_INT8 = 256,
  DT_UINT16 = 512,
  DT_UINT32 = 768,
  DT_INT64 = 1024,
  DT_UINT64 = 1280,
};

struct Image {
  std::string fname;
  unsigned char hdr[348];   // header as read (native byte order after reading)
  int dim[8] = {0};
  float pixdim[8] = {0};
  int16_t datatype = 0;
  int16_t qform_code = 0, sform_code = 0;
  float qto_xyz[16];        // row-major 4 x 4 (nifti_image::qto_xyz)
  std::vector<float> data;  // nx * ny * nz values, x fastest
  int nx() const { return dim[1]; }
  int ny() const { return dim[0] >= 2 ? dim[2] : 1; }
  int nz() const { return dim[0] >= 3 ? dim[3] : 1; }
  size_t nvox() const { return data.size(); }
  bool is_float() const { return datatype == DT_FLOAT32; }
  bool is_double() const { return datatype == DT_FLOAT64; }
};

// True if `path` names a readable NIfTI-1 dataset (header size 348 and a
// valid magic string), as is_nifti_file does for the reference's parser.
bool is_nifti_file(const std::string& path);

// Reads header and voxels; throws std::runtime_error on any problem.
// Only the first volume of a 4D image is read.
Image read(const std::string& path);

// Writes `values` (one per voxel of `geom`) with geom's header as a
// single-file dataset; gzipped when `path` ends in .gz.  Float32 or float64
// following geom's data type (float32 for any other type).
void write(const Image& geom, const std::vector<float>& values, const std::string& path);

// Largest absolute difference of two qform matrices <= tol
// (same_orientation, nifti_manipulation.inl:572-580).
bool same_orientation(const Image& a, const Image& b, float tol = 1e-4f);

}  // namespace nifti
}  // namespace drb
