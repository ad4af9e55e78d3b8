// Minimal NIfTI-1 reader/writer for the antsRegistration front end: scalar images and the
// vector displacement fields antsRegistration writes as prefix0Warp.nii.gz (5-D, intent vector,
// component planes), with gzip through zlib.  Geometry is kept in ITK's LPS convention
// (origin and direction); the file's RAS sform/qform are converted on the way in and out.
#pragma once

#include <string>
#include <vector>

namespace nifti {

struct Image {
  int dim = 3;                 // spatial dimension (2 or 3)
  int components = 1;          // 1 for scalar images, dim for displacement fields
  long long size[3] = {1, 1, 1};
  double spacing[3] = {1, 1, 1};
  double origin[3] = {0, 0, 0};     // LPS
  double direction[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};  // LPS, row-major
  std::vector<float> data;     // scalar: x fastest; vector: component planes (component slowest)
  int out_datatype = 16;       // NIfTI datatype write() stores (reading leaves it float32): 2 uchar,
                               // 4 int16, 8 int32, 16 float32, 64 float64, 256 int8
  bool time_series = false;    // a 4-D series: `components` volumes along dim[4] (stored like planes)
  double time_step = 1.0;      // pixdim[4] of a series
  long long voxels() const { return size[0] * size[1] * size[2]; }
};

// Throws std::runtime_error with a message on failure.
Image read(const std::string& path);
void write(const std::string& path, const Image& img);

}  // namespace nifti
