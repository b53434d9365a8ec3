// One-time host set-up of a volume: masks, indices and the kriging matrix.
#pragma once

#include <string>
#include <vector>

#include "../../include/dualres_b200.h"

namespace drb {

struct HostVolume {
  int g[3] = {0, 0, 0};       // grid of the data voxels (max ijk + 1)
  int E[3] = {0, 0, 0};       // embedding
  long long N = 0;
  int box[3] = {0, 0, 0};     // box covering data + output voxels
  std::vector<int> d_flat, o_flat;   // flat embedding indices
  std::vector<int> box_to_d, box_to_o;
  std::vector<float> Yh, Ys;
  std::vector<int> w_rowptr, w_col;
  std::vector<float> w_val;
  std::vector<int> wt_rowptr, wt_col;
  std::vector<float> wt_val;
  float Q[16];
  double theta[3];
  int covfun = 0;
  float radius = 0.f;
  double kriging_seconds = 0.0;
  int n_offsets = 0;
};

// Returns DR_OK or a DR_ERR_* code with a message in *err.
int host_prepare(const dr_volume_desc* d, HostVolume* hv, std::string* err);

// Kriging CSR of kriging_matrix.h:148-343 (exposed for tests through the volume).
int kriging_build(const float* hr, int nx, int ny, int nz, const float* Qhr, const float* sr, int sx, int sy, int sz,
                  const float* Qsr, const float* theta, float radius, std::vector<int>* rowptr, std::vector<int>* col,
                  std::vector<float>* val, int* n_offsets, std::string* err);

}  // namespace drb
