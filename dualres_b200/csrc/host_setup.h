// One-time host set-up of a volume: masks, indices and the kriging matrix.
#pragma once

#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "../../include/dualres_b200.h"

namespace drb {

// Allocator whose value-less construction leaves the elements uninitialised: large buffers that are written in
// full right after allocation (in parallel) skip a serial zero-fill of hundreds of MB on scanner-sized volumes.
template <class T>
struct uninit_allocator : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = uninit_allocator<U>;
  };
  uninit_allocator() = default;
  template <class U>
  uninit_allocator(const uninit_allocator<U>&) noexcept {}
  template <class U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
};
template <class T>
using fill_vector = std::vector<T, uninit_allocator<T>>;

// The part of the kriging build that fixes the sparsity (kriging_matrix.h:148-299)
// and the covariances the per-row solves need.
struct KrigingPlan {
  int m = 0;                   // neighbourhood offsets
  int nrows = 0;               // std-res data voxels
  std::vector<double> K;       // m x m covariance of the offsets (unit diagonal)
  std::vector<double> S;       // K^-1, empty when K is not positive definite (or not computed yet)
  bool inverse_wanted = true;  // the Schur route is allowed (DRB_KRIGING_DIRECT unset)
  std::vector<int> row_start;  // nrows + 1, into pid / col / kp
  fill_vector<int> pid;        // offset id of each present neighbour
  fill_vector<int> col;        // its high-res data ordinal (the CSR column)
  fill_vector<double> kp;      // its covariance with the std-res voxel centre
};

// A row with cnt of m neighbours present solves through the Schur complement of
// S when that is cheaper than a direct solve.
inline bool kriging_schur_route(int cnt, int m, bool have_inv) {
  const double nb = (double)(m - cnt), c = (double)cnt;
  return have_inv && nb * nb * nb / 3.0 + c * c < c * c * c / 3.0;
}

struct HostVolume {
  int g[3] = {0, 0, 0};       // grid of the data voxels (max ijk + 1)
  int E[3] = {0, 0, 0};       // embedding
  long long N = 0;
  int box[3] = {0, 0, 0};     // box covering data + output voxels
  std::vector<int> d_flat, o_flat;   // flat embedding indices
  std::vector<int> box_to_d, box_to_o;
  std::vector<float> Yh, Ys;
  std::vector<int> w_rowptr, wt_rowptr;
  fill_vector<int> w_col, wt_col;
  fill_vector<float> w_val, wt_val;
  float Q[16];
  double theta[3];
  int covfun = 0;
  float radius = 0.f;
  double kriging_seconds = 0.0;
  double kriging_plan_seconds = 0.0;
  double kriging_solve_seconds = 0.0;
  int n_offsets = 0;
  KrigingPlan kplan;           // kept until the weights are solved
  bool kriging_pending = false;
  int kriging_device_rows = 0;  // rows solved on the device
  int kriging_host_rows = 0;    // rows the device left to the host (not positive definite)
};

// Returns DR_OK or a DR_ERR_* code with a message in *err.  With defer_kriging
// the kriging weights are left to the device (hv->kriging_pending, hv->kplan).
int host_prepare(const dr_volume_desc* d, HostVolume* hv, std::string* err, bool defer_kriging = false);

// W^T from W (rows ordered by data voxel, columns ascending).
void build_transpose(HostVolume* hv);

// host_inverse = false leaves K^-1 to the caller (the device solve computes it).
int kriging_plan(const float* hr, int nx, int ny, int nz, const float* Qhr, const float* sr, int sx, int sy, int sz,
                 const float* Qsr, const float* theta, float radius, KrigingPlan* plan, int* n_offsets,
                 std::string* err, bool host_inverse = true);
void kriging_solve_host(const KrigingPlan& plan, std::vector<int>* rowptr, fill_vector<int>* col,
                        fill_vector<float>* val);
// One row by the host route (Schur or Cholesky, QR if not positive definite);
// false when its weight sum is NaN.
bool kriging_solve_row_host(const KrigingPlan& plan, int ri, std::vector<double>* x);
// CSR from per-candidate weights; rows with keep = 0 are emptied (NaN weight sums).
void kriging_assemble(const KrigingPlan& plan, const double* w, const std::vector<char>& keep,
                      std::vector<int>* rowptr, fill_vector<int>* col, fill_vector<float>* val);

// Kriging CSR of kriging_matrix.h:148-343 (exposed for tests through the volume).
int kriging_build(const float* hr, int nx, int ny, int nz, const float* Qhr, const float* sr, int sx, int sy, int sz,
                  const float* Qsr, const float* theta, float radius, std::vector<int>* rowptr, std::vector<int>* col,
                  std::vector<float>* val, int* n_offsets, std::string* err);

// Host part of a dense-tile plan for the tensor-core kriging products: rows
// ordered along the Z-order curve of their keys (3 x 10-bit coordinates) and
// cut into tiles of 128; the sorted union of each tile's columns cut into
// chunks of 32; dest[k] = the blob position of nonzero k (element (m, kk) of
// chunk q at q * 4096 + (kk / 4) * 512 + m * 4 + kk % 4).  The chunks are split into at most
// g_max equal ranges, one per CTA, and the ranges at tile boundaries into
// segments {tile, first chunk, end chunk, 0}, ordered by chunk.
struct TcPlanHost {
  int T = 0, G = 0;
  long long chunks = 0;
  std::vector<int> tile_rows, chunk_cols, segs, cta_seg_ptr, tile_seg_ptr;
  fill_vector<int> dest;  // every entry is written by the plan
};
// false when the blob would not be addressable with 32-bit positions.
bool tc_plan(const std::vector<int>& rowptr, const int* col, size_t nnz, const std::vector<uint32_t>& key, int g_max,
             TcPlanHost* P);
// Z-order key of integer voxel coordinates (10 bits each).
uint32_t zorder_key(int x, int y, int z);

}  // namespace drb
