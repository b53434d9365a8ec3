// Minimum-contrast summary of an image on the device
// (compute_mce_summary_data_impl, estimate_kernel_parameters.h:50-101).
//
// For every lattice offset p and every pair of voxels (x, x + p) inside the
// grid whose values are both non-zero and not NaN: the sums of x*y, x and y in
// double and the pair count.  The image (a few MB) stays in L2; a CTA takes a
// slab of x-rows and a chunk of offsets, walks the rows of the slab with the
// threads along x (coalesced loads of both rows of a pair), and reduces each
// offset's sums over the CTA.  A second kernel adds the slabs in a fixed order,
// so results do not depend on scheduling.
#pragma once

#include "common.cuh"

namespace drb {

constexpr int MCE_THREADS = 128;
constexpr int MCE_OFFSETS_PER_CTA = 32;

struct MceSums {
  double sxy, sx, sy;
  int n;
};

__device__ __forceinline__ bool mce_nonzero(float v) { return !(isnan(v) || v == 0.0f); }

__global__ void __launch_bounds__(MCE_THREADS) k_mce_partial(const float* __restrict__ img, int nx, int ny, int nz,
                                                            const int* __restrict__ P, int n_off, int rows_per_slab,
                                                            MceSums* __restrict__ part) {
  __shared__ double red[3][MCE_THREADS / 32];
  __shared__ int redn[MCE_THREADS / 32];
  const int slab = blockIdx.x;
  const int rows = ny * nz;
  const int r0 = slab * rows_per_slab, r1 = min(rows, r0 + rows_per_slab);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int o0 = blockIdx.y * MCE_OFFSETS_PER_CTA, o1 = min(n_off, o0 + MCE_OFFSETS_PER_CTA);
  for (int o = o0; o < o1; o++) {
    const int dx = P[3 * o], dy = P[3 * o + 1], dz = P[3 * o + 2];
    const int i0 = max(0, -dx), i1 = min(nx, nx - dx);
    double sxy = 0.0, sx = 0.0, sy = 0.0;
    int n = 0;
    for (int r = r0; r < r1; r++) {
      const int j = r % ny, k = r / ny;
      const int j2 = j + dy, k2 = k + dz;
      if (j2 < 0 || j2 >= ny || k2 < 0 || k2 >= nz) continue;  // uniform over the CTA
      const float* xr = img + (long long)r * nx;
      const float* yr = img + ((long long)k2 * ny + j2) * nx + dx;
      for (int i = i0 + threadIdx.x; i < i1; i += MCE_THREADS) {
        const float xv = __ldg(xr + i);
        if (!mce_nonzero(xv)) continue;
        const float yv = __ldg(yr + i);
        if (!mce_nonzero(yv)) continue;
        sxy += (double)xv * (double)yv;
        sx += (double)xv;
        sy += (double)yv;
        n++;
      }
    }
    for (int off = 16; off > 0; off >>= 1) {
      sxy += __shfl_xor_sync(0xffffffffu, sxy, off);
      sx += __shfl_xor_sync(0xffffffffu, sx, off);
      sy += __shfl_xor_sync(0xffffffffu, sy, off);
      n += __shfl_xor_sync(0xffffffffu, n, off);
    }
    if (lane == 0) {
      red[0][warp] = sxy;
      red[1][warp] = sx;
      red[2][warp] = sy;
      redn[warp] = n;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      MceSums s{0.0, 0.0, 0.0, 0};
      for (int w = 0; w < MCE_THREADS / 32; w++) {
        s.sxy += red[0][w];
        s.sx += red[1][w];
        s.sy += red[2][w];
        s.n += redn[w];
      }
      part[(long long)slab * n_off + o] = s;
    }
    __syncthreads();
  }
}

// Slab sums in order; covariance (sum_xy - sum_x sum_y / n) / (n - 1) for n > 1, else 0.
__global__ void k_mce_finish(const MceSums* __restrict__ part, int n_slabs, int n_off, float* covariance,
                             int* npairs, double* sums) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n_off) return;
  double sxy = 0.0, sx = 0.0, sy = 0.0;
  int n = 0;
  for (int s = 0; s < n_slabs; s++) {
    const MceSums& p = part[(long long)s * n_off + o];
    sxy += p.sxy;
    sx += p.sx;
    sy += p.sy;
    n += p.n;
  }
  npairs[o] = n;
  covariance[o] = n > 1 ? (float)((sxy - sx * sy / n) / (double)(n - 1)) : 0.0f;
  if (sums) {
    sums[3 * o] = sxy;
    sums[3 * o + 1] = sx;
    sums[3 * o + 2] = sy;
  }
}

}  // namespace drb
