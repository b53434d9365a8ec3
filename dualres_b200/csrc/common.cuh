// Shared device helpers: complex arithmetic, counter-based RNG, reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace drb {

// ---------------------------------------------------------------- complex
template <class R> struct cplx_of;
template <> struct cplx_of<float> { using type = float2; };
template <> struct cplx_of<double> { using type = double2; };

__host__ __device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }
__host__ __device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// ---------------------------------------------------------------- RNG
// Philox4x32-10: J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11.  Counter-based, so
// every draw is a pure function of (seed, counter) and no state is stored.
struct u32x4 { uint32_t x, y, z, w; };

__host__ __device__ __forceinline__ uint32_t mulhilo32(uint32_t a, uint32_t b, uint32_t* hi) {
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  return (uint32_t)p;
}

__host__ __device__ __forceinline__ u32x4 philox(u32x4 c, uint64_t key) {
  uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t hi0, hi1;
    const uint32_t lo0 = mulhilo32(0xD2511F53u, c.x, &hi0);
    const uint32_t lo1 = mulhilo32(0xCD9E8D57u, c.z, &hi1);
    c = u32x4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// Stream identifiers (counter word w).
enum : uint32_t {
  RNG_MOMENTUM = 1u,   // x = mode pair, y = iteration, z = chain
  RNG_INIT_MU = 2u,    // x = mode pair, y = 0, z = chain
  RNG_SCALAR = 3u,     // x = sub-stream, y = iteration, z = chain
  RNG_INIT_SIGMA = 4u, // x = sub-stream, y = 0, z = chain
};

// Uniform in (0, 1), 24-bit float.
__host__ __device__ __forceinline__ float u01f(uint32_t v) { return ((float)(v >> 8) + 0.5f) * (1.0f / 16777216.0f); }
// Uniform in (0, 1), 53-bit double from two words.
__host__ __device__ __forceinline__ double u01d(uint32_t a, uint32_t b) {
  const uint64_t m = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
  return ((double)m + 0.5) * (1.0 / 9007199254740992.0);
}

// Box-Muller: two standard normals from two uniforms.
__device__ __forceinline__ float2 box_muller(float u1, float u2) {
  const float r = sqrtf(-2.0f * logf(u1));
  float s, c;
  sincospif(2.0f * u2, &s, &c);
  return make_float2(r * c, r * s);
}
__device__ __forceinline__ double2 box_muller_d(double u1, double u2) {
  const double r = sqrt(-2.0 * log(u1));
  double s, c;
  sincospi(2.0 * u2, &s, &c);
  return make_double2(r * c, r * s);
}

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum of per-thread doubles (fixed tree).  `scratch`
// needs blockDim.x / 32 doubles.  The result is valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < nw; i++) s += scratch[i];
  return s;
}

// ---------------------------------------------------------------- bounds checks
// Builds with DRB_BOUNDS_CHECK (the checked library, a debug build that stands in for a memory checker) test every
// data-dependent index before its access: an index outside [0, n) records 4 in the error word (when one is given)
// and the caller skips the access, so the kernel neither faults nor reads out of range, and the host reports the
// failure after the launch.  In other builds the test is a constant true and costs nothing.
constexpr int ERR_BOUNDS = 4;
__device__ __forceinline__ bool in_bounds(long long i, long long n, int* err) {
#ifdef DRB_BOUNDS_CHECK
  if (i >= 0 && i < n) return true;
  if (err) atomicExch(err, ERR_BOUNDS);
  return false;
#else
  (void)i;
  (void)n;
  (void)err;
  return true;
#endif
}

// Waits until the grid this one depends on (programmatic dependent launch) has completed and its memory is
// visible; returns at once when the kernel was launched without that dependency.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

}  // namespace drb
