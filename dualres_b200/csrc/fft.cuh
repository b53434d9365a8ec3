// Shared-memory Stockham FFT for power-of-two lengths 2..512.
//
// A tile of `nlines` independent lines sits in shared memory; element i of
// line l lives at sm[l * ls + i * es].  Each stage of radix R splits every
// sub-array of the current length M into R sub-arrays of length M/R (Stockham
// autosort: the output is in natural order, no bit reversal pass).  Within a
// stage every thread holds its butterflies in registers: all threads read,
// the block synchronises, then all threads write back in place.
//
// Thread mapping is line-fastest: consecutive threads work on consecutive
// lines.  With an element-major layout (ls = 1) or a line-major layout whose
// pitch is odd in complex units, the shared-memory accesses of a warp are
// bank-conflict free.
//
// Sign convention: forward = exp(-2 pi i jk/n), inverse = exp(+2 pi i jk/n),
// both unnormalised (the FFTW convention used by sized_fft.h:138-214 of the
// reference).
#pragma once

#include "common.cuh"

namespace drb {

// cos / sin of 2 pi k / 16 (exact constants of the 16th roots of unity).
template <class R>
__device__ __forceinline__ void cs16(int k, R& c, R& s) {
  const R a = (R)0.92387953251128675613, b = (R)0.38268343236508977173, h = (R)0.70710678118654752440;
  switch (k & 15) {
    case 0: c = 1; s = 0; break;
    case 1: c = a; s = b; break;
    case 2: c = h; s = h; break;
    case 3: c = b; s = a; break;
    case 4: c = 0; s = 1; break;
    case 5: c = -b; s = a; break;
    case 6: c = -h; s = h; break;
    case 7: c = -a; s = b; break;
    case 8: c = -1; s = 0; break;
    case 9: c = -a; s = -b; break;
    case 10: c = -h; s = -h; break;
    case 11: c = -b; s = -a; break;
    case 12: c = 0; s = -1; break;
    case 13: c = b; s = -a; break;
    case 14: c = h; s = -h; break;
    default: c = a; s = -b; break;
  }
}

// v * exp(DIR * 2 pi i k / 16), DIR = -1 forward, +1 inverse.
template <int DIR, class C>
__device__ __forceinline__ C mul_w16(C v, int k) {
  k &= 15;
  if (k == 0) return v;
  if (k == 8) return mk(-v.x, -v.y);
  if (k == 4) return DIR < 0 ? mk(v.y, -v.x) : mk(-v.y, v.x);
  if (k == 12) return DIR < 0 ? mk(-v.y, v.x) : mk(v.y, -v.x);
  decltype(v.x) c, s;
  cs16(k, c, s);
  if (DIR < 0) s = -s;
  return mk(v.x * c - v.y * s, v.x * s + v.y * c);
}

template <int R>
__host__ __device__ constexpr int brev_const(int i) {
  int r = 0;
  for (int b = 1; b < R; b <<= 1) {
    r = (r << 1) | (i & 1);
    i >>= 1;
  }
  return r;
}

// In-register DFT of R (2..16) points, radix-2 decimation in time.
template <int R, int DIR, class C>
__device__ __forceinline__ void reg_fft(C* a) {
#pragma unroll
  for (int i = 0; i < R; i++) {
    const int j = brev_const<R>(i);
    if (i < j) {
      C t = a[i];
      a[i] = a[j];
      a[j] = t;
    }
  }
#pragma unroll
  for (int len = 2; len <= R; len <<= 1) {
#pragma unroll
    for (int i = 0; i < R; i += len) {
#pragma unroll
      for (int k = 0; k < len / 2; k++) {
        const C u = a[i + k];
        const C v = mul_w16<DIR>(a[i + k + len / 2], k * (16 / len));
        a[i + k] = u + v;
        a[i + k + len / 2] = u - v;
      }
    }
  }
}

// One Stockham stage. N: length; R: radix; P: product of earlier radices.
// MAXB: butterflies per thread upper bound (>= ceil(N/R * nlines / nthr)).
// tw: forward twiddles exp(-2 pi i m / N), m < N.
template <int N, int R, int P, int DIR, int MAXB, class C>
__device__ __forceinline__ void fft_stage(C* sm, int ls, int es, int nlines, const C* __restrict__ tw, int tid,
                                          int nthr) {
  constexpr int M = N / P, Mn = M / R, NB = N / R;
  const int total = NB * nlines;
  C x[MAXB][R];
#pragma unroll
  for (int bb = 0; bb < MAXB; bb++) {
    const int w = tid + bb * nthr;
    if (w < total) {
      const int line = w % nlines, b = w / nlines;
      const int p = b / Mn, t = b % Mn;
      const C* base = sm + line * ls;
#pragma unroll
      for (int j = 0; j < R; j++) x[bb][j] = base[(p * M + t + Mn * j) * es];
      reg_fft<R, DIR>(x[bb]);
      if (Mn > 1) {
#pragma unroll
        for (int k = 1; k < R; k++) {
          C wv = tw[P * t * k];
          if (DIR > 0) wv.y = -wv.y;
          x[bb][k] = cmul(x[bb][k], wv);
        }
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int bb = 0; bb < MAXB; bb++) {
    const int w = tid + bb * nthr;
    if (w < total) {
      const int line = w % nlines, b = w / nlines;
      const int p = b / Mn, t = b % Mn;
      C* base = sm + line * ls;
#pragma unroll
      for (int k = 0; k < R; k++) base[((p + P * k) * Mn + t) * es] = x[bb][k];
    }
  }
  __syncthreads();
}

constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }

// Full FFT of nlines lines of length N held in shared memory.  MAXLINES and
// NTHR bound the per-thread butterfly count at compile time.  The caller must
// have synchronised after filling the tile; on return the tile is complete.
template <int N, int DIR, int MAXLINES, int NTHR, class C>
__device__ __forceinline__ void fft_smem(C* sm, int ls, int es, int nlines, const C* __restrict__ tw) {
  const int tid = threadIdx.x;
  if constexpr (N == 1) {
    return;
  } else if constexpr (N <= 16) {
    fft_stage<N, N, 1, DIR, cdiv(MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
  } else if constexpr (N == 32) {
    fft_stage<32, 8, 1, DIR, cdiv(4 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
    fft_stage<32, 4, 8, DIR, cdiv(8 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
  } else if constexpr (N == 64) {
    fft_stage<64, 8, 1, DIR, cdiv(8 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
    fft_stage<64, 8, 8, DIR, cdiv(8 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
  } else if constexpr (N == 128) {
    fft_stage<128, 16, 1, DIR, cdiv(8 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
    fft_stage<128, 8, 16, DIR, cdiv(16 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
  } else if constexpr (N == 256) {
    fft_stage<256, 16, 1, DIR, cdiv(16 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
    fft_stage<256, 16, 16, DIR, cdiv(16 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
  } else if constexpr (N == 512) {
    fft_stage<512, 8, 1, DIR, cdiv(64 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
    fft_stage<512, 8, 8, DIR, cdiv(64 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
    fft_stage<512, 8, 64, DIR, cdiv(64 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
  }
}

// Offset of the twiddle table for length N in the concatenated table
// (lengths 2, 4, ..., 512; entry m of length N is exp(-2 pi i m / N)).
__host__ __device__ constexpr int tw_offset(int N) { return N - 2; }
constexpr int TW_TOTAL = 1022;

}  // namespace drb
