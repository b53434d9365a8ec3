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

// Warp-synchronous Stockham stage: lane `b` of the line's lane group owns
// butterfly b (lanes with b >= N/R idle).  A line never leaves its warp, so
// the read / write phases need only __syncwarp.
template <int N, int R, int P, int DIR, class C>
__device__ __forceinline__ void warp_stage(C* L, int es, int b, bool on, const C* __restrict__ tw) {
  constexpr int M = N / P, Mn = M / R, NB = N / R;
  const bool act = on && b < NB;
  const int p = b / Mn, t = b % Mn;
  C x[R];
  if (act) {
#pragma unroll
    for (int j = 0; j < R; j++) x[j] = L[(p * M + t + Mn * j) * es];
    reg_fft<R, DIR>(x);
    if (Mn > 1) {
#pragma unroll
      for (int k = 1; k < R; k++) {
        C wv = tw[P * t * k];
        if (DIR > 0) wv.y = -wv.y;
        x[k] = cmul(x[k], wv);
      }
    }
  }
  __syncwarp();
  if (act) {
#pragma unroll
    for (int k = 0; k < R; k++) L[((p + P * k) * Mn + t) * es] = x[k];
  }
  __syncwarp();
}

// Largest butterfly count per line over the stages of the plan for N.
template <int N>
__host__ __device__ constexpr int plan_nbmax() {
  return N <= 16 ? 1 : (N == 32 ? 8 : (N == 64 ? 8 : (N == 128 ? 16 : 16)));
}

// Warp-synchronous FFT of nlines lines (N <= 256): each warp takes groups of
// 32 / nbmax lines; every stage runs with warp-level synchronisation only.
// The block synchronises once at the end, so the tile is complete on return.
template <int N, int DIR, class C>
__device__ __forceinline__ void fft_smem_warp(C* sm, int ls, int es, int nlines, const C* __restrict__ tw) {
  constexpr int NBM = plan_nbmax<N>(), LPW = 32 / NBM;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int li = lane / NBM, b = lane % NBM;
  for (int base = warp * LPW; base < nlines; base += nw * LPW) {
    const int line = base + li;
    const bool on = li < LPW && line < nlines;
    C* L = sm + (on ? line : 0) * ls;
    if constexpr (N <= 16) {
      warp_stage<N, N, 1, DIR, C>(L, es, b, on, tw);
    } else if constexpr (N == 32) {
      warp_stage<32, 8, 1, DIR, C>(L, es, b, on, tw);
      warp_stage<32, 4, 8, DIR, C>(L, es, b, on, tw);
    } else if constexpr (N == 64) {
      warp_stage<64, 8, 1, DIR, C>(L, es, b, on, tw);
      warp_stage<64, 8, 8, DIR, C>(L, es, b, on, tw);
    } else if constexpr (N == 128) {
      warp_stage<128, 16, 1, DIR, C>(L, es, b, on, tw);
      warp_stage<128, 8, 16, DIR, C>(L, es, b, on, tw);
    } else {
      warp_stage<256, 16, 1, DIR, C>(L, es, b, on, tw);
      warp_stage<256, 16, 16, DIR, C>(L, es, b, on, tw);
    }
  }
  __syncthreads();
}

// Full FFT of nlines lines of length N held in shared memory.  MAXLINES and
// NTHR bound the per-thread butterfly count at compile time.  The caller must
// have synchronised after filling the tile; on return the tile is complete.
// PLAN picks the radix plan for N = 64, 128 and 256: 0 (8 x 8, 16 x 8,
// 16 x 16) or 1 (16 x 4, 8 x 16, 8 x 8 x 4); a chain set's tuner times both.
template <int N, int DIR, int MAXLINES, int NTHR, class C, int PLAN = 0>
__device__ __forceinline__ void fft_smem(C* sm, int ls, int es, int nlines, const C* __restrict__ tw) {
  const int tid = threadIdx.x;
  if constexpr (N == 1) {
    return;
  } else if constexpr (N <= 16) {
    fft_stage<N, N, 1, DIR, cdiv(MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
  } else if constexpr (N == 32) {
    fft_stage<32, 8, 1, DIR, cdiv(4 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
    fft_stage<32, 4, 8, DIR, cdiv(8 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
  } else if constexpr (N == 64 && PLAN == 1) {
    fft_stage<64, 16, 1, DIR, cdiv(4 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
    fft_stage<64, 4, 16, DIR, cdiv(16 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
  } else if constexpr (N == 64) {
    fft_stage<64, 8, 1, DIR, cdiv(8 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
    fft_stage<64, 8, 8, DIR, cdiv(8 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
  } else if constexpr (N == 128 && PLAN == 1) {
    fft_stage<128, 8, 1, DIR, cdiv(16 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
    fft_stage<128, 16, 8, DIR, cdiv(8 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
  } else if constexpr (N == 128) {
    fft_stage<128, 16, 1, DIR, cdiv(8 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
    fft_stage<128, 8, 16, DIR, cdiv(16 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
  } else if constexpr (N == 256 && PLAN == 1) {
    fft_stage<256, 8, 1, DIR, cdiv(32 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
    fft_stage<256, 8, 8, DIR, cdiv(32 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
    fft_stage<256, 4, 64, DIR, cdiv(64 * MAXLINES, NTHR), C>(sm, ls, es, nlines, tw, tid, NTHR);
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

// ----------------------------------------------------------------- padded 2D planes
// An E x E plane stored with one pad slot after every 8 elements along both
// axes: phys(y, x) = (y + y/8) * RP + x + x/8, with the row pitch RP = 8 mod 16
// (complex units).  With the lane mappings below, every shared-memory access
// of the two radix stages (including the stride-8 transpose between them) hits
// 16 distinct 8-byte bank pairs per half-warp.
template <int E>
struct PaddedPlane {
  static constexpr int RP = (E + E / 8) + ((8 - (E + E / 8) % 16) + 16) % 16;  // >= E + E/8, = 8 mod 16
  static constexpr int ROWS = E + E / 8;
  static constexpr int SIZE = ROWS * RP;                       // complex elements
  __device__ __forceinline__ static int phys(int y, int x) { return (y + (y >> 3)) * RP + x + (x >> 3); }
};

// Two-stage plan (radices R1 then R2) of one line, with the line's element i at
// sm[idx(i)].  LINE_FAST = false: lane = li * NBM + b (rows); true: lane =
// li + 8 * bb, each lane owning butterflies bb, bb + 4, ... (columns).
template <int N, int R1, int R2>
struct Plan2 {
  static constexpr int NB1 = N / R1, NB2 = N / R2;
  static constexpr int NBM = NB1 > NB2 ? NB1 : NB2;
};

// Line elements at or beyond rlim are read as zero (they are never loaded), and elements at or beyond wlim are not
// written (nothing reads them): the pruned input of the first stage and the pruned output of the last.
// at(pp) is the address of padded position pp = i + i / 8 of the line.  Where a butterfly's element offsets are
// multiples of 8, or its first element is, the padded positions are the first one's plus constants
// (pad(i0 + o) = pad(i0) + o + o / 8), so one position per butterfly is computed and the rest are immediates.
__device__ __forceinline__ constexpr int plane_pad(int i) { return i + (i >> 3); }
// Between the read and write phases of a stage: __syncwarp when one warp owns its lines (bar = 0), else named barrier
// `bar` over the two warps that share them.
__device__ __forceinline__ void line_sync(int bar) {
  if (bar == 0) __syncwarp();
  else asm volatile("bar.sync %0, 64;" ::"r"(bar) : "memory");
}
template <int N, int R, int P, int DIR, int PER_LANE, class At>
__device__ __forceinline__ void plane_stage(float2* sm, At at, const int (&bl)[PER_LANE], bool on,
                                            const float2* __restrict__ tw, int rlim = N, int wlim = N, int bar = 0) {
  constexpr int M = N / P, Mn = M / R, NB = N / R;
  constexpr bool LIN_IN = (Mn % 8 == 0) || (Mn == 1 && M % 8 == 0);
  constexpr bool LIN_OUT = ((P * Mn) % 8 == 0) || (Mn == 1 && P == 1);
  float2 x[PER_LANE][R];
#pragma unroll
  for (int q = 0; q < PER_LANE; q++) {
    const int b = bl[q];
    if (on && b < NB) {
      const int p = b / Mn, t = b % Mn;
      const int i0 = p * M + t, pp0 = plane_pad(i0);
#pragma unroll
      for (int j = 0; j < R; j++) {
        const int i = i0 + Mn * j;
        const int pp = LIN_IN ? pp0 + Mn * j + ((Mn * j) >> 3) : plane_pad(i);
        x[q][j] = i < rlim ? sm[at(pp)] : make_float2(0.f, 0.f);
      }
      reg_fft<R, DIR>(x[q]);
      if (Mn > 1) {
#pragma unroll
        for (int k = 1; k < R; k++) {
          float2 wv = tw[P * t * k];
          if (DIR > 0) wv.y = -wv.y;
          x[q][k] = cmul(x[q][k], wv);
        }
      }
    }
  }
  line_sync(bar);
#pragma unroll
  for (int q = 0; q < PER_LANE; q++) {
    const int b = bl[q];
    if (on && b < NB) {
      const int p = b / Mn, t = b % Mn;
      const int o0 = p * Mn + t, po0 = plane_pad(o0);
#pragma unroll
      for (int k = 0; k < R; k++) {
        const int i = o0 + P * Mn * k;
        const int pp = LIN_OUT ? po0 + P * Mn * k + ((P * Mn * k) >> 3) : plane_pad(i);
        if (i < wlim) sm[at(pp)] = x[q][k];
      }
    }
  }
  line_sync(bar);
}

// Row FFTs (lines = y rows, elements along x) of a padded plane, all E rows; x >= rlim read as zero, x >= wlim not
// written.
template <int E, int R1, int R2, int DIR>
__device__ __forceinline__ void plane_rows(float2* sm, const float2* __restrict__ tw, int rlim = E, int wlim = E) {
  using PL = PaddedPlane<E>;
  constexpr int NBM = Plan2<E, R1, R2>::NBM, LPW = 32 / NBM;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int li = lane / NBM;
  const int bl[1] = {lane % NBM};
  for (int base = warp * LPW; base < E; base += nw * LPW) {
    const int y = base + li;
    const bool on = li < LPW && y < E;
    const int row = on ? (y + (y >> 3)) * PL::RP : 0;
    auto at = [row](int pp) { return row + pp; };
    plane_stage<E, R1, 1, DIR, 1>(sm, at, bl, on, tw, rlim, E);
    plane_stage<E, R2, R1, DIR, 1>(sm, at, bl, on, tw, E, wlim);
  }
  __syncthreads();
}

// Column FFTs (lines = x columns, elements along y) of the first ncols columns; y >= rlim read as zero, y >= wlim
// not written.
template <int E, int R1, int R2, int DIR>
__device__ __forceinline__ void plane_cols(float2* sm, int ncols, const float2* __restrict__ tw, int rlim = E,
                                           int wlim = E) {
  using PL = PaddedPlane<E>;
  constexpr int NBM = Plan2<E, R1, R2>::NBM, PL_LANE = NBM / 4;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int li = lane & 7, bb = lane >> 3;
  if constexpr (PL_LANE % 2 == 0) {
    // At most half as many 8-column groups as warps (a pruned box): the two warps of a pair split each column's
    // butterflies instead of half the warps idling, and the pair synchronises its stages on named barrier 1 + pair.
    if (2 * ((ncols + 7) / 8) <= nw && nw % 2 == 0 && nw <= 30) {
      constexpr int H = PL_LANE / 2;
      const int pair = warp >> 1, half = warp & 1;
      int bh[H];
#pragma unroll
      for (int q = 0; q < H; q++) bh[q] = bb + 4 * (half * H + q);
      for (int base = pair * 8; base < ncols; base += (nw / 2) * 8) {
        const int x = base + li;
        const bool on = x < ncols;
        const int col = on ? x + (x >> 3) : 0;
        auto at = [col](int pp) { return pp * PL::RP + col; };
        plane_stage<E, R1, 1, DIR, H>(sm, at, bh, on, tw, rlim, E, 1 + pair);
        plane_stage<E, R2, R1, DIR, H>(sm, at, bh, on, tw, E, wlim, 1 + pair);
      }
      __syncthreads();
      return;
    }
  }
  int bl[PL_LANE];
#pragma unroll
  for (int q = 0; q < PL_LANE; q++) bl[q] = bb + 4 * q;
  for (int base = warp * 8; base < ncols; base += nw * 8) {
    const int x = base + li;
    const bool on = x < ncols;
    const int col = on ? x + (x >> 3) : 0;
    auto at = [col](int pp) { return pp * PL::RP + col; };
    plane_stage<E, R1, 1, DIR, PL_LANE>(sm, at, bl, on, tw, rlim, E);
    plane_stage<E, R2, R1, DIR, PL_LANE>(sm, at, bl, on, tw, E, wlim);
  }
  __syncthreads();
}

}  // namespace drb
