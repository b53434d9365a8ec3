// Kriging products on the 5th-generation tensor cores.
//
// W mu_D and W^T rs for all chains of a chain set are dense GEMMs once W is cut
// into tiles of 128 spatially adjacent rows: the union of a tile's columns is a
// few times its nonzero count (about 6x for W and 3x for W^T on a 32^3 volume
// at a 6.9 mm neighbourhood), so the tile is stored dense and multiplied on the
// tensor cores, D[128 x N] = A[128 x K] B[K x N] with N = chains (padded to a
// power of two >= 16).
//
// Precision: each FP32 operand is split as x = hi + lo (hi = the TF32 bits of
// x, lo = x - hi, exact), and D accumulates hi_A hi_B + hi_A lo_B + lo_A hi_B
// in FP32 (three kind::tf32 MMAs per K step), which keeps about 21 bits of
// every product -- the FP32 CSR products' accuracy, not TF32's.  The blob holds
// A in FP32 (16 KB per chunk); both splits are made in shared memory by the
// gather warps, A's while their B loads are in flight.
//
// k_tc_product: one CTA per SM over a contiguous range of chunks (32 columns
// of one tile).  Warp roles:
//   warp 0     one thread bulk-copies the chunk's A block (16 KB) into the
//              stage (mbarrier transaction count);
//   warp 1     allocates TMEM; one thread issues the MMAs of a chunk when both
//              its A and B are in, then commits the stage back to the
//              producers; at a tile boundary it commits the accumulator;
//   warps 2..  gather groups of 4 warps (three, or two with two stages, see
//              tc_groups), taking chunks in turn: the
//              chunk's chain vectors X[col][chain] are loaded (coalesced over
//              chains), all of a thread's loads before any is used -- or, for
//              W^T rs, taken from shared memory where warp 0's TMA row gathers
//              (tile::gather4) put them; meanwhile the landed A block is split
//              in place into hi and lo; then B is split and written as hi / lo
//              in the K-major layout, and the stage is handed to the MMA thread;
//   last 4     epilogue: TMEM -> registers -> the segment's partial slot.
// Every mbarrier wait is bounded; a wait that gives up records 3 in ch.err,
// the roles drain their copies and MMAs, and TMEM is released.
//
// k_tc_finish: one block per 16 rows of a tile sums the tile's segment
// partials in segment order (deterministic), then applies the epilogue as the
// CSR kernels k_spmv_w / k_spmv_wt do: rs = Ys - W mu_D with the ||rs||^2
// partials, or gD = sigma_h^-2 (Yh - mu_D) + sigma_s^-2 W^T rs with the
// ||Yh - mu_D||^2 partials (MultiResParameters.h:357-364).
#pragma once

#include <cuda.h>

#include "drb.h"
#include "umma.cuh"

namespace drb {

constexpr int TC_M = 128;               // tile rows (MMA M)
constexpr int TC_KC = 32;               // columns per chunk
constexpr int TC_BLK = TC_M * TC_KC;    // floats in one block (hi or lo) of a chunk
constexpr int TC_HDR = 4096;            // barriers, TMEM address, chain offsets

// Barrier of the nthreads threads (whole warps) that use barrier id, returning the AND of their v: every thread of
// the group reaches it once per chunk, so a wait that gave up in one warp ends the group's loop in all of them.
__device__ __forceinline__ bool group_all(bool v, int id, int nthreads) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id), "r"(nthreads)
      : "memory");
  return r != 0;
}

__host__ __device__ constexpr int tc_stages(int N) { return N <= 64 ? 4 : (N <= 128 ? 3 : 2); }
// Gather groups (chunks in flight in the gather): at most 3, and never more than the stages.  A group handles
// chunks G apart and waits for stage s by the parity of empty[s]'s phase; before that wait it has only seen the
// MMA of its previous chunk's stage complete (chunk q - G - S), so the phase before the awaited one (the MMA of
// chunk q - 2S) is certain to be complete only if G <= S.  With G > S the barrier can be two phases behind, the
// parity test then reports the preceding phase of the same parity as the awaited one, the group overwrites a
// stage whose MMA has not run, and fullB's 128-arrival phases mix two groups' arrivals, after which the MMA thread
// waits for a phase that never completes.
__host__ __device__ constexpr int tc_groups(int N) { return tc_stages(N) < 3 ? tc_stages(N) : 3; }
__host__ __device__ constexpr int tc_threads(int N) { return 32 * (2 + 4 * tc_groups(N) + 4); }
__host__ __device__ inline int tc_stage_bytes(int N) { return 2 * TC_BLK * 4 + 2 * N * TC_KC * 4; }
__host__ __device__ inline int tc_smem_bytes(int N) { return TC_HDR + tc_stages(N) * tc_stage_bytes(N); }

// mode 0: X = mu_D (each chain's accepted half xor sel), mode 1: X = rs.  N: chains, a power of two in [16, 256].
// TG: the chain vectors of a chunk's columns arrive by TMA row gathers (tile::gather4 over xmap, a 2D map of X with
// rows of Cp chains and a one-row box of N chains) issued by warp 0 into the stage's B blocks -- for mu_D both
// halves, half 0 into the hi block and half 1 into the lo block; padding columns fetch row 0, which meets zero
// columns of A -- and the gather groups only read them from shared memory.  Without TG the gather groups load them.
template <int N, bool TG>
__global__ void __launch_bounds__(tc_threads(N), 1)
    k_tc_product(DevTcMatrix A, DevChains ch, int n_h, int sel, int mode, float* __restrict__ partial,
                 const __grid_constant__ CUtensorMap xmap) {
  grid_dep_wait();
  extern __shared__ __align__(1024) unsigned char tsm[];
  uint64_t* fullA = reinterpret_cast<uint64_t*>(tsm);
  uint64_t* fullB = fullA + 4;
  uint64_t* empty = fullA + 8;
  uint64_t* accf = fullA + 12;
  uint64_t* acce = fullA + 13;
  uint64_t* done = fullA + 14;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tsm + 128);
  long long* xoff = reinterpret_cast<long long*>(tsm + 256);
  int* xhalf = reinterpret_cast<int*>(tsm + 2304);
  unsigned char* stage0 = tsm + TC_HDR;
  const int stages = tc_stages(N), sbytes = tc_stage_bytes(N);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int seg0 = A.cta_seg_ptr[blockIdx.x], seg1 = A.cta_seg_ptr[blockIdx.x + 1];
  const uint32_t ncols = N < 32 ? 32 : N;

  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; s++) {
      mbar_init(fullA + s, 1);
      mbar_init(fullB + s, 128);
      mbar_init(empty + s, 1);
    }
    mbar_init(accf, 1);
    mbar_init(acce, 128);
    mbar_init(done, 1);
    mbar_fence_init();
  }
  constexpr int G = tc_groups(N);
  for (int n = threadIdx.x; n < N; n += tc_threads(N)) {
    long long o = -1;
    int h = -1;
    if (n < ch.C) {
      h = mode == 0 ? (ch.st[n].acc ^ sel) : 0;
      o = (long long)h * n_h * ch.Cp + n;
    }
    xoff[n] = o;
    xhalf[n] = h;
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, ncols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool ok = true;

  if (warp == 0) {
    // the whole warp: lane 0 bulk-copies A, lanes 0-7 (and 8-15 for the second half of mu_D) gather 4 rows each.
    // A CTA's chunks are one contiguous range (its segments in order), and the column indices of the next chunk
    // are loaded while the current one is issued.
    const int halves = mode == 0 ? 2 : 1;
    const uint32_t xbytes = TG ? (uint32_t)halves * TC_KC * N * 4 : 0u;
    const int c_begin = seg0 < seg1 ? A.segs[seg0].y : 0, c_end = seg0 < seg1 ? A.segs[seg1 - 1].z : 0;
    int jn = 0;
    if constexpr (TG) {
      if (c_begin < c_end) jn = __ldg(A.chunk_cols + (long long)c_begin * TC_KC + lane);
    }
    int q = 0;
    for (int c = c_begin; c < c_end; c++, q++) {
      const int s = q % stages;
      int j = jn;
      if constexpr (TG) {
        if (c + 1 < c_end) jn = __ldg(A.chunk_cols + (long long)(c + 1) * TC_KC + lane);
        if (j < 0) j = 0;
      }
      if (!__all_sync(0xffffffffu, q < stages || mbar_wait_bounded(empty + s, ((q / stages) & 1) ^ 1))) {
        ok = false;
        break;
      }
      if (lane == 0) {
        mbar_arrive_expect_tx(fullA + s, TC_BLK * 4 + xbytes);
        bulk_g2s(stage0 + s * sbytes, A.blob + (long long)c * TC_BLK, TC_BLK * 4, fullA + s);
      }
      if constexpr (TG) {
        __syncwarp();
        const int h = lane >> 3, r4 = (lane & 7) * 4;
        const int y0 = __shfl_sync(0xffffffffu, j, r4), y1 = __shfl_sync(0xffffffffu, j, r4 + 1);
        const int y2 = __shfl_sync(0xffffffffu, j, r4 + 2), y3 = __shfl_sync(0xffffffffu, j, r4 + 3);
        if (h < halves) {
          const int ro = h * n_h;
          unsigned char* dst = stage0 + s * sbytes + 2 * TC_BLK * 4 + h * N * TC_KC * 4 + r4 * N * 4;
          tma_gather4(dst, &xmap, 0, y0 + ro, y1 + ro, y2 + ro, y3 + ro, fullA + s);
        }
      }
    }
    // the copies still in flight land before the CTA may exit
    if (lane == 0)
      for (int r = q - stages < 0 ? 0 : q - stages; r < q; r++) mbar_wait_bounded(fullA + r % stages, (r / stages) & 1);
    if (!ok && lane == 0) atomicExch(ch.err, 3);
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_tf32(TC_M, N);
      const uint32_t lbo_b = 16u * N;
      int q = 0;
      for (int g = seg0; g < seg1 && ok; g++) {
        const int4 sg = A.segs[g];
        if (g > seg0) {  // the epilogue has read the previous segment's accumulator
          if (!mbar_wait_bounded(acce, (g - seg0 - 1) & 1)) {
            ok = false;
            break;
          }
          tc_fence_after();
        }
        uint32_t accum = 0;
        for (int c = sg.y; c < sg.z; c++, q++) {
          const int s = q % stages;
          const uint32_t par = (q / stages) & 1;
          // the gather group arrives once A is split and B is written
          if (!mbar_wait_bounded(fullB + s, par)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a = smem_addr(stage0 + s * sbytes);
          const uint32_t b = a + 2 * TC_BLK * 4;
          const uint32_t bl = b + N * TC_KC * 4;
#pragma unroll
          for (int ks = 0; ks < TC_KC / 8; ks++) {
            // A block: element (m, k) at float (k/4)*512 + m*4 + k%4 -> K step ks starts 4096 B further;
            // LBO (next 4 k) 2048 B, SBO (next 8 rows) 128 B.  B block: (n, k) at (k/4)*4N + n*4 + k%4.
            const uint64_t ahi = sdesc_kmajor(a + ks * 4096, 2048, 128);
            const uint64_t alo = sdesc_kmajor(a + TC_BLK * 4 + ks * 4096, 2048, 128);
            const uint64_t bhi = sdesc_kmajor(b + ks * 32 * N, lbo_b, 128);
            const uint64_t blo = sdesc_kmajor(bl + ks * 32 * N, lbo_b, 128);
            umma_tf32(tmem, ahi, bhi, idesc, accum);
            umma_tf32(tmem, ahi, blo, idesc, 1u);
            umma_tf32(tmem, alo, bhi, idesc, 1u);
            accum = 1u;
          }
          umma_commit(empty + s);
        }
        if (!ok) break;
        umma_commit(accf);
      }
      umma_commit(done);
      mbar_wait_bounded(done, 0);
      if (!ok) atomicExch(ch.err, 3);
    }
  } else if (warp < 2 + 4 * G) {
    // Gather group grp takes chunks q = grp (mod G).  Each chunk waits only for MMAs of earlier chunks, so the
    // smallest chunk not yet handed over can always proceed; G <= stages keeps every parity wait within one phase
    // of its barrier (tc_groups).
    constexpr int NI = N * (TC_KC / 4) / 128;  // (chain, 4 columns) pairs per thread and chunk
    const int grp = (warp - 2) / 4, t = threadIdx.x - 64 - 128 * grp;
    const long long Cp = ch.Cp;
    const float* __restrict__ X = mode == 0 ? ch.muD : ch.rs;
    int q = 0;
    for (int g = seg0; g < seg1 && ok; g++) {
      const int4 sg = A.segs[g];
      for (int c = sg.y; c < sg.z; c++, q++) {
        if (q % G != grp) continue;
        const int s = q % stages;
        bool got = q < stages || mbar_wait_bounded(empty + s, ((q / stages) & 1) ^ 1);
        float4* bh = reinterpret_cast<float4*>(stage0 + s * sbytes + 2 * TC_BLK * 4);
        float4* bl = bh + N * (TC_KC / 4);
        float xv[NI][4];
        if constexpr (TG) {
          // A and the gathered rows have landed: row k of half h at float h * 32N + k * N of the B blocks
          got = got && mbar_wait_bounded(fullA + s, (q / stages) & 1);
          if (got) {
            const float* xs = reinterpret_cast<const float*>(bh);
#pragma unroll
            for (int i = 0; i < NI; i++) {
              const int idx = t + 128 * i;
              const int n = idx & (N - 1), kc4 = idx / N;
              const int h = xhalf[n];
              const float* r = xs + (h > 0 ? h : 0) * N * TC_KC + 4 * kc4 * N + n;
#pragma unroll
              for (int kk = 0; kk < 4; kk++) xv[i][kk] = h >= 0 ? r[kk * N] : 0.f;
            }
          }
          // every thread of the group has read the staged rows before the blocks are overwritten, and the group
          // goes on only if every thread's waits succeeded
          if (!group_all(got, 1 + grp, 128)) {
            ok = false;
            break;
          }
        } else {
          if (!got) {
            ok = false;
            break;
          }
          const int4* cols = reinterpret_cast<const int4*>(A.chunk_cols + (long long)c * TC_KC);
          // all of this thread's chain-vector loads are issued before any is used (coalesced over chains)
#pragma unroll
          for (int i = 0; i < NI; i++) {
            const int idx = t + 128 * i;
            const int n = idx & (N - 1), kc4 = idx / N;
            const long long o = xoff[n];
            const int4 j = __ldg(cols + kc4);
            const bool on = o >= 0;
            xv[i][0] = (on && j.x >= 0 && in_bounds(j.x, A.n_cols, ch.err)) ? __ldg(X + o + j.x * Cp) : 0.f;
            xv[i][1] = (on && j.y >= 0 && in_bounds(j.y, A.n_cols, ch.err)) ? __ldg(X + o + j.y * Cp) : 0.f;
            xv[i][2] = (on && j.z >= 0 && in_bounds(j.z, A.n_cols, ch.err)) ? __ldg(X + o + j.z * Cp) : 0.f;
            xv[i][3] = (on && j.w >= 0 && in_bounds(j.w, A.n_cols, ch.err)) ? __ldg(X + o + j.w * Cp) : 0.f;
          }
          // A: hi in place, lo into the second block, while the loads above are in flight
          if (!mbar_wait_bounded(fullA + s, (q / stages) & 1)) {
            ok = false;
            break;
          }
        }
        float4* ah = reinterpret_cast<float4*>(stage0 + s * sbytes);
        float4* al = ah + TC_BLK / 4;
#pragma unroll
        for (int i = 0; i < TC_BLK / 4 / 128; i++) {
          const float4 a = ah[t + 128 * i];
          const float4 h = make_float4(tf32_hi(a.x), tf32_hi(a.y), tf32_hi(a.z), tf32_hi(a.w));
          ah[t + 128 * i] = h;
          al[t + 128 * i] = make_float4(a.x - h.x, a.y - h.y, a.z - h.z, a.w - h.w);
        }
#pragma unroll
        for (int i = 0; i < NI; i++) {
          const int idx = t + 128 * i;
          const int n = idx & (N - 1), kc4 = idx / N;
          const float4 h = make_float4(tf32_hi(xv[i][0]), tf32_hi(xv[i][1]), tf32_hi(xv[i][2]), tf32_hi(xv[i][3]));
          bh[kc4 * N + n] = h;
          bl[kc4 * N + n] = make_float4(xv[i][0] - h.x, xv[i][1] - h.y, xv[i][2] - h.z, xv[i][3] - h.w);
        }
        fence_proxy_async_smem();
        mbar_arrive(fullB + s);
      }
    }
    if (!ok) atomicExch(ch.err, 3);
  } else {
    const int quarter = warp & 3;
    const int m = 32 * quarter + lane;
    for (int g = seg0; g < seg1; g++) {
      // the TMEM loads below are warp-collective: the warp goes on only if every lane saw the accumulator
      if (!__all_sync(0xffffffffu, mbar_wait_bounded(accf, (g - seg0) & 1))) {
        if (lane == 0) atomicExch(ch.err, 3);
        break;
      }
      tc_fence_after();
      float* P = partial + (long long)g * N * TC_M + m;
      for (int cb = 0; cb < N / 16; cb++) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(16 * cb), v);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; i++) P[(long long)(16 * cb + i) * TC_M] = v[i];
      }
      tc_fence_before();
      mbar_arrive(acce);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, ncols);
  }
}

// Sums the segment partials of TC_FR rows of one tile and applies the product's epilogue (mode 0: W, mode 1: W^T).
// Block (tile t, row group r) = blockIdx.x = t * (128 / TC_FR) + r; its per-chain squared-residual sums go to
// partial-sum slot blockIdx.x.  Phase 1 reads the partials coalesced along rows (all segment loads of a thread's
// elements in flight together) and sums them in segment order; phase 2 works along chains, so that mu_D, rs and
// gD are read and written coalesced.
constexpr int TC_FR = 16;  // tile rows per finishing block
__host__ __device__ inline int tc_finish_blocks(int T) { return T * (TC_M / TC_FR); }
__host__ __device__ inline int tc_finish_smem_bytes(int N) { return N * (TC_FR + 1) * 4 + 256 * 8; }

template <int N>
__global__ void __launch_bounds__(256) k_tc_finish(DevTcMatrix A, const float* __restrict__ partial, DevVolume v,
                                                   DevChains ch, int step, int sel, int chain_only, int mode) {
  grid_dep_wait();
  constexpr int EPT = N * TC_FR / 256;  // elements per thread (N >= 16)
  extern __shared__ __align__(16) unsigned char fsm[];
  float* S = reinterpret_cast<float*>(fsm);
  double* red = reinterpret_cast<double*>(fsm + (size_t)N * (TC_FR + 1) * 4);
  __shared__ int rows[TC_FR];
  const int t = blockIdx.x / (TC_M / TC_FR), m0 = (blockIdx.x % (TC_M / TC_FR)) * TC_FR;
  const int s0 = A.tile_seg_ptr[t], s1 = A.tile_seg_ptr[t + 1];
  if (threadIdx.x < TC_FR) {
    const int row = A.tile_rows[(long long)t * TC_M + m0 + threadIdx.x];
    rows[threadIdx.x] = (row < 0 || in_bounds(row, A.n_rows, ch.err)) ? row : -1;
  }
  {
    // element i of this thread: row m0 + mi, chain nb + 16 i (rows fastest across the warp); the segments are
    // summed in order, four segments' loads in flight at a time
    const int mi = threadIdx.x % TC_FR, nb = threadIdx.x / TC_FR;
    float acc[EPT];
#pragma unroll
    for (int i = 0; i < EPT; i++) acc[i] = 0.f;
    const long long seg = (long long)N * TC_M;
    const float* P = partial + (long long)s0 * seg + m0 + mi + (long long)nb * TC_M;
    int g = s0;
    for (; g + 3 < s1; g += 4, P += 4 * seg) {
      float x[4][EPT];
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int i = 0; i < EPT; i++) x[u][i] = __ldg(P + u * seg + (long long)(256 / TC_FR) * i * TC_M);
#pragma unroll
      for (int i = 0; i < EPT; i++) acc[i] = (((acc[i] + x[0][i]) + x[1][i]) + x[2][i]) + x[3][i];
    }
    for (; g < s1; g++, P += seg) {
#pragma unroll
      for (int i = 0; i < EPT; i++) acc[i] += __ldg(P + (long long)(256 / TC_FR) * i * TC_M);
    }
#pragma unroll
    for (int i = 0; i < EPT; i++) S[(nb + (256 / TC_FR) * i) * (TC_FR + 1) + mi] = acc[i];
  }
  __syncthreads();
  // element j of this thread: row r0 + dr j, chain n (chains fastest)
  const int n = threadIdx.x & (N - 1);
  const int r0 = threadIdx.x / N;
  constexpr int dr = 256 / N;
  bool act = n < ch.C && (chain_only < 0 || n == chain_only);
  if (act) act = step < 0 || step <= ch.st[n].L_cur;
  double sq = 0.0;
  if (act) {
    const long long Cp = ch.Cp;
    const float* Sn = S + n * (TC_FR + 1);
    if (mode == 0) {
      float y[EPT];
#pragma unroll
      for (int j = 0; j < EPT; j++) {
        const int row = rows[r0 + dr * j];
        y[j] = row >= 0 ? __ldg(v.Ys + row) : 0.f;
      }
#pragma unroll
      for (int j = 0; j < EPT; j++) {
        const int row = rows[r0 + dr * j];
        if (row < 0) continue;
        const float r = y[j] - Sn[r0 + dr * j];
        ch.rs[row * Cp + n] = r;
        sq += (double)r * r;
      }
    } else {
      const ChainState& st = ch.st[n];
      const float* mu = ch.muD + (long long)(st.acc ^ sel) * v.n_h * Cp + n;
      const float sh = st.sh, ss = st.ss;
      float y[EPT], mv[EPT];
#pragma unroll
      for (int j = 0; j < EPT; j++) {
        const int row = rows[r0 + dr * j];
        y[j] = row >= 0 ? __ldg(v.Yh + row) : 0.f;
        mv[j] = row >= 0 ? mu[row * Cp] : 0.f;
      }
#pragma unroll
      for (int j = 0; j < EPT; j++) {
        const int row = rows[r0 + dr * j];
        if (row < 0) continue;
        const float rh = y[j] - mv[j];
        ch.gD[row * Cp + n] = sh * rh + ss * Sn[r0 + dr * j];
        sq += (double)rh * rh;
      }
    }
  }
  red[threadIdx.x] = sq;
  __syncthreads();
  if ((int)threadIdx.x < N && act) {
    double s = 0.0;
    for (int k = 0; k < dr; k++) s += red[k * N + n];
    const int L = ch.st[n].L_cur;
    const int slot = mode == 0 ? (step <= 0 ? SL_RS0 : (step == L ? SL_RSL : SL_SCRATCH))
                               : (step <= 0 ? SL_RH0 : (step == L ? SL_RHL : SL_SCRATCH));
    ch.part[((long long)n * NSLOT + slot) * ch.maxblk + blockIdx.x] = s;
  }
}

// Scatters the CSR values into the dense blob (zeroed first): value k at dest[k].
__global__ void k_tc_fill(const float* __restrict__ val, const int* __restrict__ dest, int nnz, float* __restrict__ blob) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nnz) blob[dest[k]] = val[k];
}

}  // namespace drb
