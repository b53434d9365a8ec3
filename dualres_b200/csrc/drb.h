// Internal device-side data structures of the sampler (not part of the ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace drb {

// Largest FFT length per axis handled by the shared-memory kernels.
constexpr int MAX_AXIS = 512;
// Lines per tile in the pass kernels.
constexpr int TILE_LINES = 32;

// Slots of the per-block partial sums (double) that feed the accept step.
enum Slot : int {
  SL_E0 = 0,   // sum |w|^2 over all modes (momentum draw); with a fixed momentum: sum_live |q|^2 / lambda_m
  SL_LP0 = 1,  // sum_live |u|^2 / lambda at mu
  SL_RH0 = 2,  // ||Yh - mu_D||^2 at mu
  SL_RS0 = 3,  // ||Ys - W mu_D||^2 at mu
  SL_LPL = 4,  // sum_live |u*|^2 / lambda at the proposal
  SL_KL = 5,   // sum_live |q|^2 / lambda_m at the end of the trajectory
  SL_RHL = 6,
  SL_RSL = 7,
  SL_SCRATCH = 8,
  NSLOT = 9
};

// Per-chain scalar state.  The first block mirrors HMCParameters<float>
// (include/dualres/HMCParameters.h:66-87); the rest is the chain's place in
// MultiResParameters<float> and mcmc_summary<float>.
struct ChainState {
  double A, eps, eps0, eps_bar, eps_target, gamma, h_bar, mh_running_sum, mh_target, t0, kappa;
  int warmup, eps_start_found, burnin, integrator_steps, iteration, n_save, thin;
  // current iteration
  float eps_cur;   // step size used by this iteration
  int L_cur;       // leapfrog steps of this iteration; < 0 = chain idle
  float sh, ss;    // sigma_h^-2, sigma_s^-2
  int acc;         // which half of U / muD / muO holds the accepted state
  int saved;       // samples saved
  int done;        // nsave reached
  int save_now;    // this iteration was a save iteration
  long long accepted, grad_evals;
  double last_log_ratio;
  double last_E0, last_Ep;  // initial and proposed energy of the last transition
  double Rh_acc, Rs_acc;  // squared residual norms at the accepted state
  double ll_sum, sigh_sum, sigs_sum;
  float maxabs;    // max |mu| over output voxels at the last save
  int err;         // bounded-loop failures (gamma sampler)
};

// One volume on the device.  All pointers are device pointers.
struct DevVolume {
  int E0, E1, E2;
  long long N;
  int bx, by, bz;           // real-space box covering data and output voxels
  int n_h, n_s, n_o;
  const float* sinv;        // [N] 1/Re(lambda) on live modes, -1 on S
  const int* box_to_d;      // [bx*by*bz] data ordinal or -1 (box index x + bx (y + by z))
  const int* box_to_o;      // [bx*by*bz] output ordinal or -1
  const int* d_flat;        // [n_h] flat embedding index of each data voxel
  const int* o_flat;        // [n_o]
  const float* Yh;          // [n_h]
  const float* Ys;          // [n_s]
  const int* w_rowptr;      // W: n_s x n_h CSR
  const int* w_col;
  const float* w_val;
  const int* wt_rowptr;     // W^T: n_h x n_s CSR
  const int* wt_col;
  const float* wt_val;
};

// The per-chain device buffers of one chainset.
struct DevChains {
  int C;                    // chains
  int Cp;                   // pitch of the chain-minor arrays (>= C)
  int CG;                   // lanes per chain group in the kriging kernels (power of two <= 32)
  float2* U;                // [C][2][N]  spectral state: accepted / proposal halves
  float2* Q;                // [C][N]     spectral momentum
  float2* T1;               // [C][E2*E1*bx]
  float2* T2;               // [C][E2*by*bx]
  long long t1_stride, t2_stride;
  float* muD;               // [2][n_h][Cp] Re mu at data voxels
  float* muO;               // [2][n_o][Cp] Re mu at output voxels
  float* gD;                // [n_h][Cp] data gradient
  float* rs;                // [n_s][Cp] Ys - W mu_D
  double* part;             // [C][NSLOT][maxblk]
  int maxblk;
  int nb_x, nb_w, nb_wt;    // blocks writing partials in the x-line / W / W^T kernels
  ChainState* st;           // [C]
  double* s1;               // [n_o][Cp] sum mu
  double* s2;               // [n_o][Cp] sum mu^2
  double* sa;               // [n_o][Cp] sum |mu| / max|mu|
  float* samples;           // [nsave][n_o][Cp] or null
  double* save_rec;         // [nsave][C][3]: sigma_h, sigma_s, log likelihood per saved iteration, or null
  uint64_t seed;
  int chain0;               // global id of chain 0 (RNG key component)
  int* err;                 // device error word: bounded waits that gave up
  int ztile;                // chains per z-pass tile with 8 or more chains: 8 (4 lines x 8 chains) or 1 (32 lines)
  int fftplan;              // FP_* bits: the transforms that use the second radix plan of fft_smem (64, 128, 256 points)
};

// A kriging matrix (W or W^T) cut into dense tiles for the tensor-core
// products: rows in tiles of 128 (spatially ordered), the union of a tile's
// columns in chunks of 32.  Chunk q holds one 128 x 32 FP32 block in the
// K-major core-matrix layout: element (m, k) at float (k / 4) * 512 + m * 4 +
// k % 4 of the block.  The chunks are
// split into contiguous ranges, one per CTA; a range cut at tile boundaries
// gives segments, each summing into its own partial slot.
struct DevTcMatrix {
  int n_rows, n_cols;       // the matrix's shape (W: n_s x n_h; W^T: n_h x n_s)
  int T;                    // tiles
  int G;                    // CTAs of the product kernel (0: no nonzeros)
  int n_segs;
  int chunks;
  const int* tile_rows;     // [T * 128] matrix row of each tile row, or -1
  const int* chunk_cols;    // [chunks * 32] matrix column of each chunk column, or -1
  const float* blob;        // [chunks][128 * 32]
  const int4* segs;         // [n_segs] {tile, first chunk, end chunk, 0}, ordered by chunk
  const int* cta_seg_ptr;   // [G + 1] segments of each CTA
  const int* tile_seg_ptr;  // [T + 1] segments of each tile
};

// Pass-kernel arguments: a batched 1D FFT along the middle axis of an
// [A][n][B] array (B innermost), with pruned input / output extents.
struct PassArgs {
  const void* in;
  void* out;
  long long in_cs, out_cs;  // per-chain strides (complex elements)
  int A, B, n_in, n_out;
  double scale;
  int step;                 // hot-path step for chain masking; -1 = all chains
  int sel;                  // 0: accepted half of muD/muO; 1: proposal half
  int write_o;              // gather epilogue: 0 never, 1 always, 2 when step == L_cur
  int chain_only;           // >= 0: only this chain (API calls); -1: all
};

enum PassPro : int { PRO_LOAD = 0, PRO_DATAGRAD = 1 };
enum PassEpi : int { EPI_STORE = 0, EPI_GATHER = 1 };

// x-line kernel flags
// XF_L2_PREFETCH: the update kernels ask L2 for their blocks' state (u, q, 1/lambda) at entry, so that its DRAM
// latency overlaps the inverse transforms.
enum XFlags : int { XF_FIXED_MOMENTUM = 1, XF_WRITE_Q_LAST = 2, XF_L2_PREFETCH = 4 };
// Transforms that a chain set's tuning may switch to the second radix plan (fft_smem PLAN 1), one bit each.
enum FftPlanBits : int { FP_ZINV = 1, FP_ZFWD = 2, FP_XLINE = 4 };

}  // namespace drb
