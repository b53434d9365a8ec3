// Kriging weights on the device (get_sparse_kriging_matrix_data,
// kriging_matrix.h:148-343): one weight vector per std-res voxel,
// w = K_AA^-1 k_A over the present neighbours A, normalised to sum 1.
//
// With S = K^-1 over the full neighbourhood F (computed once per volume) a row
// whose absent neighbours are B solves, by the identity
//   K_AA^-1 k_A = [S v]_A,   v_A = k_A,  v_B = -y,  S_BB y = [S v0]_B,  v0 = (k_A, 0),
// one system of size |B| instead of |A|; the host picks the cheaper route per
// row (kriging_schur_route).  Every system is symmetric positive definite and is
// factored in FP64 by a blocked Cholesky: the 32 x 32 diagonal block by one
// warp, its triangular inverse, the panel below it as a product with that
// inverse, then a 64 x 64-tiled rank-32 update of the trailing matrix.  One
// CTA solves one row at a time, taking rows from a shared counter in
// descending order of cost; its matrix lives in a private slot of global
// memory, the lower triangle packed by rows.  A row whose pivot is not
// positive is reported, and the caller solves that row by QR as the host
// builder does.
#pragma once

namespace drb {

constexpr int KR_NT = 256;   // threads per CTA
constexpr int KR_NB = 32;    // panel width
constexpr int KR_TILE = 64;  // trailing-update tile
constexpr int KR_LDT = KR_NB + 1;

enum : int { KR_ROUTE_SCHUR = 0, KR_ROUTE_DIRECT = 1 };
enum : int { KR_OK = 0, KR_DROP = 1, KR_NOT_SPD = 2 };

struct KrigArgs {
  int m;                      // neighbourhood size
  const double* K;            // m x m
  const double* S;            // m x m inverse (Schur route only)
  const int* row_start;       // per std-res row, into pid / kp
  const int* pid;             // offset id of each present neighbour
  const double* kp;           // covariance of each present neighbour with the std-res centre
  const int* task_row;        // rows to solve, in order of decreasing cost
  const int* task_route;
  int ntasks;
  int* counter;               // next task
  double* w;                  // output weights, indexed like pid
  int* status;                // per row: KR_OK, KR_DROP (weight sum NaN), KR_NOT_SPD
  double* scratch;            // per CTA: nmax (nmax + 1) / 2 (packed matrix) + m (v) + nmax (t) doubles, then m ints
  size_t slot;                // doubles per CTA slot
  int nmax;
};

// Shared memory of one CTA (dynamic).
struct KrigSmem {
  double D[KR_NB][KR_LDT];      // diagonal block / its factor
  double Di[KR_NB][KR_LDT];     // inverse of the factor
  double PA[KR_TILE][KR_LDT];   // panel rows (tile I)
  double PB[KR_TILE][KR_LDT];   // panel rows (tile J)
  double red[KR_NT / 32];
  int flag;
  int task;
  int nb;
};

__device__ __forceinline__ double kr_block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < KR_NT / 32; i++) s += red[i];  // fixed order: every thread gets the same sum
  __syncthreads();
  return s;
}

// Factor the kb x kb block D in place (lower) with warp 0 and write its
// inverse to Di.  Returns false (block-uniform) if a pivot is not positive.
__device__ bool kr_factor_diag(double (*D)[KR_LDT], double (*Di)[KR_LDT], int& flag, int kb) {
  const int lane = threadIdx.x & 31;
  if (threadIdx.x < 32) {
    int bad = 0;
    for (int j = 0; j < kb; j++) {
      if (lane == j) {
        const double d = D[j][j];
        if (!(d > 0.0)) bad = 1;
        D[j][j] = sqrt(fmax(d, 1e-300));
      }
      bad = __shfl_sync(0xffffffffu, bad, j);
      __syncwarp();
      const double djj = D[j][j];
      if (lane > j && lane < kb) D[lane][j] /= djj;
      __syncwarp();
      if (lane > j && lane < kb) {
        const double lij = D[lane][j];
        for (int l = j + 1; l <= lane; l++) D[lane][l] -= lij * D[l][j];
      }
      __syncwarp();
    }
    if (lane == 0) flag = bad;
  }
  __syncthreads();
  if (flag) return false;
  // inverse of the lower-triangular factor, one column per thread (forward substitution)
  if (threadIdx.x < kb) {
    const int j = threadIdx.x;
    for (int i = 0; i < kb; i++) {
      double s = i == j ? 1.0 : 0.0;
      for (int l = j; l < i; l++) s -= D[i][l] * Di[l][j];
      Di[i][j] = i < j ? 0.0 : s / D[i][i];
    }
  }
  __syncthreads();
  return true;
}
__device__ bool kr_factor_diag(KrigSmem& sm, int kb) { return kr_factor_diag(sm.D, sm.Di, sm.flag, kb); }

// Position of (i, j), j <= i, in a lower triangle packed by rows: row i starts at i (i + 1) / 2.
__device__ __forceinline__ size_t kr_at(int i, int j) { return (size_t)i * (i + 1) / 2 + j; }

// In-place Cholesky M = L L^T of the n x n matrix (lower triangle, packed by rows: kr_at).
__device__ bool kr_cholesky(double* M, int n, KrigSmem& sm) {
  const int tid = threadIdx.x;
  for (int k0 = 0; k0 < n; k0 += KR_NB) {
    const int kb = min(KR_NB, n - k0);
    for (int e = tid; e < kb * kb; e += KR_NT) {
      const int i = e / kb, j = e % kb;
      sm.D[i][j] = j <= i ? M[kr_at(k0 + i, k0 + j)] : 0.0;
    }
    __syncthreads();
    if (!kr_factor_diag(sm, kb)) return false;
    for (int e = tid; e < kb * kb; e += KR_NT) {
      const int i = e / kb, j = e % kb;
      if (j <= i) M[kr_at(k0 + i, k0 + j)] = sm.D[i][j];
    }
    const int r0 = k0 + kb;
    // panel: L[i, k0:k0+kb] = A[i, k0:k0+kb] Di^T, in chunks of KR_TILE rows
    for (int c0 = r0; c0 < n; c0 += KR_TILE) {
      const int ch = min(KR_TILE, n - c0);
      __syncthreads();
      for (int e = tid; e < ch * kb; e += KR_NT) {
        const int i = e / kb, l = e % kb;
        sm.PA[i][l] = M[kr_at(c0 + i, k0 + l)];
      }
      __syncthreads();
      for (int e = tid; e < ch * kb; e += KR_NT) {
        const int i = e / kb, j = e % kb;
        double s = 0.0;
        for (int l = 0; l <= j; l++) s += sm.PA[i][l] * sm.Di[j][l];
        M[kr_at(c0 + i, k0 + j)] = s;
      }
    }
    __syncthreads();
    // trailing update A[i, j] -= L[i, panel] . L[j, panel] for r0 <= j <= i < n, 64 x 64 tiles
    const int T = (n - r0 + KR_TILE - 1) / KR_TILE;
    for (int tI = 0; tI < T; tI++) {
      const int i0 = r0 + tI * KR_TILE, ni = min(KR_TILE, n - i0);
      for (int e = tid; e < ni * kb; e += KR_NT) {
        const int i = e / kb, l = e % kb;
        sm.PA[i][l] = M[kr_at(i0 + i, k0 + l)];
      }
      for (int tJ = 0; tJ <= tI; tJ++) {
        const int j0 = r0 + tJ * KR_TILE, nj = min(KR_TILE, n - j0);
        __syncthreads();
        for (int e = tid; e < nj * kb; e += KR_NT) {
          const int j = e / kb, l = e % kb;
          sm.PB[j][l] = M[kr_at(j0 + j, k0 + l)];
        }
        __syncthreads();
        // each thread: a 4 x 4 micro-tile (rows ty*4.., cols tx*4..) of the 64 x 64 tile
        const int ty = tid / 16, tx = tid % 16;
        double acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
        for (int l = 0; l < kb; l++) {
          double pa[4], pb[4];
#pragma unroll
          for (int a = 0; a < 4; a++) pa[a] = sm.PA[ty * 4 + a][l];
#pragma unroll
          for (int b = 0; b < 4; b++) pb[b] = sm.PB[tx * 4 + b][l];
#pragma unroll
          for (int a = 0; a < 4; a++)
#pragma unroll
            for (int b = 0; b < 4; b++) acc[a][b] = fma(pa[a], pb[b], acc[a][b]);
        }
#pragma unroll
        for (int a = 0; a < 4; a++) {
          const int i = ty * 4 + a;
          if (i >= ni) continue;
#pragma unroll
          for (int b = 0; b < 4; b++) {
            const int j = tx * 4 + b;
            if (j >= nj || j0 + j > i0 + i) continue;
            M[kr_at(i0 + i, j0 + j)] -= acc[a][b];
          }
        }
      }
      __syncthreads();
    }
  }
  __syncthreads();
  return true;
}

// Solves L L^T x = b in place (b: n doubles in global memory), L from kr_cholesky.
__device__ void kr_solve(const double* L, int n, double* b, KrigSmem& sm) {
  const int tid = threadIdx.x;
  const int nblk = (n + KR_NB - 1) / KR_NB;
  auto load_inverse = [&](int k0, int kb) {
    __syncthreads();
    for (int e = tid; e < kb * kb; e += KR_NT) {
      const int i = e / kb, j = e % kb;
      sm.D[i][j] = j <= i ? L[kr_at(k0 + i, k0 + j)] : 0.0;
    }
    __syncthreads();
    if (tid < kb) {
      const int j = tid;
      for (int i = 0; i < kb; i++) {
        double s = i == j ? 1.0 : 0.0;
        for (int l = j; l < i; l++) s -= sm.D[i][l] * sm.Di[l][j];
        sm.Di[i][j] = i < j ? 0.0 : s / sm.D[i][i];
      }
    }
    __syncthreads();
  };
  // forward: y_k = Di (b_k - sum_{l<k} L_kl y_l), right-looking updates
  for (int kbk = 0; kbk < nblk; kbk++) {
    const int k0 = kbk * KR_NB, kb = min(KR_NB, n - k0);
    load_inverse(k0, kb);
    if (tid < kb) {
      double s = 0.0;
      for (int l = 0; l <= tid; l++) s += sm.Di[tid][l] * b[k0 + l];
      sm.PA[0][tid] = s;
    }
    __syncthreads();
    if (tid < kb) b[k0 + tid] = sm.PA[0][tid];
    __syncthreads();
    for (int i = k0 + kb + tid; i < n; i += KR_NT) {
      const double* Li = L + kr_at(i, k0);
      double s = 0.0;
      for (int l = 0; l < kb; l++) s += Li[l] * sm.PA[0][l];
      b[i] -= s;
    }
  }
  // backward: x_k = Di^T (y_k - sum_{l>k} L_lk^T x_l)
  for (int kbk = nblk - 1; kbk >= 0; kbk--) {
    const int k0 = kbk * KR_NB, kb = min(KR_NB, n - k0);
    load_inverse(k0, kb);
    if (tid < kb) {
      double s = 0.0;
      for (int l = tid; l < kb; l++) s += sm.Di[l][tid] * b[k0 + l];
      sm.PA[0][tid] = s;
    }
    __syncthreads();
    if (tid < kb) b[k0 + tid] = sm.PA[0][tid];
    __syncthreads();
    for (int i = tid; i < k0; i += KR_NT) {
      double s = 0.0;
      for (int l = 0; l < kb; l++) s += L[kr_at(k0 + l, i)] * sm.PA[0][l];
      b[i] -= s;
    }
  }
  __syncthreads();
}

// Warp-per-row dense products out[r] = sum_j Mat[rows[r]][j] v[j] over the m offsets.
__device__ void kr_rows_dot(const double* Mat, int m, const int* rows, int nrows, const double* v, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int r = warp; r < nrows; r += KR_NT / 32) {
    const double* Mr = Mat + (size_t)rows[r] * m;
    double s = 0.0;
    for (int j = lane; j < m; j += 32) s += Mr[j] * v[j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[r] = s;
  }
}

// ---------------------------------------------------------------- K^-1 over the whole GPU
// S = K^-1 of the neighbourhood covariance (m up to 5000), once per volume:
//   right-looking blocked Cholesky K = L L^T in panels of KR_NB columns: the diagonal block by one CTA
//   (k_chol_diag, which also keeps the inverse of the block's factor), the panel below it by one CTA per 64 rows
//   (k_chol_panel), the trailing update by one CTA per 64 x 64 tile of the lower triangle (k_chol_update);
//   X = L^-1 one block row at a time, X_ij = -Dinv_i sum_{j <= k < i} L_ik X_kj, one CTA per block column
//   (k_trinv_row);  S = X^T X, one CTA per 32 x 32 tile of the lower triangle, stored to both triangles so that S is
//   exactly symmetric (k_trinv_gram).
// A pivot that is not positive clears *ok and every later launch returns at once.

// The kb x kb diagonal block at k0: factored in place, its factor's inverse to Dinv[k0 / KR_NB] (32 x 32, zero
// outside kb x kb).
__global__ void __launch_bounds__(KR_NT) k_chol_diag(double* M, int n, int k0, double* Dinv, int* ok) {
  __shared__ double D[KR_NB][KR_LDT], Di[KR_NB][KR_LDT];
  __shared__ int flag;
  if (!*ok) return;
  const int kb = min(KR_NB, n - k0), tid = threadIdx.x;
  for (int e = tid; e < KR_NB * KR_NB; e += KR_NT) {
    const int i = e / KR_NB, j = e % KR_NB;
    D[i][j] = (i < kb && j <= i) ? M[(size_t)(k0 + i) * n + k0 + j] : 0.0;
    Di[i][j] = 0.0;
  }
  __syncthreads();
  const bool good = kr_factor_diag(D, Di, flag, kb);
  if (!good) {
    if (tid == 0) *ok = 0;
    return;
  }
  double* Dg = Dinv + (size_t)(k0 / KR_NB) * KR_NB * KR_NB;
  for (int e = tid; e < KR_NB * KR_NB; e += KR_NT) {
    const int i = e / KR_NB, j = e % KR_NB;
    if (i < kb && j <= i) M[(size_t)(k0 + i) * n + k0 + j] = D[i][j];
    Dg[e] = (i < kb && j < kb) ? Di[i][j] : 0.0;
  }
}

// L[i, k0:k0+kb] = A[i, k0:k0+kb] Dinv^T for the 64 rows i of this CTA below the diagonal block.
__global__ void __launch_bounds__(KR_NT) k_chol_panel(double* M, int n, int k0, const double* Dinv, const int* ok) {
  __shared__ double Di[KR_NB][KR_LDT], PA[KR_TILE][KR_LDT];
  if (!*ok) return;
  const int kb = min(KR_NB, n - k0), tid = threadIdx.x;
  const int c0 = k0 + kb + blockIdx.x * KR_TILE, ch = min(KR_TILE, n - c0);
  const double* Dg = Dinv + (size_t)(k0 / KR_NB) * KR_NB * KR_NB;
  for (int e = tid; e < KR_NB * KR_NB; e += KR_NT) Di[e / KR_NB][e % KR_NB] = Dg[e];
  for (int e = tid; e < ch * kb; e += KR_NT) {
    const int i = e / kb, l = e % kb;
    PA[i][l] = M[(size_t)(c0 + i) * n + k0 + l];
  }
  __syncthreads();
  for (int e = tid; e < ch * kb; e += KR_NT) {
    const int i = e / kb, j = e % kb;
    double s = 0.0;
    for (int l = 0; l <= j; l++) s += PA[i][l] * Di[j][l];
    M[(size_t)(c0 + i) * n + k0 + j] = s;
  }
}

// Lower-triangle tile index b -> (tI, tJ), tJ <= tI.
__device__ __forceinline__ void kr_tri_tile(int b, int* tI, int* tJ) {
  int i = (int)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
  while (i * (i + 1) / 2 > b) i--;
  while ((i + 1) * (i + 2) / 2 <= b) i++;
  *tI = i;
  *tJ = b - i * (i + 1) / 2;
}

// A[i, j] -= L[i, panel] . L[j, panel] on one 64 x 64 tile of the trailing lower triangle.
__global__ void __launch_bounds__(KR_NT) k_chol_update(double* M, int n, int k0, const int* ok) {
  __shared__ double PA[KR_TILE][KR_LDT], PB[KR_TILE][KR_LDT];
  if (!*ok) return;
  const int kb = min(KR_NB, n - k0), r0 = k0 + kb, tid = threadIdx.x;
  int tI, tJ;
  kr_tri_tile(blockIdx.x, &tI, &tJ);
  const int i0 = r0 + tI * KR_TILE, j0 = r0 + tJ * KR_TILE;
  const int ni = min(KR_TILE, n - i0), nj = min(KR_TILE, n - j0);
  for (int e = tid; e < KR_TILE * kb; e += KR_NT) {
    const int i = e / kb, l = e % kb;
    PA[i][l] = i < ni ? M[(size_t)(i0 + i) * n + k0 + l] : 0.0;
    PB[i][l] = i < nj ? M[(size_t)(j0 + i) * n + k0 + l] : 0.0;
  }
  __syncthreads();
  const int ty = tid / 16, tx = tid % 16;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
  for (int l = 0; l < kb; l++) {
    double pa[4], pb[4];
#pragma unroll
    for (int a = 0; a < 4; a++) pa[a] = PA[ty * 4 + a][l];
#pragma unroll
    for (int b = 0; b < 4; b++) pb[b] = PB[tx * 4 + b][l];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) acc[a][b] = fma(pa[a], pb[b], acc[a][b]);
  }
#pragma unroll
  for (int a = 0; a < 4; a++) {
    const int i = ty * 4 + a;
    if (i >= ni) continue;
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const int j = tx * 4 + b;
      if (j >= nj || j0 + j > i0 + i) continue;
      M[(size_t)(i0 + i) * n + j0 + j] -= acc[a][b];
    }
  }
}

// One 32 x 32 tile product acc += A^T? B over shared tiles: acc[p][q] += sum_r TA[p][r] TB[r][q] (TRANS = false) or
// sum_r TA[r][p] TB[r][q] (TRANS = true); each of the 256 threads owns 4 entries (p = tid / 8, q = 4 (tid % 8) + b).
template <bool TRANS>
__device__ __forceinline__ void kr_tile_mac(const double (*TA)[KR_LDT], const double (*TB)[KR_LDT], double acc[4]) {
  const int p = threadIdx.x / 8, q0 = 4 * (threadIdx.x % 8);
  for (int r = 0; r < KR_NB; r++) {
    const double a = TRANS ? TA[r][p] : TA[p][r];
#pragma unroll
    for (int b = 0; b < 4; b++) acc[b] = fma(a, TB[r][q0 + b], acc[b]);
  }
}

// Loads the 32 x 32 tile of the n x n row-major matrix at block (bi, bj), zero outside n x n.
__device__ __forceinline__ void kr_load_tile(double (*T)[KR_LDT], const double* A, int n, int bi, int bj) {
  for (int e = threadIdx.x; e < KR_NB * KR_NB; e += KR_NT) {
    const int i = e / KR_NB, j = e % KR_NB, gi = bi * KR_NB + i, gj = bj * KR_NB + j;
    T[i][j] = (gi < n && gj < n) ? A[(size_t)gi * n + gj] : 0.0;
  }
}

// Block row bi of X = L^-1: CTA bj < bi computes X[bi][bj] = -Dinv_bi sum_{bj <= k < bi} L[bi][k] X[k][bj];
// CTA bj = bi writes X[bi][bi] = Dinv_bi.
__global__ void __launch_bounds__(KR_NT) k_trinv_row(const double* L, int n, int bi, const double* Dinv, double* X,
                                                     const int* ok) {
  __shared__ double TA[KR_NB][KR_LDT], TB[KR_NB][KR_LDT];
  if (!*ok) return;
  const int bj = blockIdx.x, p = threadIdx.x / 8, q0 = 4 * (threadIdx.x % 8);
  const double* Dg = Dinv + (size_t)bi * KR_NB * KR_NB;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  if (bj == bi) {
#pragma unroll
    for (int b = 0; b < 4; b++) acc[b] = Dg[p * KR_NB + q0 + b];
  } else {
    for (int k = bj; k < bi; k++) {
      __syncthreads();
      kr_load_tile(TA, L, n, bi, k);
      kr_load_tile(TB, X, n, k, bj);
      __syncthreads();
      kr_tile_mac<false>(TA, TB, acc);
    }
    // X[bi][bj] = -Dinv_bi acc (acc through shared memory)
    __syncthreads();
#pragma unroll
    for (int b = 0; b < 4; b++) TB[p][q0 + b] = acc[b];
    for (int e = threadIdx.x; e < KR_NB * KR_NB; e += KR_NT) TA[e / KR_NB][e % KR_NB] = Dg[e];
    __syncthreads();
    double r[4] = {0.0, 0.0, 0.0, 0.0};
    kr_tile_mac<false>(TA, TB, r);
#pragma unroll
    for (int b = 0; b < 4; b++) acc[b] = -r[b];
  }
#pragma unroll
  for (int b = 0; b < 4; b++) {
    const int gi = bi * KR_NB + p, gj = bj * KR_NB + q0 + b;
    if (gi < n && gj < n) X[(size_t)gi * n + gj] = acc[b];
  }
}

// S[ba][bb] = sum_{k >= ba} X[k][ba]^T X[k][bb] for the tile (ba >= bb) of this CTA, stored with its transpose.
__global__ void __launch_bounds__(KR_NT) k_trinv_gram(const double* X, int n, double* S, const int* ok) {
  __shared__ double TA[KR_NB][KR_LDT], TB[KR_NB][KR_LDT];
  if (!*ok) return;
  int ba, bb;
  kr_tri_tile(blockIdx.x, &ba, &bb);
  const int nb = (n + KR_NB - 1) / KR_NB, p = threadIdx.x / 8, q0 = 4 * (threadIdx.x % 8);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int k = ba; k < nb; k++) {
    __syncthreads();
    kr_load_tile(TA, X, n, k, ba);
    kr_load_tile(TB, X, n, k, bb);
    __syncthreads();
    kr_tile_mac<true>(TA, TB, acc);
  }
#pragma unroll
  for (int b = 0; b < 4; b++) {
    const int gi = ba * KR_NB + p, gj = bb * KR_NB + q0 + b;
    if (gi < n && gj < n) {
      S[(size_t)gi * n + gj] = acc[b];
      S[(size_t)gj * n + gi] = acc[b];
    }
  }
}

__global__ void __launch_bounds__(KR_NT) k_kriging_rows(KrigArgs a) {
  extern __shared__ __align__(16) unsigned char kr_smraw[];
  KrigSmem& sm = *reinterpret_cast<KrigSmem*>(kr_smraw);
  const int tid = threadIdx.x;
  double* M = a.scratch + (size_t)blockIdx.x * a.slot;
  double* v = M + kr_at(a.nmax, 0);  // the packed lower triangle of an nmax x nmax matrix
  double* t = v + a.m;
  int* ids = reinterpret_cast<int*>(t + a.nmax);
  const int m = a.m;
  for (;;) {
    __syncthreads();
    if (tid == 0) sm.task = atomicAdd(a.counter, 1);
    __syncthreads();
    const int ti = sm.task;
    if (ti >= a.ntasks) break;
    const int row = a.task_row[ti], route = a.task_route[ti];
    const int r0 = a.row_start[row], cnt = a.row_start[row + 1] - r0;
    const int* pid = a.pid + r0;
    const double* k = a.kp + r0;
    double* x = a.w + r0;
    bool ok = true;
    if (route == KR_ROUTE_DIRECT) {
      const int n = cnt;
      for (size_t e = tid; e < (size_t)n * n; e += KR_NT) {
        const int i = (int)(e / n), j = (int)(e % n);
        if (j <= i) M[kr_at(i, j)] = a.K[(size_t)pid[i] * m + pid[j]];
      }
      for (int i = tid; i < n; i += KR_NT) x[i] = k[i];
      __syncthreads();
      ok = kr_cholesky(M, n, sm);
      if (ok) kr_solve(M, n, x, sm);
    } else {
      // v0 = (k_A, 0) over the offsets; absent offsets B in ascending order
      for (int j = tid; j < m; j += KR_NT) {
        v[j] = 0.0;
        ids[j] = 1;
      }
      __syncthreads();
      for (int i = tid; i < cnt; i += KR_NT) {
        v[pid[i]] = k[i];
        ids[pid[i]] = 0;
      }
      __syncthreads();
      if (tid == 0) {  // compact the absent offsets (ascending); m <= 5000
        int nb = 0;
        for (int j = 0; j < m; j++)
          if (ids[j]) ids[nb++] = j;
        sm.nb = nb;
      }
      __syncthreads();
      const int nb = sm.nb;
      if (nb > 0) {
        kr_rows_dot(a.S, m, ids, nb, v, t);  // t = [S v0]_B
        for (size_t e = tid; e < (size_t)nb * nb; e += KR_NT) {
          const int i = (int)(e / nb), j = (int)(e % nb);
          if (j <= i) M[kr_at(i, j)] = a.S[(size_t)ids[i] * m + ids[j]];
        }
        __syncthreads();
        ok = kr_cholesky(M, nb, sm);
        if (ok) {
          kr_solve(M, nb, t, sm);
          for (int q = tid; q < nb; q += KR_NT) v[ids[q]] = -t[q];
          __syncthreads();
        }
      }
      if (ok) {
        kr_rows_dot(a.S, m, pid, cnt, v, x);
        __syncthreads();
      }
    }
    int st = KR_OK;
    if (!ok) {
      st = KR_NOT_SPD;
    } else {
      double s = 0.0;
      for (int i = tid; i < cnt; i += KR_NT) s += x[i];
      double wsum = kr_block_sum(s, sm.red);
      if (isnan(wsum)) {
        st = KR_DROP;
      } else {
        if (wsum == 0.0) wsum = 1.0;  // kriging_matrix.h:318-319
        for (int i = tid; i < cnt; i += KR_NT) x[i] /= wsum;
      }
    }
    if (tid == 0) a.status[row] = st;
  }
}

}  // namespace drb
