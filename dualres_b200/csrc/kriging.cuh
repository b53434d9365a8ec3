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
// memory (L2-resident for the sizes that occur).  A row whose pivot is not
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
  double* scratch;            // per CTA: nmax^2 (matrix) + m (v) + nmax (t) doubles, then m ints
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

// Factor the kb x kb block in sm.D in place (lower) with warp 0 and write its
// inverse to sm.Di.  Returns false (block-uniform) if a pivot is not positive.
__device__ bool kr_factor_diag(KrigSmem& sm, int kb) {
  const int lane = threadIdx.x & 31;
  if (threadIdx.x < 32) {
    int bad = 0;
    for (int j = 0; j < kb; j++) {
      if (lane == j) {
        const double d = sm.D[j][j];
        if (!(d > 0.0)) bad = 1;
        sm.D[j][j] = sqrt(fmax(d, 1e-300));
      }
      bad = __shfl_sync(0xffffffffu, bad, j);
      __syncwarp();
      const double djj = sm.D[j][j];
      if (lane > j && lane < kb) sm.D[lane][j] /= djj;
      __syncwarp();
      if (lane > j && lane < kb) {
        const double lij = sm.D[lane][j];
        for (int l = j + 1; l <= lane; l++) sm.D[lane][l] -= lij * sm.D[l][j];
      }
      __syncwarp();
    }
    if (lane == 0) sm.flag = bad;
  }
  __syncthreads();
  if (sm.flag) return false;
  // inverse of the lower-triangular factor, one column per thread (forward substitution)
  if (threadIdx.x < kb) {
    const int j = threadIdx.x;
    for (int i = 0; i < kb; i++) {
      double s = i == j ? 1.0 : 0.0;
      for (int l = j; l < i; l++) s -= sm.D[i][l] * sm.Di[l][j];
      sm.Di[i][j] = i < j ? 0.0 : s / sm.D[i][i];
    }
  }
  __syncthreads();
  return true;
}

// In-place Cholesky M = L L^T of the n x n matrix (row-major, lower triangle read and written).
__device__ bool kr_cholesky(double* M, int n, KrigSmem& sm) {
  const int tid = threadIdx.x;
  for (int k0 = 0; k0 < n; k0 += KR_NB) {
    const int kb = min(KR_NB, n - k0);
    for (int e = tid; e < kb * kb; e += KR_NT) {
      const int i = e / kb, j = e % kb;
      sm.D[i][j] = j <= i ? M[(size_t)(k0 + i) * n + k0 + j] : 0.0;
    }
    __syncthreads();
    if (!kr_factor_diag(sm, kb)) return false;
    for (int e = tid; e < kb * kb; e += KR_NT) {
      const int i = e / kb, j = e % kb;
      if (j <= i) M[(size_t)(k0 + i) * n + k0 + j] = sm.D[i][j];
    }
    const int r0 = k0 + kb;
    // panel: L[i, k0:k0+kb] = A[i, k0:k0+kb] Di^T, in chunks of KR_TILE rows
    for (int c0 = r0; c0 < n; c0 += KR_TILE) {
      const int ch = min(KR_TILE, n - c0);
      __syncthreads();
      for (int e = tid; e < ch * kb; e += KR_NT) {
        const int i = e / kb, l = e % kb;
        sm.PA[i][l] = M[(size_t)(c0 + i) * n + k0 + l];
      }
      __syncthreads();
      for (int e = tid; e < ch * kb; e += KR_NT) {
        const int i = e / kb, j = e % kb;
        double s = 0.0;
        for (int l = 0; l <= j; l++) s += sm.PA[i][l] * sm.Di[j][l];
        M[(size_t)(c0 + i) * n + k0 + j] = s;
      }
    }
    __syncthreads();
    // trailing update A[i, j] -= L[i, panel] . L[j, panel] for r0 <= j <= i < n, 64 x 64 tiles
    const int T = (n - r0 + KR_TILE - 1) / KR_TILE;
    for (int tI = 0; tI < T; tI++) {
      const int i0 = r0 + tI * KR_TILE, ni = min(KR_TILE, n - i0);
      for (int e = tid; e < ni * kb; e += KR_NT) {
        const int i = e / kb, l = e % kb;
        sm.PA[i][l] = M[(size_t)(i0 + i) * n + k0 + l];
      }
      for (int tJ = 0; tJ <= tI; tJ++) {
        const int j0 = r0 + tJ * KR_TILE, nj = min(KR_TILE, n - j0);
        __syncthreads();
        for (int e = tid; e < nj * kb; e += KR_NT) {
          const int j = e / kb, l = e % kb;
          sm.PB[j][l] = M[(size_t)(j0 + j) * n + k0 + l];
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
            M[(size_t)(i0 + i) * n + j0 + j] -= acc[a][b];
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
      sm.D[i][j] = j <= i ? L[(size_t)(k0 + i) * n + k0 + j] : 0.0;
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
      const double* Li = L + (size_t)i * n + k0;
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
      for (int l = 0; l < kb; l++) s += L[(size_t)(k0 + l) * n + i] * sm.PA[0][l];
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

// K = L L^T in place by one block (M holds K on entry); *ok = 1 when K is positive definite.
__global__ void __launch_bounds__(KR_NT) k_spd_factor(double* M, int n, int* ok) {
  extern __shared__ __align__(16) unsigned char kr_smraw[];
  KrigSmem& sm = *reinterpret_cast<KrigSmem*>(kr_smraw);
  const bool good = kr_cholesky(M, n, sm);
  if (threadIdx.x == 0) *ok = good ? 1 : 0;
}

// Rows of S = K^-1 from the factor: each block solves L L^T x = e_j for its
// share of j (x in its scratch vector) and stores x as row j of S.
__global__ void __launch_bounds__(KR_NT) k_spd_inverse(const double* L, int n, double* S, double* scratch) {
  extern __shared__ __align__(16) unsigned char kr_smraw[];
  KrigSmem& sm = *reinterpret_cast<KrigSmem*>(kr_smraw);
  double* b = scratch + (size_t)blockIdx.x * n;
  for (int j = blockIdx.x; j < n; j += gridDim.x) {
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += KR_NT) b[i] = i == j ? 1.0 : 0.0;
    __syncthreads();
    kr_solve(L, n, b, sm);
    for (int i = threadIdx.x; i < n; i += KR_NT) S[(size_t)j * n + i] = b[i];
  }
}

// S = (S + S^T) / 2 (the two triangular solves leave O(eps) asymmetry).
__global__ void k_symmetrize(double* S, int n) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * n) return;
  const int i = (int)(e / n), j = (int)(e % n);
  if (j >= i) return;
  const double a = 0.5 * (S[(size_t)i * n + j] + S[(size_t)j * n + i]);
  S[(size_t)i * n + j] = a;
  S[(size_t)j * n + i] = a;
}

__global__ void __launch_bounds__(KR_NT) k_kriging_rows(KrigArgs a) {
  extern __shared__ __align__(16) unsigned char kr_smraw[];
  KrigSmem& sm = *reinterpret_cast<KrigSmem*>(kr_smraw);
  const int tid = threadIdx.x;
  double* M = a.scratch + (size_t)blockIdx.x * a.slot;
  double* v = M + (size_t)a.nmax * a.nmax;
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
        if (j <= i) M[e] = a.K[(size_t)pid[i] * m + pid[j]];
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
          if (j <= i) M[e] = a.S[(size_t)ids[i] * m + ids[j]];
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
