/*
 * dr_oracle_common.c -- precision-independent part of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see dr_oracle.h).  Parity unpinned: the reference
 * has no golden vectors and cannot be compiled in this image.
 */
#include "dr_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* nifti_manipulation.inl:335-360 -- nonzero = !(isnan(v) || v == 0), i fastest. */
int orc_nonzero_indices(const float* img, int nx, int ny, int nz, int* ijk, int max_out) {
  const long nvox = (long)nx * ny * nz;
  int n = 0;
  for (long i = 0; i < nvox; i++) {
    const float v = img[i];
    if (!(isnan(v) || v == 0.0f)) {
      if (n >= max_out) return -1;
      ijk[3 * n + 0] = (int)(i % nx);
      ijk[3 * n + 1] = (int)((i / nx) % ny);
      ijk[3 * n + 2] = (int)((i / ((long)nx * ny)) % nz);
      n++;
    }
  }
  return n;
}

/* nifti_manipulation.inl:210-219 */
int orc_bounding_box(const float* img, int nx, int ny, int nz, int* bbmin, int* bbmax) {
  int n = 0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const float v = img[(long)k * nx * ny + (long)j * nx + i];
        if (isnan(v) || v == 0.0f) continue;
        if (n == 0) {
          bbmin[0] = bbmax[0] = i; bbmin[1] = bbmax[1] = j; bbmin[2] = bbmax[2] = k;
        } else {
          if (i < bbmin[0]) bbmin[0] = i;
          if (i > bbmax[0]) bbmax[0] = i;
          if (j < bbmin[1]) bbmin[1] = j;
          if (j > bbmax[1]) bbmax[1] = j;
          if (k < bbmin[2]) bbmin[2] = k;
          if (k > bbmax[2]) bbmax[2] = k;
        }
        n++;
      }
  return n;
}

/* MultiResParameters.h:191-206; circulant_base.inl:44-57 */
int orc_embedding_dims(const int* g, int* E) {
  for (int d = 0; d < 3; d++) {
    if (g[d] <= 1) return -1;
    const int target = 2 * (g[d] - 1);
    int p = 1;
    while (p < target) p <<= 1;
    E[d] = p;
  }
  return 0;
}

/* kriging_matrix.h:63-106 with nifti_manipulation.inl:600-605 (voxel dims are
 * the column norms of the qform's first three columns). Float arithmetic. */
int orc_neighborhood(const float* Q, float radius, int* P, int max_out) {
  if (radius < 0) return -2;
  float vd[3];
  int nr[3];
  for (int c = 0; c < 3; c++) {
    float s = 0.0f;
    for (int r = 0; r < 4; r++) s += Q[4 * r + c] * Q[4 * r + c];
    vd[c] = sqrtf(s);
    nr[c] = (int)(radius / vd[c]);
  }
  int n = 0;
  /* expand_grid_3d (kriging_matrix.h:41-56): i fastest, then j, then k. */
  for (int k = -nr[2]; k <= nr[2]; k++)
    for (int j = -nr[1]; j <= nr[1]; j++)
      for (int i = -nr[0]; i <= nr[0]; i++) {
        float q2 = 0.0f;
        for (int r = 0; r < 3; r++) {
          const float q = Q[4 * r + 0] * (float)i + Q[4 * r + 1] * (float)j + Q[4 * r + 2] * (float)k;
          q2 += q * q;
        }
        if (sqrtf(q2) <= radius) {
          if (n >= max_out) return -1;
          P[3 * n + 0] = i; P[3 * n + 1] = j; P[3 * n + 2] = k;
          n++;
        }
      }
  return n;
}

static int is_nz(float v) { return !(isnan(v) || v == 0.0f); }

/* dualgpm.cpp:125-155, 288; gaussian_process_model.h:104-117;
 * nifti_manipulation.inl:75-125 (apply_mask), 20-66 (add_to), 377-398. */
int orc_prepare_highres(float* hr, const float* hmask, const float* omask,
                        int nx, int ny, int nz,
                        int* D_ijk, float* Yh, int* O_ijk, int* n_o, int max_out) {
  const long nvox = (long)nx * ny * nz;
  float* hm = (float*)malloc(sizeof(float) * nvox);
  float* om = (float*)malloc(sizeof(float) * nvox);
  if (!hm || !om) { free(hm); free(om); return -10; }
  /* Both masks default to the (unmasked) high-res image itself. */
  memcpy(hm, hmask ? hmask : hr, sizeof(float) * nvox);
  memcpy(om, omask ? omask : hr, sizeof(float) * nvox);
  for (long i = 0; i < nvox; i++)
    if (hm[i] == 0.0f || isnan(hr[i])) hr[i] = 0.0f;
  for (long i = 0; i < nvox; i++) hm[i] += om[i]; /* hmask becomes the union mask */
  int bbmin[3], bbmax[3];
  if (orc_bounding_box(hm, nx, ny, nz, bbmin, bbmax) <= 0) { free(hm); free(om); return -11; }
  int nh = 0, no = 0, ny_ = 0;
  for (long idx = 0; idx < nvox; idx++) {
    const int i = (int)(idx % nx), j = (int)((idx / nx) % ny), k = (int)(idx / ((long)nx * ny));
    const int inbox = i >= bbmin[0] && i <= bbmax[0] && j >= bbmin[1] && j <= bbmax[1] &&
                      k >= bbmin[2] && k <= bbmax[2];
    if (is_nz(hr[idx])) {
      if (ny_ >= max_out) { free(hm); free(om); return -1; }
      Yh[ny_++] = hr[idx];
      if (inbox) {
        D_ijk[3 * nh + 0] = i - bbmin[0]; D_ijk[3 * nh + 1] = j - bbmin[1]; D_ijk[3 * nh + 2] = k - bbmin[2];
        nh++;
      }
    }
    if (is_nz(om[idx]) && inbox) {
      if (no >= max_out) { free(hm); free(om); return -1; }
      O_ijk[3 * no + 0] = i - bbmin[0]; O_ijk[3 * no + 1] = j - bbmin[1]; O_ijk[3 * no + 2] = k - bbmin[2];
      no++;
    }
  }
  free(hm); free(om);
  *n_o = no;
  /* The reference indexes Yh by data ordinal; a mismatch is undefined there. */
  if (ny_ != nh) return -12;
  return nh;
}

/* kernels.inl:8-15 (rbf) and 59-74 (rational quadratic); theta = (v, b|psi, e|nu). */
double orc_cov(int covfun, double d, const double* theta) {
  if (covfun == 0) return theta[0] * exp(-theta[1] * pow(fabs(d), theta[2]));
  return theta[0] * pow(1.0 + theta[1] / theta[2] * d * d, -theta[2]);
}

static double rbf_d(double d, const double* th) { return th[0] * exp(-th[1] * pow(fabs(d), th[2])); }

/* Lower Cholesky of the m x m row-major SPD matrix A (unblocked, dot-product
 * form).  Returns 0 if a pivot is not positive. */
static int cholesky_inplace(double* A, int m) {
  for (int j = 0; j < m; j++) {
    double* Aj = A + (long)j * m;
    double d = Aj[j];
    for (int p = 0; p < j; p++) d -= Aj[p] * Aj[p];
    if (!(d > 0.0)) return 0;
    const double l = sqrt(d);
    Aj[j] = l;
    for (int i = j + 1; i < m; i++) {
      double* Ai = A + (long)i * m;
      double s = Ai[j];
      for (int p = 0; p < j; p++) s -= Ai[p] * Aj[p];
      Ai[j] = s / l;
    }
  }
  return 1;
}

static void cholesky_solve_inplace(const double* L, int m, double* b) {
  for (int i = 0; i < m; i++) {
    double s = b[i];
    for (int p = 0; p < i; p++) s -= L[(long)i * m + p] * b[p];
    b[i] = s / L[(long)i * m + i];
  }
  for (int i = m - 1; i >= 0; i--) {
    double s = b[i];
    for (int p = i + 1; p < m; p++) s -= L[(long)p * m + i] * b[p];
    b[i] = s / L[(long)i * m + i];
  }
}

/* Column-pivoted Householder QR solve of the m x m system A x = b (A row-major,
 * destroyed).  Components beyond the numerical rank are set to zero, as in a
 * rank-revealing basic solution. */
static void colpiv_qr_solve(double* A, int m, double* b, double* x) {
  int* perm = (int*)malloc(sizeof(int) * m);
  double* cn = (double*)malloc(sizeof(double) * m);
  double* v = (double*)malloc(sizeof(double) * m);
  for (int j = 0; j < m; j++) {
    perm[j] = j;
    double s = 0.0;
    for (int i = 0; i < m; i++) s += A[(long)i * m + j] * A[(long)i * m + j];
    cn[j] = s;
  }
  double r00 = 0.0;
  int rank = m;
  for (int k = 0; k < m; k++) {
    /* pivot: largest remaining column norm (recomputed exactly for stability) */
    int best = k;
    double bn = -1.0;
    for (int j = k; j < m; j++) {
      double s = 0.0;
      for (int i = k; i < m; i++) s += A[(long)i * m + j] * A[(long)i * m + j];
      cn[j] = s;
      if (s > bn) { bn = s; best = j; }
    }
    if (best != k) {
      for (int i = 0; i < m; i++) {
        double t = A[(long)i * m + k]; A[(long)i * m + k] = A[(long)i * m + best]; A[(long)i * m + best] = t;
      }
      int t = perm[k]; perm[k] = perm[best]; perm[best] = t;
    }
    double alpha = sqrt(bn);
    if (k == 0) r00 = alpha;
    if (alpha <= (double)m * DBL_EPSILON * r00) { rank = k; break; }
    const double akk = A[(long)k * m + k];
    if (akk > 0) alpha = -alpha;
    /* v = x - alpha e1, normalised so that H = I - 2 v v^T / (v^T v) */
    double vnorm2 = 0.0;
    for (int i = k; i < m; i++) v[i] = A[(long)i * m + k];
    v[k] -= alpha;
    for (int i = k; i < m; i++) vnorm2 += v[i] * v[i];
    if (vnorm2 > 0.0) {
      for (int j = k; j < m; j++) {
        double s = 0.0;
        for (int i = k; i < m; i++) s += v[i] * A[(long)i * m + j];
        s = 2.0 * s / vnorm2;
        for (int i = k; i < m; i++) A[(long)i * m + j] -= s * v[i];
      }
      double s = 0.0;
      for (int i = k; i < m; i++) s += v[i] * b[i];
      s = 2.0 * s / vnorm2;
      for (int i = k; i < m; i++) b[i] -= s * v[i];
    }
  }
  /* back substitution on the leading rank x rank block */
  double* y = (double*)calloc((size_t)m, sizeof(double));
  for (int i = rank - 1; i >= 0; i--) {
    double s = b[i];
    for (int j = i + 1; j < rank; j++) s -= A[(long)i * m + j] * y[j];
    y[i] = s / A[(long)i * m + i];
  }
  for (int j = 0; j < m; j++) x[perm[j]] = y[j];
  free(y); free(perm); free(cn); free(v);
}

static void mat4_inverse(const double* a, double* inv) {
  /* Gauss-Jordan with partial pivoting on a 4x4 row-major matrix. */
  double m[4][8];
  for (int i = 0; i < 4; i++) {
    for (int j = 0; j < 4; j++) { m[i][j] = a[4 * i + j]; m[i][j + 4] = (i == j) ? 1.0 : 0.0; }
  }
  for (int c = 0; c < 4; c++) {
    int p = c;
    for (int r = c + 1; r < 4; r++) if (fabs(m[r][c]) > fabs(m[p][c])) p = r;
    if (p != c) for (int j = 0; j < 8; j++) { double t = m[c][j]; m[c][j] = m[p][j]; m[p][j] = t; }
    const double d = m[c][c];
    for (int j = 0; j < 8; j++) m[c][j] /= d;
    for (int r = 0; r < 4; r++) {
      if (r == c) continue;
      const double f = m[r][c];
      for (int j = 0; j < 8; j++) m[r][j] -= f * m[c][j];
    }
  }
  for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) inv[4 * i + j] = m[i][j + 4];
}

/* kriging_matrix.h:148-343 */
int64_t orc_kriging_build(const float* hr, int nx, int ny, int nz, const float* Qhr,
                          const float* sr, int sx, int sy, int sz, const float* Qsr,
                          const float* theta, float radius, int solve,
                          int* rowptr, int max_rows, int* col, double* val,
                          int64_t max_nnz, int* n_rows_out) {
  const long nvox_hr = (long)nx * ny * nz;
  int cap = 8192;
  int* P = (int*)malloc(sizeof(int) * 3 * cap);
  int m = orc_neighborhood(Qhr, radius, P, cap);
  if (m == -1) { free(P); return -2; }   /* > 8192 offsets: certainly > 5000 */
  if (m <= 0) { free(P); return -4; }
  if (m > 5000) { free(P); return -2; } /* kriging_matrix.h:172-174 */
  const double th[3] = {theta[0], theta[1], theta[2]};

  /* perturbation_kernel_distances (kriging_matrix.h:111-138): unit diagonal. */
  double* Pmm = (double*)malloc(sizeof(double) * 3 * m);
  for (int i = 0; i < m; i++)
    for (int r = 0; r < 3; r++)
      Pmm[3 * i + r] = (double)Qhr[4 * r + 0] * P[3 * i + 0] + (double)Qhr[4 * r + 1] * P[3 * i + 1] +
                       (double)Qhr[4 * r + 2] * P[3 * i + 2];
  double* K = NULL;
  if (solve) {
    K = (double*)malloc(sizeof(double) * (size_t)m * m);
    for (int i = 0; i < m; i++) {
      K[(long)i * m + i] = 1.0;
      for (int j = 0; j < i; j++) {
        const double dx = Pmm[3 * i] - Pmm[3 * j], dy = Pmm[3 * i + 1] - Pmm[3 * j + 1],
                     dz = Pmm[3 * i + 2] - Pmm[3 * j + 2];
        const double v = rbf_d(sqrt(dx * dx + dy * dy + dz * dz), th);
        K[(long)i * m + j] = v; K[(long)j * m + i] = v;
      }
    }
  }

  /* bounding box + bounded nonzero ordinal map of the (masked) hr image
   * (nifti_manipulation.inl:244-275). */
  int bbmin[3], bbmax[3];
  if (orc_bounding_box(hr, nx, ny, nz, bbmin, bbmax) <= 0) { free(P); free(Pmm); free(K); return -5; }
  const int bd[3] = {bbmax[0] - bbmin[0] + 1, bbmax[1] - bbmin[1] + 1, bbmax[2] - bbmin[2] + 1};
  const long bprod = (long)bd[0] * bd[1] * bd[2];
  int* bmap = (int*)malloc(sizeof(int) * bprod);
  {
    int count = 0;
    for (int k = 0; k < bd[2]; k++)
      for (int j = 0; j < bd[1]; j++)
        for (int i = 0; i < bd[0]; i++) {
          const long ni = (long)(k + bbmin[2]) * nx * ny + (long)(j + bbmin[1]) * nx + (i + bbmin[0]);
          const long bi = (long)k * bd[0] * bd[1] + (long)j * bd[0] + i;
          bmap[bi] = is_nz(hr[ni]) ? count++ : -1;
        }
  }

  double Qh[16], Qs[16], Qhi[16], map[16];
  for (int i = 0; i < 16; i++) { Qh[i] = Qhr[i]; Qs[i] = Qsr[i]; }
  mat4_inverse(Qh, Qhi);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0.0;
      for (int k = 0; k < 4; k++) s += Qhi[4 * i + k] * Qs[4 * k + j];
      map[4 * i + j] = s;
    }

  const long nvox_s = (long)sx * sy * sz;
  /* phase 1: candidate columns, offsets and k' of every std-res row */
  long nrows_all = 0;
  for (long sidx = 0; sidx < nvox_s; sidx++) nrows_all += is_nz(sr[sidx]);
  if (nrows_all > max_rows) { free(P); free(Pmm); free(K); free(bmap); return -1; }
  int** rcols = (int**)calloc(nrows_all, sizeof(int*));
  int** rpid = (int**)calloc(nrows_all, sizeof(int*));
  double** rkp = (double**)calloc(nrows_all, sizeof(double*));
  double** rw = (double**)calloc(nrows_all, sizeof(double*));
  int* rcnt = (int*)calloc(nrows_all, sizeof(int));
  int* rkeep = (int*)malloc(sizeof(int) * nrows_all);
  int64_t status = 0;
  int row = 0;
  for (long sidx = 0; sidx < nvox_s && status == 0; sidx++) {
    if (!is_nz(sr[sidx])) continue;
    const double s[4] = {(double)(sidx % sx), (double)((sidx / sx) % sy), (double)(sidx / ((long)sx * sy)), 1.0};
    int base[3];
    double sm[3];
    for (int r = 0; r < 3; r++) {
      double a = 0.0, b = 0.0;
      for (int k = 0; k < 4; k++) { a += map[4 * r + k] * s[k]; b += Qs[4 * r + k] * s[k]; }
      base[r] = (int)a; /* truncation toward zero, kriging_matrix.h:255 */
      sm[r] = b;
    }
    rcols[row] = (int*)malloc(sizeof(int) * m);
    rpid[row] = (int*)malloc(sizeof(int) * m);
    rkp[row] = (double*)malloc(sizeof(double) * m);
    int cnt = 0;
    for (int j = 0; j < m; j++) {
      const int h0 = base[0] + P[3 * j], h1 = base[1] + P[3 * j + 1], h2 = base[2] + P[3 * j + 2];
      const long flat = (long)h2 * ny * nx + (long)h1 * nx + h0; /* flat-offset-only bound check */
      if (flat < 0 || flat >= nvox_hr) continue;
      if (!is_nz(hr[flat])) continue;
      const long bhr = (long)(h2 - bbmin[2]) * bd[0] * bd[1] + (long)(h1 - bbmin[1]) * bd[0] + (h0 - bbmin[0]);
      if (bhr < 0 || bhr >= bprod) { status = -3; break; }
      if (bmap[bhr] < 0) continue;
      rcols[row][cnt] = bmap[bhr];
      rpid[row][cnt] = j;
      double hm[3];
      for (int r = 0; r < 3; r++)
        hm[r] = Qh[4 * r + 0] * h0 + Qh[4 * r + 1] * h1 + Qh[4 * r + 2] * h2 + Qh[4 * r + 3];
      const double dx = sm[0] - hm[0], dy = sm[1] - hm[1], dz = sm[2] - hm[2];
      rkp[row][cnt] = rbf_d(sqrt(dx * dx + dy * dy + dz * dz) + 1e-5, th);
      cnt++;
    }
    rcnt[row] = cnt;
    rkeep[row] = 1;
    row++;
  }
  /* phase 2: K_sub w = k' per row (Cholesky; column-pivoted QR if K_sub is not
   * numerically positive definite).  Rows whose neighbourhood is complete share
   * K, so a row with the same k' as an earlier complete row reuses its w. */
  if (solve && status == 0) {
    int full_ref = -1;
    for (int r = 0; r < row; r++)
      if (rcnt[r] == m) { full_ref = r; break; }
#pragma omp parallel
    {
      double* A = (double*)malloc(sizeof(double) * (size_t)m * m);
      double* b = (double*)malloc(sizeof(double) * m);
#pragma omp for schedule(dynamic, 1)
      for (int r = -1; r < row; r++) {
        const int rr = r < 0 ? full_ref : r;
        if (rr < 0) continue;
        if (r >= 0 && rcnt[r] == m && full_ref >= 0 && r != full_ref &&
            memcmp(rkp[r], rkp[full_ref], sizeof(double) * m) == 0)
          continue; /* filled from the shared solution below */
        if (r >= 0 && r == full_ref) continue; /* solved by the r = -1 pass */
        const int cnt = rcnt[rr];
        if (cnt <= 0) continue;
        for (int a = 0; a < cnt; a++)
          for (int c = 0; c < cnt; c++) A[(long)a * cnt + c] = K[(long)rpid[rr][a] * m + rpid[rr][c]];
        double* w = (double*)malloc(sizeof(double) * cnt);
        memcpy(b, rkp[rr], sizeof(double) * cnt);
        if (cholesky_inplace(A, cnt)) {
          cholesky_solve_inplace(A, cnt, b);
          memcpy(w, b, sizeof(double) * cnt);
        } else {
          for (int a = 0; a < cnt; a++)
            for (int c = 0; c < cnt; c++) A[(long)a * cnt + c] = K[(long)rpid[rr][a] * m + rpid[rr][c]];
          memcpy(b, rkp[rr], sizeof(double) * cnt);
          colpiv_qr_solve(A, cnt, b, w);
        }
        rw[rr] = w;
      }
      free(A); free(b);
    }
    for (int r = 0; r < row; r++) {
      if (rcnt[r] == 0) continue;
      if (!rw[r]) {
        if (full_ref < 0 || !rw[full_ref]) { rkeep[r] = 0; continue; }
        rw[r] = (double*)malloc(sizeof(double) * m);
        memcpy(rw[r], rw[full_ref], sizeof(double) * m);
      }
      double wsum = 0.0;
      for (int a = 0; a < rcnt[r]; a++) wsum += rw[r][a];
      if (wsum == 0.0) wsum = 1.0;
      if (isnan(wsum)) rkeep[r] = 0;
      else for (int a = 0; a < rcnt[r]; a++) rw[r][a] /= wsum;
    }
  }
  /* phase 3: CSR */
  int64_t nnz = 0;
  rowptr[0] = 0;
  for (int r = 0; r < row && status == 0; r++) {
    const int keep = rkeep[r] ? rcnt[r] : 0;
    if (nnz + keep > max_nnz) { status = -1; break; }
    for (int a = 0; a < keep; a++) {
      col[nnz + a] = rcols[r][a];
      if (solve) val[nnz + a] = rw[r][a];
    }
    nnz += keep;
    rowptr[r + 1] = (int)nnz;
  }
  *n_rows_out = row;
  for (int r = 0; r < row; r++) { free(rcols[r]); free(rpid[r]); free(rkp[r]); free(rw[r]); }
  free(rcols); free(rpid); free(rkp); free(rw); free(rcnt); free(rkeep);
  free(P); free(Pmm); free(K); free(bmap);
  return status ? status : nnz;
}

/* ---------------------------- HMCParameters ------------------------------ */
/* HMCParameters.h:97-149.  The oracle mirrors the float build (value_type =
 * float), which rounds eps() and the sqrt(iteration) factor to float. */
int orc_hmc_init(orc_hmc* h, int burnin, int n_save, int thin, int L,
                 double starting_eps, double mh_target) {
  if (burnin < 0 || n_save < 0 || thin < 0 || L <= 0 || starting_eps <= 0 ||
      mh_target <= 0 || mh_target >= 1)
    return -1;
  memset(h, 0, sizeof(*h));
  h->warmup = burnin > 0;
  h->eps_start_found = !h->warmup;
  h->burnin = burnin;
  h->integrator_steps = L;
  h->iteration = 0;
  h->n_save = n_save;
  h->thin = (thin == 0) ? 1 : thin;
  h->A = 1;
  h->eps0 = 1e-5;
  h->eps = fmax((double)(float)starting_eps, h->eps0);
  h->eps_bar = 1;
  h->gamma = (double)0.05f;
  h->h_bar = 0;
  h->mh_running_sum = 0;
  h->mh_target = (double)(float)mh_target;
  h->t0 = 10;
  h->kappa = (double)0.75f;
  return 0;
}

/* HMCParameters.h:212-221 */
double orc_hmc_eps(const orc_hmc* h, double u01) {
  if (h->warmup) return (double)(float)h->eps;
  const double U = 0.9 + 0.2 * u01;
  return (double)(float)fmax(h->eps * U, h->eps0);
}

/* HMCParameters.h:172-179 */
int orc_hmc_integrator_steps(const orc_hmc* h) { return h->eps_start_found ? h->integrator_steps : 1; }

/* HMCParameters.h:158-161 */
int orc_hmc_save_iteration(const orc_hmc* h) {
  return (h->iteration > h->burnin) && ((h->iteration - h->burnin) % h->thin == 0);
}

int orc_hmc_max_iterations(const orc_hmc* h) { return h->burnin + h->thin * h->n_save; }

double orc_hmc_mh_rate(const orc_hmc* h) {
  const int d = h->iteration - h->burnin;
  return (double)(float)(h->mh_running_sum / (d > 1 ? d : 1));
}

/* HMCParameters.h:259-297 */
void orc_hmc_update(orc_hmc* h, double mh_rate_in) {
  const double mh_rate = (double)(float)mh_rate_in; /* value_type argument */
  if (h->iteration == h->burnin) {
    h->warmup = 0;
    h->eps_start_found = 1;
    if (h->eps_bar > h->eps0) h->eps = h->eps_bar;
  }
  if (h->warmup) {
    if (!h->eps_start_found) {
      if (h->iteration == 0) h->A = 2 * (int)(mh_rate > 0.5) - 1;
      if (pow(mh_rate, h->A) > pow(2.0, -h->A)) {
        h->eps *= pow(2.0, h->A);
      } else {
        h->eps_start_found = 1;
        h->eps_target = log(10.0 * h->eps);
      }
    } else {
      const double it = (double)h->iteration;
      h->h_bar = (1 - 1 / (it + h->t0)) * h->h_bar + (h->mh_target - mh_rate) / (it + h->t0);
      h->eps = exp(h->eps_target - (double)sqrtf((float)h->iteration) * h->h_bar / h->gamma);
      h->eps = fmax(h->eps, h->eps0);
      const double pk = pow((double)(float)h->iteration, -h->kappa);
      h->eps_bar = exp(pk * log(h->eps) + (1 - pk) * log(h->eps_bar));
    }
  } else {
    h->mh_running_sum += mh_rate;
  }
  h->iteration++;
}


/* ------------------------------------------------------------------ minimum contrast summary */
/* perturbation_matrix_3d (perturbation_matrix.h:62-109): 14 unit directions
 * (perturbations_3d_unit_directions, :19-38) times every (a, b, c) in
 * {1..18}^3 with a fastest (perturbation_permutations_3d, :44-56), then the
 * axis offsets 19..25, duplicates removed keeping the first. */
int orc_mce_offsets(int* P, int max_out) {
  static const int U[14][3] = {{0, 0, 0},  {1, 0, 0}, {0, 1, 0},  {0, 0, 1},  {1, 1, 0},  {1, 0, 1},   {-1, 1, 0},
                               {1, 0, -1}, {0, 1, 1}, {0, 1, -1}, {1, 1, 1},  {1, 1, -1}, {-1, 1, 1}, {-1, 1, -1}};
  const int n = 18, extra = 25 - 18;
  const int total = 14 * n * n * n + 3 * extra;
  int* all = (int*)malloc(sizeof(int) * 3 * total);
  int r = 0;
  for (int c = 1; c <= n; c++)
    for (int b = 1; b <= n; b++)
      for (int a = 1; a <= n; a++)
        for (int j = 0; j < 14; j++, r++) {
          all[3 * r] = U[j][0] * a;
          all[3 * r + 1] = U[j][1] * b;
          all[3 * r + 2] = U[j][2] * c;
        }
  for (int i = 0; i < extra; i++)
    for (int j = 0; j < 3; j++, r++) {
      all[3 * r] = all[3 * r + 1] = all[3 * r + 2] = 0;
      all[3 * r + j] = n + i + 1;
    }
  /* dedupe through a presence grid over [-25, 25]^3 */
  const int W = 51;
  unsigned char* seen = (unsigned char*)calloc(W * W * W, 1);
  int u = 0;
  for (int i = 0; i < total; i++) {
    const int key = ((all[3 * i + 2] + 25) * W + (all[3 * i + 1] + 25)) * W + (all[3 * i] + 25);
    if (seen[key]) continue;
    seen[key] = 1;
    if (P && u < max_out) {
      P[3 * u] = all[3 * i];
      P[3 * u + 1] = all[3 * i + 1];
      P[3 * u + 2] = all[3 * i + 2];
    }
    u++;
  }
  free(seen);
  free(all);
  return u;
}

/* compute_mce_summary_data_impl (estimate_kernel_parameters.h:50-101). */
int orc_mce_summary(const float* img, int nx, int ny, int nz, const float* Q, const int* P, int n_off,
                    float* distance, float* covariance, int* npairs, double* sums) {
  for (int o = 0; o < n_off; o++) {
    /* (P with a zero 4th column) * Q^T, row norm, in float */
    float s2 = 0.0f;
    for (int r = 0; r < 4; r++) {
      float t = 0.0f;
      for (int c = 0; c < 3; c++) t += (float)P[3 * o + c] * Q[4 * r + c];
      s2 += t * t;
    }
    distance[o] = sqrtf(s2);
  }
  const long long nxy = (long long)nx * ny;
#pragma omp parallel for schedule(dynamic, 16)
  for (int o = 0; o < n_off; o++) {
    const int dx = P[3 * o], dy = P[3 * o + 1], dz = P[3 * o + 2];
    double sxy = 0, sx = 0, sy = 0;
    int n = 0;
    for (int k = 0; k < nz; k++) {
      const int k2 = k + dz;
      if (k2 < 0 || k2 >= nz) continue;
      for (int j = 0; j < ny; j++) {
        const int j2 = j + dy;
        if (j2 < 0 || j2 >= ny) continue;
        const float* xr = img + k * nxy + (long long)j * nx;
        const float* yr = img + k2 * nxy + (long long)j2 * nx;
        for (int i = 0; i < nx; i++) {
          const int i2 = i + dx;
          if (i2 < 0 || i2 >= nx) continue;
          const double x = xr[i], y = yr[i2];
          if (isnan(x) || x == 0 || isnan(y) || y == 0) continue;
          sxy += x * y;
          sx += x;
          sy += y;
          n++;
        }
      }
    }
    npairs[o] = n;
    covariance[o] = n > 1 ? (float)((sxy - sx * sy / n) / (n - 1)) : 0.0f;
    if (sums) {
      sums[3 * o] = sxy;
      sums[3 * o + 1] = sx;
      sums[3 * o + 2] = sy;
    }
  }
  return 0;
}
