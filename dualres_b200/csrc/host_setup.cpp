// One-time host set-up of a volume (images -> indices -> kriging CSR).
//
// Restates src/dualgpm.cpp:125-245, 288 (masking, covariance checks, default
// neighbourhood), gaussian_process_model.h:104-117 (input bounding box, data
// and output indices), MultiResParameters.h:191-206, 287-289, 647-667 (grid,
// embedding, flat indices) and kriging_matrix.h:41-343 (the kriging matrix).
// The sparsity pattern follows the reference step by step (offset order,
// truncation, flat-offset bounds check, ordinal map), so it is bit-exact for
// inputs without borderline truncations.  The weights are solved in FP64
// (blocked Cholesky, column-pivoted Householder QR when the sub-matrix is not
// numerically positive definite) where the reference uses FP32
// colPivHouseholderQr.
#include "host_setup.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace drb {

static inline bool has_data(float v) { return !(std::isnan(v) || v == 0.0f); }

// ---------------------------------------------------------------- dense solves
// In-place lower Cholesky of the m x m row-major SPD matrix A (blocked,
// right-looking).  Returns false when a pivot is not positive.
static bool cholesky(double* A, int m) {
  const int NB = 64;
  for (int kb = 0; kb < m; kb += NB) {
    const int ke = std::min(m, kb + NB);
    for (int j = kb; j < ke; j++) {
      double* Aj = A + (size_t)j * m;
      double d = Aj[j];
      for (int p = kb; p < j; p++) d -= Aj[p] * Aj[p];
      if (!(d > 0.0)) return false;
      const double ljj = std::sqrt(d);
      Aj[j] = ljj;
      const double inv = 1.0 / ljj;
      for (int i = j + 1; i < m; i++) {
        double* Ai = A + (size_t)i * m;
        double s = Ai[j];
        for (int p = kb; p < j; p++) s -= Ai[p] * Aj[p];
        Ai[j] = s * inv;
      }
    }
    // trailing update A22 -= L21 L21^T (lower triangle), rows in groups of 4
    const int w = ke - kb;
    for (int i = ke; i < m; i += 4) {
      const int ni = std::min(4, m - i);
      const double* r[4];
      for (int t = 0; t < 4; t++) r[t] = A + (size_t)(i + std::min(t, ni - 1)) * m + kb;
      const int jmax = i + ni - 1;
      for (int j = ke; j <= jmax; j++) {
        const double* rj = A + (size_t)j * m + kb;
        double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        for (int p = 0; p < w; p++) {
          const double x = rj[p];
          s0 += r[0][p] * x;
          s1 += r[1][p] * x;
          s2 += r[2][p] * x;
          s3 += r[3][p] * x;
        }
        const double s[4] = {s0, s1, s2, s3};
        for (int t = 0; t < ni; t++)
          if (j <= i + t) A[(size_t)(i + t) * m + j] -= s[t];
      }
    }
  }
  return true;
}

// L L^T x = b with a row-major transposed copy Lt of L (contiguous backward pass).
static void cholesky_solve_t(const double* L, const double* Lt, int m, double* b) {
  for (int i = 0; i < m; i++) {
    const double* Li = L + (size_t)i * m;
    double s = b[i];
    for (int p = 0; p < i; p++) s -= Li[p] * b[p];
    b[i] = s / Li[i];
  }
  for (int i = m - 1; i >= 0; i--) {
    const double* Ti = Lt + (size_t)i * m;
    double s = b[i];
    for (int p = i + 1; p < m; p++) s -= Ti[p] * b[p];
    b[i] = s / Ti[i];
  }
}

static void cholesky_solve(const double* L, int m, double* b) {
  for (int i = 0; i < m; i++) {
    const double* Li = L + (size_t)i * m;
    double s = b[i];
    for (int p = 0; p < i; p++) s -= Li[p] * b[p];
    b[i] = s / Li[i];
  }
  for (int i = m - 1; i >= 0; i--) {
    double s = b[i];
    for (int p = i + 1; p < m; p++) s -= L[(size_t)p * m + i] * b[p];
    b[i] = s / L[(size_t)i * m + i];
  }
}

// Column-pivoted Householder QR solve (A destroyed); components beyond the
// numerical rank are zero (basic solution).
static void qr_solve(double* A, int m, double* b, double* x) {
  std::vector<int> perm(m);
  std::vector<double> v(m), y(m, 0.0);
  for (int j = 0; j < m; j++) perm[j] = j;
  int rank = m;
  double r00 = 0.0;
  for (int k = 0; k < m; k++) {
    int best = k;
    double bn = -1.0;
    for (int j = k; j < m; j++) {
      double s = 0.0;
      for (int i = k; i < m; i++) s += A[(size_t)i * m + j] * A[(size_t)i * m + j];
      if (s > bn) { bn = s; best = j; }
    }
    if (best != k) {
      for (int i = 0; i < m; i++) std::swap(A[(size_t)i * m + k], A[(size_t)i * m + best]);
      std::swap(perm[k], perm[best]);
    }
    double alpha = std::sqrt(bn);
    if (k == 0) r00 = alpha;
    if (alpha <= (double)m * 2.220446049250313e-16 * r00) { rank = k; break; }
    if (A[(size_t)k * m + k] > 0) alpha = -alpha;
    double vn = 0.0;
    for (int i = k; i < m; i++) v[i] = A[(size_t)i * m + k];
    v[k] -= alpha;
    for (int i = k; i < m; i++) vn += v[i] * v[i];
    if (vn > 0.0) {
      for (int j = k; j < m; j++) {
        double s = 0.0;
        for (int i = k; i < m; i++) s += v[i] * A[(size_t)i * m + j];
        s = 2.0 * s / vn;
        for (int i = k; i < m; i++) A[(size_t)i * m + j] -= s * v[i];
      }
      double s = 0.0;
      for (int i = k; i < m; i++) s += v[i] * b[i];
      s = 2.0 * s / vn;
      for (int i = k; i < m; i++) b[i] -= s * v[i];
    }
  }
  for (int i = rank - 1; i >= 0; i--) {
    double s = b[i];
    for (int j = i + 1; j < rank; j++) s -= A[(size_t)i * m + j] * y[j];
    y[i] = s / A[(size_t)i * m + i];
  }
  for (int j = 0; j < m; j++) x[perm[j]] = y[j];
}

static double rbf(double d, const double* th) { return th[0] * std::exp(-th[1] * std::pow(std::fabs(d), th[2])); }

// ---------------------------------------------------------------- neighbourhood
// kriging_matrix.h:63-106 in float arithmetic (voxel dims = column norms of Q,
// nifti_manipulation.inl:600-605), offsets i fastest (kriging_matrix.h:41-56).
static int neighbourhood(const float* Q, float radius, std::vector<int>* P) {
  float vd[3];
  int nr[3];
  for (int c = 0; c < 3; c++) {
    float s = 0.0f;
    for (int r = 0; r < 4; r++) s += Q[4 * r + c] * Q[4 * r + c];
    vd[c] = std::sqrt(s);
    nr[c] = (int)(radius / vd[c]);
  }
  P->clear();
  long total = 0, inside = 0;
  for (int k = -nr[2]; k <= nr[2]; k++)
    for (int j = -nr[1]; j <= nr[1]; j++)
      for (int i = -nr[0]; i <= nr[0]; i++) {
        total++;
        float q2 = 0.0f;
        for (int r = 0; r < 3; r++) {
          const float q = Q[4 * r + 0] * (float)i + Q[4 * r + 1] * (float)j + Q[4 * r + 2] * (float)k;
          q2 += q * q;
        }
        if (std::sqrt(q2) <= radius) {
          P->push_back(i); P->push_back(j); P->push_back(k);
          inside++;
        }
      }
  return (int)inside;
}

static void mat4_inverse(const double* a, double* inv) {
  double m[4][8];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) { m[i][j] = a[4 * i + j]; m[i][j + 4] = i == j ? 1.0 : 0.0; }
  for (int c = 0; c < 4; c++) {
    int p = c;
    for (int r = c + 1; r < 4; r++) if (std::fabs(m[r][c]) > std::fabs(m[p][c])) p = r;
    if (p != c) for (int j = 0; j < 8; j++) std::swap(m[c][j], m[p][j]);
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

int kriging_plan(const float* hr, int nx, int ny, int nz, const float* Qhr, const float* sr, int sx, int sy, int sz,
                 const float* Qsr, const float* theta, float radius, KrigingPlan* plan, int* n_offsets,
                 std::string* err, bool host_inverse) {
  if (radius < 0) { *err = "neighborhood_perturbation: radius cannot be negative"; return DR_ERR_INVALID; }
  std::vector<int> P;
  const int m = neighbourhood(Qhr, radius, &P);
  *n_offsets = m;
  if (m == 0) { *err = "neighborhood_perturbation: no perturbations within radius"; return DR_ERR_DOMAIN; }
  if (m > 5000) { *err = "get_sparse_kriging_array_data: neighborhood >5e3 voxels"; return DR_ERR_DOMAIN; }
  const double th[3] = {theta[0], theta[1], theta[2]};
  // K over the offsets (kriging_matrix.h:111-138): unit diagonal.
  std::vector<double> Pm(3 * (size_t)m);
  std::vector<double>& K = plan->K;
  K.assign((size_t)m * m, 0.0);
  for (int i = 0; i < m; i++)
    for (int r = 0; r < 3; r++)
      Pm[3 * i + r] = (double)Qhr[4 * r] * P[3 * i] + (double)Qhr[4 * r + 1] * P[3 * i + 1] +
                      (double)Qhr[4 * r + 2] * P[3 * i + 2];
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < m; i++) {
    K[(size_t)i * m + i] = 1.0;
    for (int j = 0; j < i; j++) {
      const double dx = Pm[3 * i] - Pm[3 * j], dy = Pm[3 * i + 1] - Pm[3 * j + 1], dz = Pm[3 * i + 2] - Pm[3 * j + 2];
      const double v = rbf(std::sqrt(dx * dx + dy * dy + dz * dz), th);
      K[(size_t)i * m + j] = v;
      K[(size_t)j * m + i] = v;
    }
  }
  // bounded nonzero ordinal map of the high-res image (nifti_manipulation.inl:244-275)
  int bbmin[3] = {nx, ny, nz}, bbmax[3] = {-1, -1, -1};
  const long nvox = (long)nx * ny * nz;
  for (long idx = 0; idx < nvox; idx++) {
    if (!has_data(hr[idx])) continue;
    const int ii[3] = {(int)(idx % nx), (int)((idx / nx) % ny), (int)(idx / ((long)nx * ny))};
    for (int d = 0; d < 3; d++) { bbmin[d] = std::min(bbmin[d], ii[d]); bbmax[d] = std::max(bbmax[d], ii[d]); }
  }
  if (bbmax[0] < 0) { *err = "kriging: high-res image has no data"; return DR_ERR_INVALID; }
  const int bd[3] = {bbmax[0] - bbmin[0] + 1, bbmax[1] - bbmin[1] + 1, bbmax[2] - bbmin[2] + 1};
  const long bprod = (long)bd[0] * bd[1] * bd[2];
  std::vector<int> bmap(bprod);
  {
    int count = 0;
    for (int k = 0; k < bd[2]; k++)
      for (int j = 0; j < bd[1]; j++)
        for (int i = 0; i < bd[0]; i++) {
          const long ni = (long)(k + bbmin[2]) * nx * ny + (long)(j + bbmin[1]) * nx + (i + bbmin[0]);
          bmap[(long)k * bd[0] * bd[1] + (long)j * bd[0] + i] = has_data(hr[ni]) ? count++ : -1;
        }
  }
  double Qh[16], Qs[16], Qhi[16], mp[16];
  for (int i = 0; i < 16; i++) { Qh[i] = Qhr[i]; Qs[i] = Qsr[i]; }
  mat4_inverse(Qh, Qhi);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0.0;
      for (int k = 0; k < 4; k++) s += Qhi[4 * i + k] * Qs[4 * k + j];
      mp[4 * i + j] = s;
    }
  // std-res rows in column-major nonzero order (nifti_manipulation.inl:335-360)
  std::vector<long> rows;
  const long nvs = (long)sx * sy * sz;
  for (long s = 0; s < nvs; s++)
    if (has_data(sr[s])) rows.push_back(s);
  const int nrows = (int)rows.size();
  int bad = 0;
  // candidates per row (kriging_matrix.h:242-299), enumerated twice: a counting pass sizes the rows, then each row
  // is written straight into its place in the flat arrays
  auto row_frame = [&](int ri, int base[3], double sm[3]) {
    const long sidx = rows[ri];
    const double s[4] = {(double)(sidx % sx), (double)((sidx / sx) % sy), (double)(sidx / ((long)sx * sy)), 1.0};
    for (int r = 0; r < 3; r++) {
      double a = 0.0, b = 0.0;
      for (int k = 0; k < 4; k++) { a += mp[4 * r + k] * s[k]; b += Qs[4 * r + k] * s[k]; }
      base[r] = (int)a;  // truncation toward zero (kriging_matrix.h:255)
      sm[r] = b;
    }
  };
  // ordinal of candidate j of a row at `base`, -1 when absent, -2 when outside the bounded map
  auto candidate = [&](const int base[3], int j, int* h) -> int {
    h[0] = base[0] + P[3 * j];
    h[1] = base[1] + P[3 * j + 1];
    h[2] = base[2] + P[3 * j + 2];
    const long flat = (long)h[2] * ny * nx + (long)h[1] * nx + h[0];  // flat-offset-only check (:263-266)
    if (flat < 0 || flat >= nvox || !has_data(hr[flat])) return -1;
    const long b = (long)(h[2] - bbmin[2]) * bd[0] * bd[1] + (long)(h[1] - bbmin[1]) * bd[0] + (h[0] - bbmin[0]);
    if (b < 0 || b >= bprod) return -2;
    return bmap[b];
  };
  plan->row_start.assign(nrows + 1, 0);
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : bad)
  for (int ri = 0; ri < nrows; ri++) {
    int base[3], h[3];
    double sm[3];
    row_frame(ri, base, sm);
    int n = 0;
    for (int j = 0; j < m; j++) {
      const int o = candidate(base, j, h);
      if (o == -2) bad++;
      n += o >= 0;
    }
    plan->row_start[ri + 1] = n;
  }
  if (bad) {
    *err = "kriging: a neighbourhood index falls outside the bounded high-res index map (undefined in the reference)";
    return DR_ERR_DOMAIN;
  }
  // S = K^-1 once per volume (FP64).  A row with present offsets A and absent
  // offsets B then has (K_AA)^-1 = S_AA - S_AB (S_BB)^-1 S_BA, which costs
  // O(|A|^2 + |B|^3) instead of the O(|A|^3) of a direct solve; each row takes
  // the cheaper route.  Not positive definite K (variance > 1) -> direct solves.
  std::vector<double>& Sinv = plan->S;
  Sinv.clear();
  bool have_inv = false;
  plan->inverse_wanted = !std::getenv("DRB_KRIGING_DIRECT");
  if (plan->inverse_wanted && host_inverse) {
    std::vector<double> Lf(K);
    if (cholesky(Lf.data(), m)) {
      Sinv.assign((size_t)m * m, 0.0);
      std::vector<double> Lt((size_t)m * m, 0.0);
      for (int i = 0; i < m; i++)
        for (int j = 0; j <= i; j++) Lt[(size_t)j * m + i] = Lf[(size_t)i * m + j];
#pragma omp parallel
      {
        std::vector<double> e(m);
#pragma omp for schedule(dynamic, 8)
        for (int j = 0; j < m; j++) {
          std::fill(e.begin(), e.end(), 0.0);
          e[j] = 1.0;
          cholesky_solve_t(Lf.data(), Lt.data(), m, e.data());
          for (int i = 0; i < m; i++) Sinv[(size_t)i * m + j] = e[i];
        }
      }
      // symmetrise (the two triangular solves leave O(eps) asymmetry)
      for (int i = 0; i < m; i++)
        for (int j = 0; j < i; j++) {
          const double a = 0.5 * (Sinv[(size_t)i * m + j] + Sinv[(size_t)j * m + i]);
          Sinv[(size_t)i * m + j] = Sinv[(size_t)j * m + i] = a;
        }
      have_inv = true;
    }
  }
  (void)have_inv;
  plan->m = m;
  plan->nrows = nrows;
  for (int ri = 0; ri < nrows; ri++) plan->row_start[ri + 1] += plan->row_start[ri];
  const size_t tot = (size_t)plan->row_start[nrows];
  plan->pid.resize(tot);
  plan->col.resize(tot);
  plan->kp.resize(tot);
#pragma omp parallel for schedule(dynamic, 16)
  for (int ri = 0; ri < nrows; ri++) {
    int base[3], h[3];
    double sm[3];
    row_frame(ri, base, sm);
    size_t o = (size_t)plan->row_start[ri];
    for (int j = 0; j < m; j++) {
      const int c = candidate(base, j, h);
      if (c < 0) continue;
      plan->col[o] = c;
      plan->pid[o] = j;
      double hm[3];
      for (int r = 0; r < 3; r++) hm[r] = Qh[4 * r] * h[0] + Qh[4 * r + 1] * h[1] + Qh[4 * r + 2] * h[2] + Qh[4 * r + 3];
      const double dx = sm[0] - hm[0], dy = sm[1] - hm[1], dz = sm[2] - hm[2];
      plan->kp[o] = rbf(std::sqrt(dx * dx + dy * dy + dz * dz) + 1e-5, th);
      o++;
    }
  }
  return DR_OK;
}

// One row of the host solve: Schur route or direct Cholesky, QR when the
// direct system is not numerically positive definite.  x gets the normalised
// weights; false when the weight sum is NaN (the row is dropped).
bool kriging_solve_row_host(const KrigingPlan& plan, int ri, std::vector<double>* xout) {
  const int m = plan.m;
  const std::vector<double>& K = plan.K;
  const std::vector<double>& Sinv = plan.S;
  const bool have_inv = !Sinv.empty();
  const int r0 = plan.row_start[ri];
  const int cnt = plan.row_start[ri + 1] - r0;
  const double* k = plan.kp.data() + r0;
  const int* pid = plan.pid.data() + r0;
  std::vector<double> A, b(k, k + cnt), x(cnt, 0.0);
  const int nb = m - cnt;
  bool solved = false;
  if (kriging_schur_route(cnt, m, have_inv)) {
    // Schur route: w = S_AA k - S_AB (S_BB^-1 (S_BA k))
    std::vector<char> present(m, 0);
    for (int a = 0; a < cnt; a++) present[pid[a]] = 1;
    std::vector<int> B;
    B.reserve(nb);
    for (int j = 0; j < m; j++)
      if (!present[j]) B.push_back(j);
    std::vector<double> t(nb, 0.0);
    for (int q = 0; q < nb; q++) {
      const double* Srow = Sinv.data() + (size_t)B[q] * m;
      double acc = 0.0;
      for (int a = 0; a < cnt; a++) acc += Srow[pid[a]] * k[a];
      t[q] = acc;
    }
    A.resize((size_t)nb * nb);
    for (int q = 0; q < nb; q++)
      for (int r = 0; r < nb; r++) A[(size_t)q * nb + r] = Sinv[(size_t)B[q] * m + B[r]];
    if (nb == 0 || cholesky(A.data(), nb)) {
      if (nb > 0) cholesky_solve(A.data(), nb, t.data());
      for (int a = 0; a < cnt; a++) {
        const double* Srow = Sinv.data() + (size_t)pid[a] * m;
        double acc = 0.0;
        for (int c = 0; c < cnt; c++) acc += Srow[pid[c]] * k[c];
        for (int q = 0; q < nb; q++) acc -= Srow[B[q]] * t[q];
        x[a] = acc;
      }
      solved = true;
    }
  }
  if (!solved) {
    A.resize((size_t)cnt * cnt);
    for (int a = 0; a < cnt; a++)
      for (int c = 0; c < cnt; c++) A[(size_t)a * cnt + c] = K[(size_t)pid[a] * m + pid[c]];
    if (cholesky(A.data(), cnt)) {
      cholesky_solve(A.data(), cnt, b.data());
      x = b;
    } else {
      for (int a = 0; a < cnt; a++)
        for (int c = 0; c < cnt; c++) A[(size_t)a * cnt + c] = K[(size_t)pid[a] * m + pid[c]];
      b.assign(k, k + cnt);
      qr_solve(A.data(), cnt, b.data(), x.data());
    }
  }
  double wsum = 0.0;
  for (int a = 0; a < cnt; a++) wsum += x[a];
  if (wsum == 0.0) wsum = 1.0;  // kriging_matrix.h:318-319
  if (std::isnan(wsum)) return false;
  for (int a = 0; a < cnt; a++) x[a] /= wsum;
  *xout = std::move(x);
  return true;
}

void kriging_solve_host(const KrigingPlan& plan, std::vector<int>* rowptr, fill_vector<int>* col,
                        fill_vector<float>* val) {
  const int m = plan.m, nrows = plan.nrows;
  // Rows whose neighbourhood is complete share K; identical k' then share w.
  std::map<std::vector<double>, std::vector<double>> full_cache;
  std::mutex cache_mtx;
  std::vector<std::vector<double>> rw(nrows);
  std::vector<char> keep(nrows, 1);
#pragma omp parallel for schedule(dynamic, 1)
  for (int ri = 0; ri < nrows; ri++) {
    const int r0 = plan.row_start[ri];
    const int cnt = plan.row_start[ri + 1] - r0;
    if (cnt == 0) continue;
    std::vector<double> krow;
    if (cnt == m) {
      krow.assign(plan.kp.begin() + r0, plan.kp.begin() + r0 + cnt);
      std::lock_guard<std::mutex> lk(cache_mtx);
      auto it = full_cache.find(krow);
      if (it != full_cache.end()) {
        rw[ri] = it->second;
        continue;
      }
    }
    std::vector<double> x;
    if (!kriging_solve_row_host(plan, ri, &x)) {
      keep[ri] = 0;
      continue;
    }
    rw[ri] = x;
    if (cnt == m) {
      std::lock_guard<std::mutex> lk(cache_mtx);
      full_cache.emplace(krow, x);
    }
  }
  std::vector<double> flat(plan.col.size(), 0.0);
  for (int ri = 0; ri < nrows; ri++)
    if (keep[ri]) std::copy(rw[ri].begin(), rw[ri].end(), flat.begin() + plan.row_start[ri]);
  kriging_assemble(plan, flat.data(), keep, rowptr, col, val);
}

void kriging_assemble(const KrigingPlan& plan, const double* w, const std::vector<char>& keep,
                      std::vector<int>* rowptr, fill_vector<int>* col, fill_vector<float>* val) {
  rowptr->assign(plan.nrows + 1, 0);
  for (int ri = 0; ri < plan.nrows; ri++) {
    const int n = plan.row_start[ri + 1] - plan.row_start[ri];
    (*rowptr)[ri + 1] = (*rowptr)[ri] + (keep[ri] ? n : 0);
  }
  col->resize((size_t)(*rowptr)[plan.nrows]);
  val->resize((size_t)(*rowptr)[plan.nrows]);
#pragma omp parallel for schedule(dynamic, 64)
  for (int ri = 0; ri < plan.nrows; ri++) {
    if (!keep[ri]) continue;
    const int r0 = plan.row_start[ri], r1 = plan.row_start[ri + 1], o = (*rowptr)[ri];
    for (int k = r0; k < r1; k++) {
      (*col)[o + k - r0] = plan.col[k];
      (*val)[o + k - r0] = (float)w[k];
    }
  }
}

int kriging_build(const float* hr, int nx, int ny, int nz, const float* Qhr, const float* sr, int sx, int sy, int sz,
                  const float* Qsr, const float* theta, float radius, std::vector<int>* rowptr, std::vector<int>* col,
                  std::vector<float>* val, int* n_offsets, std::string* err) {
  KrigingPlan plan;
  const int rc = kriging_plan(hr, nx, ny, nz, Qhr, sr, sx, sy, sz, Qsr, theta, radius, &plan, n_offsets, err);
  if (rc != DR_OK) return rc;
  fill_vector<int> c;
  fill_vector<float> v;
  kriging_solve_host(plan, rowptr, &c, &v);
  col->assign(c.begin(), c.end());
  val->assign(v.begin(), v.end());
  return DR_OK;
}


// ---------------------------------------------------------------- preparation
void build_transpose(HostVolume* hv) {
  const int n_h = (int)hv->Yh.size(), n_s = (int)hv->Ys.size();
  const size_t nnz = hv->w_col.size();
  hv->wt_rowptr.assign(n_h + 1, 0);
  hv->wt_col.resize(nnz);
  hv->wt_val.resize(nnz);
  // Counting sort by column over T contiguous chunks of W's rows: chunk t's entries of column c land after those
  // of chunks 0..t-1, so every row of W^T lists its std-res rows in ascending order, as a serial pass would.
  int T = 1;
#ifdef _OPENMP
  T = std::max(1, std::min(omp_get_max_threads(), n_s / 256));
#endif
  std::vector<int> cnt((size_t)T * n_h, 0);
  auto chunk = [&](int t, int* r0, int* r1) {
    *r0 = (int)((long long)n_s * t / T);
    *r1 = (int)((long long)n_s * (t + 1) / T);
  };
#pragma omp parallel for num_threads(T) schedule(static, 1)
  for (int t = 0; t < T; t++) {
    int r0, r1;
    chunk(t, &r0, &r1);
    int* ct = cnt.data() + (size_t)t * n_h;
    for (int k = hv->w_rowptr[r0]; k < hv->w_rowptr[r1]; k++) ct[hv->w_col[k]]++;
  }
  // column totals, then each chunk's start within each column
  for (int c = 0; c < n_h; c++) {
    int run = 0;
    for (int t = 0; t < T; t++) {
      const int v = cnt[(size_t)t * n_h + c];
      cnt[(size_t)t * n_h + c] = run;
      run += v;
    }
    hv->wt_rowptr[c + 1] = run;
  }
  for (int i = 0; i < n_h; i++) hv->wt_rowptr[i + 1] += hv->wt_rowptr[i];
#pragma omp parallel for num_threads(T) schedule(static, 1)
  for (int t = 0; t < T; t++) {
    int r0, r1;
    chunk(t, &r0, &r1);
    int* ct = cnt.data() + (size_t)t * n_h;
    for (int r = r0; r < r1; r++)
      for (int k = hv->w_rowptr[r]; k < hv->w_rowptr[r + 1]; k++) {
        const int c = hv->w_col[k];
        const int at = hv->wt_rowptr[c] + ct[c]++;
        hv->wt_col[at] = r;
        hv->wt_val[at] = hv->w_val[k];
      }
  }
}

uint32_t zorder_key(int x, int y, int z) {
  uint32_t k = 0;
  for (int b = 0; b < 10; b++)
    k |= ((uint32_t)((x >> b) & 1) << (3 * b)) | ((uint32_t)((y >> b) & 1) << (3 * b + 1)) |
         ((uint32_t)((z >> b) & 1) << (3 * b + 2));
  return k;
}

bool tc_plan(const std::vector<int>& rowptr, const int* col, size_t nnz, const std::vector<uint32_t>& key, int g_max,
             TcPlanHost* P) {
  constexpr int M = 128, KC = 32, BLK = M * KC;
  const int R = (int)rowptr.size() - 1;
  std::vector<int> order(R);
  for (int i = 0; i < R; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
  P->T = (R + M - 1) / M;
  P->tile_rows.assign((size_t)P->T * M, -1);
  for (int i = 0; i < R; i++) P->tile_rows[i] = order[i];
  int n_cols = 0;
  for (size_t k = 0; k < nnz; k++) n_cols = std::max(n_cols, col[k] + 1);
  // per tile: the sorted union of its rows' columns (a per-thread stamp array marks columns already taken)
  std::vector<std::vector<int>> uni(P->T);
#pragma omp parallel
  {
    std::vector<int> stamp(n_cols, -1);
#pragma omp for schedule(dynamic, 1)
    for (int t = 0; t < P->T; t++) {
      std::vector<int>& u = uni[t];
      for (int m = 0; m < M; m++) {
        const int r = P->tile_rows[(size_t)t * M + m];
        if (r < 0) continue;
        for (int k = rowptr[r]; k < rowptr[r + 1]; k++)
          if (stamp[col[k]] != t) {
            stamp[col[k]] = t;
            u.push_back(col[k]);
          }
      }
      std::sort(u.begin(), u.end());
    }
  }
  std::vector<long long> chunk_ptr(P->T + 1, 0);
  for (int t = 0; t < P->T; t++) chunk_ptr[t + 1] = chunk_ptr[t] + (long long)(uni[t].size() + KC - 1) / KC;
  P->chunks = chunk_ptr[P->T];
  if (P->chunks * BLK > 0x7fffffffLL) return false;
  P->chunk_cols.assign((size_t)P->chunks * KC, -1);
  P->dest.resize(nnz);
#pragma omp parallel
  {
    std::vector<int> pos(n_cols, 0);
#pragma omp for schedule(dynamic, 1)
    for (int t = 0; t < P->T; t++) {
      const std::vector<int>& u = uni[t];
      std::copy(u.begin(), u.end(), P->chunk_cols.begin() + chunk_ptr[t] * KC);
      for (int i = 0; i < (int)u.size(); i++) pos[u[i]] = i;
      for (int m = 0; m < M; m++) {
        const int r = P->tile_rows[(size_t)t * M + m];
        if (r < 0) continue;
        for (int k = rowptr[r]; k < rowptr[r + 1]; k++) {
          const long long p = pos[col[k]];
          const long long q = chunk_ptr[t] + p / KC;
          const int kk = (int)(p % KC);
          P->dest[k] = (int)(q * BLK + (kk / 4) * (M * 4) + m * 4 + kk % 4);
        }
      }
    }
  }
  const long long Q = P->chunks;
  P->G = Q == 0 ? 0 : (int)std::min<long long>(Q, std::max(1, g_max));
  P->segs.clear();
  P->cta_seg_ptr.assign(P->G + 1, 0);
  int t = 0;
  for (int b = 0; b < P->G; b++) {
    long long c0 = Q * b / P->G;
    const long long c1 = Q * (b + 1) / P->G;
    while (c0 < c1) {
      while (chunk_ptr[t + 1] <= c0) t++;
      const long long e = std::min(c1, chunk_ptr[t + 1]);
      P->segs.insert(P->segs.end(), {t, (int)c0, (int)e, 0});
      c0 = e;
    }
    P->cta_seg_ptr[b + 1] = (int)(P->segs.size() / 4);
  }
  const int ns = (int)(P->segs.size() / 4);
  P->tile_seg_ptr.assign(P->T + 1, ns);
  for (int tt = P->T - 1, g = ns - 1; tt >= 0; tt--) {
    while (g >= 0 && P->segs[4 * g] >= tt) g--;
    P->tile_seg_ptr[tt] = g + 1;
  }
  return true;
}

int host_prepare(const dr_volume_desc* d, HostVolume* hv, std::string* err, bool defer_kriging) {
  if (!d || !d->highres || !d->qform_hr || d->nx <= 0 || d->ny <= 0 || d->nz <= 0) {
    *err = "dr_volume_create: highres image and qform are required";
    return DR_ERR_INVALID;
  }
  const int nx = d->nx, ny = d->ny, nz_ = d->nz;
  const long nvox = (long)nx * ny * nz_;
  // covariance checks (dualgpm.cpp:447-464)
  const float* th = d->covariance;
  if (!(th[0] > 0)) { *err = "First covariance parameter (marginal variance) must be > 0"; return DR_ERR_DOMAIN; }
  if (!(th[1] > 0)) { *err = "Second covariance parameter (bandwidth) must be > 0"; return DR_ERR_DOMAIN; }
  if (!(th[2] > 0 && th[2] <= 2)) { *err = "Third covariance parameter (exponent) must be in (0, 2]"; return DR_ERR_DOMAIN; }
  if (d->covfun != DR_COV_RBF && d->covfun != DR_COV_RQ) { *err = "Unknown covariance function"; return DR_ERR_DOMAIN; }
  for (int i = 0; i < 3; i++) hv->theta[i] = th[i];
  hv->covfun = d->covfun;
  std::memcpy(hv->Q, d->qform_hr, sizeof(float) * 16);

  // masks (dualgpm.cpp:126-155, 288; both default to the high-res image)
  std::vector<float> hr(d->highres, d->highres + nvox);
  std::vector<float> hm(d->hmask ? d->hmask : d->highres, (d->hmask ? d->hmask : d->highres) + nvox);
  const float* om = d->omask ? d->omask : d->highres;
  for (long i = 0; i < nvox; i++)
    if (hm[i] == 0.0f || std::isnan(hr[i])) hr[i] = 0.0f;
  for (long i = 0; i < nvox; i++) hm[i] += om[i];
  int bbmin[3] = {nx, ny, nz_}, bbmax[3] = {-1, -1, -1};
  for (long idx = 0; idx < nvox; idx++) {
    if (!has_data(hm[idx])) continue;
    const int ii[3] = {(int)(idx % nx), (int)((idx / nx) % ny), (int)(idx / ((long)nx * ny))};
    for (int k = 0; k < 3; k++) { bbmin[k] = std::min(bbmin[k], ii[k]); bbmax[k] = std::max(bbmax[k], ii[k]); }
  }
  if (bbmax[0] < 0) { *err = "dr_volume_create: the masks select no voxel"; return DR_ERR_INVALID; }
  std::vector<int> D, O;
  for (long idx = 0; idx < nvox; idx++) {
    const int ii[3] = {(int)(idx % nx), (int)((idx / nx) % ny), (int)(idx / ((long)nx * ny))};
    const bool inbox = ii[0] >= bbmin[0] && ii[0] <= bbmax[0] && ii[1] >= bbmin[1] && ii[1] <= bbmax[1] &&
                       ii[2] >= bbmin[2] && ii[2] <= bbmax[2];
    if (has_data(hr[idx])) {
      hv->Yh.push_back(hr[idx]);
      if (inbox) for (int k = 0; k < 3; k++) D.push_back(ii[k] - bbmin[k]);
    }
    if (has_data(om[idx]) && inbox) for (int k = 0; k < 3; k++) O.push_back(ii[k] - bbmin[k]);
  }
  const int n_h = (int)D.size() / 3, n_o = (int)O.size() / 3;
  if (n_h == 0) { *err = "dr_volume_create: no high-res data"; return DR_ERR_INVALID; }
  if ((int)hv->Yh.size() != n_h) { *err = "dr_volume_create: data voxels outside the mask bounding box"; return DR_ERR_INVALID; }
  for (int k = 0; k < 3; k++) hv->g[k] = 0;
  for (int i = 0; i < n_h; i++) for (int k = 0; k < 3; k++) hv->g[k] = std::max(hv->g[k], D[3 * i + k] + 1);
  for (int k = 0; k < 3; k++) {
    if (hv->g[k] <= 1) { *err = "circulant_base_3d: Cannot have dimensions <= 1"; return DR_ERR_DOMAIN; }
    int p = 1;
    while (p < 2 * (hv->g[k] - 1)) p <<= 1;
    hv->E[k] = p;
    if (p > 256) { *err = "dr_volume_create: embedding dimension above 256 is not supported"; return DR_ERR_UNSUPPORTED; }
  }
  hv->N = (long long)hv->E[0] * hv->E[1] * hv->E[2];
  if (hv->N > (1LL << 30)) { *err = "dr_volume_create: embedding too large"; return DR_ERR_UNSUPPORTED; }
  // output indices must lie on the embedding (MultiResParameters.h:647-667)
  for (int i = 0; i < n_o; i++)
    for (int k = 0; k < 3; k++)
      if (O[3 * i + k] >= hv->E[k]) { *err = "MultiResParameters:set_output_indices MAX"; return DR_ERR_DOMAIN; }
  for (int k = 0; k < 3; k++) {
    int b = hv->g[k];
    for (int i = 0; i < n_o; i++) b = std::max(b, O[3 * i + k] + 1);
    hv->box[k] = b;
  }
  // even x-extent: every z-plane of the pruned intermediate then starts on a
  // 16-byte boundary (bulk copies need that); E0 is even, so bx stays <= E0
  hv->box[0] += hv->box[0] & 1;
  const int bx = hv->box[0], by = hv->box[1], bz = hv->box[2];
  hv->box_to_d.assign((size_t)bx * by * bz, -1);
  hv->box_to_o.assign((size_t)bx * by * bz, -1);
  hv->d_flat.resize(n_h);
  hv->o_flat.resize(n_o);
  for (int i = 0; i < n_h; i++) {
    const int x = D[3 * i], y = D[3 * i + 1], z = D[3 * i + 2];
    hv->d_flat[i] = (z * hv->E[1] + y) * hv->E[0] + x;
    hv->box_to_d[((size_t)z * by + y) * bx + x] = i;
  }
  for (int i = 0; i < n_o; i++) {
    const int x = O[3 * i], y = O[3 * i + 1], z = O[3 * i + 2];
    hv->o_flat[i] = (z * hv->E[1] + y) * hv->E[0] + x;
    hv->box_to_o[((size_t)z * by + y) * bx + x] = i;
  }

  // std-res data and kriging matrix (dualgpm.cpp:166-227, MultiResData.h:96-127)
  if (d->stdres) {
    if (!d->qform_sr || d->sx <= 0 || d->sy <= 0 || d->sz <= 0) {
      *err = "dr_volume_create: stdres requires its grid and qform";
      return DR_ERR_INVALID;
    }
    const long nvs = (long)d->sx * d->sy * d->sz;
    std::vector<float> sr(d->stdres, d->stdres + nvs);
    if (d->smask)
      for (long i = 0; i < nvs; i++)
        if (d->smask[i] == 0.0f || std::isnan(sr[i])) sr[i] = 0.0f;
    for (long i = 0; i < nvs; i++)
      if (has_data(sr[i])) hv->Ys.push_back(sr[i]);
    float radius = d->neighborhood;
    if (radius <= 0) {
      float vmax = 0.f;
      for (int c = 0; c < 3; c++) {
        float s = 0.f;
        for (int r = 0; r < 4; r++) s += d->qform_hr[4 * r + c] * d->qform_hr[4 * r + c];
        vmax = std::max(vmax, std::sqrt(s));
      }
      radius = 3.0f * vmax;
    }
    hv->radius = radius;
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = kriging_plan(hr.data(), nx, ny, nz_, d->qform_hr, sr.data(), d->sx, d->sy, d->sz, d->qform_sr,
                                d->covariance, radius, &hv->kplan, &hv->n_offsets, err, !defer_kriging);
    if (rc != DR_OK) return rc;
    hv->kriging_plan_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int c : hv->kplan.col)
      if (c < 0 || c >= n_h) { *err = "kriging: column outside the data range"; return DR_ERR_DOMAIN; }
    if (defer_kriging) {
      hv->kriging_pending = true;
    } else {
      kriging_solve_host(hv->kplan, &hv->w_rowptr, &hv->w_col, &hv->w_val);
      hv->kplan = KrigingPlan();
      build_transpose(hv);
      hv->kriging_solve_seconds =
          std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() - hv->kriging_plan_seconds;
    }
    hv->kriging_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  } else {
    hv->wt_rowptr.assign(n_h + 1, 0);
  }
  return DR_OK;
}

}  // namespace drb
