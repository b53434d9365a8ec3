// Covariance-parameter estimation (see estimate.h).
#include "estimate.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <map>

namespace drb {

std::vector<int> mce_offsets() {
  // perturbations_3d_unit_directions (perturbation_matrix.h:19-38)
  static const int U[14][3] = {{0, 0, 0},  {1, 0, 0}, {0, 1, 0},  {0, 0, 1}, {1, 1, 0},  {1, 0, 1},   {-1, 1, 0},
                               {1, 0, -1}, {0, 1, 1}, {0, 1, -1}, {1, 1, 1}, {1, 1, -1}, {-1, 1, 1}, {-1, 1, -1}};
  const int n = 18, raster = 25;
  std::vector<int> out;
  std::vector<unsigned char> seen(51 * 51 * 51, 0);
  auto add = [&](int a, int b, int c) {
    const int key = ((c + 25) * 51 + (b + 25)) * 51 + (a + 25);
    if (seen[key]) return;
    seen[key] = 1;
    out.push_back(a);
    out.push_back(b);
    out.push_back(c);
  };
  // perturbation_permutations_3d(18) rows (a fastest), each times every unit direction
  for (int c = 1; c <= n; c++)
    for (int b = 1; b <= n; b++)
      for (int a = 1; a <= n; a++)
        for (int j = 0; j < 14; j++) add(U[j][0] * a, U[j][1] * b, U[j][2] * c);
  for (int i = 0; i < raster - n; i++)
    for (int j = 0; j < 3; j++) {
      int p[3] = {0, 0, 0};
      p[j] = n + i + 1;
      add(p[0], p[1], p[2]);
    }
  return out;
}

std::vector<float> mce_distances(const std::vector<int>& P, const float* Q) {
  const size_t n = P.size() / 3;
  std::vector<float> d(n);
  for (size_t o = 0; o < n; o++) {
    float s2 = 0.0f;
    for (int r = 0; r < 4; r++) {
      float t = 0.0f;
      for (int c = 0; c < 3; c++) t += (float)P[3 * o + c] * Q[4 * r + c];
      s2 += t * t;
    }
    d[o] = std::sqrt(s2);
  }
  return d;
}

// ------------------------------------------------------------------ COBYLA
namespace {

using Vec = std::vector<double>;
using Mat = std::vector<Vec>;

double dot(const Vec& a, const Vec& b) {
  double s = 0;
  for (size_t i = 0; i < a.size(); i++) s += a[i] * b[i];
  return s;
}
double norm(const Vec& a) { return std::sqrt(dot(a, a)); }

// Inverse of a small square matrix by Gauss-Jordan with partial pivoting; false if singular.
bool invert(Mat A, Mat* inv) {
  const int n = (int)A.size();
  Mat I(n, Vec(n, 0.0));
  for (int i = 0; i < n; i++) I[i][i] = 1.0;
  for (int c = 0; c < n; c++) {
    int p = c;
    for (int r = c + 1; r < n; r++)
      if (std::fabs(A[r][c]) > std::fabs(A[p][c])) p = r;
    if (std::fabs(A[p][c]) < 1e-300) return false;
    std::swap(A[p], A[c]);
    std::swap(I[p], I[c]);
    const double piv = A[c][c];
    for (int j = 0; j < n; j++) { A[c][j] /= piv; I[c][j] /= piv; }
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      const double f = A[r][c];
      if (f == 0.0) continue;
      for (int j = 0; j < n; j++) { A[r][j] -= f * A[c][j]; I[r][j] -= f * I[c][j]; }
    }
  }
  *inv = I;
  return true;
}

// Linear constraints g_k . d >= b_k of the trust-region subproblem.
struct LinCons {
  Mat g;
  Vec b;
};

// Minimum-norm solution of G_S d = b_S for the rows S; false if G_S is rank deficient.
bool min_norm_on(const LinCons& L, const std::vector<int>& S, int n, Vec* d, Mat* GGinv) {
  const int s = (int)S.size();
  *d = Vec(n, 0.0);
  if (s == 0) {
    GGinv->clear();
    return true;
  }
  Mat M(s, Vec(s));
  for (int i = 0; i < s; i++)
    for (int j = 0; j < s; j++) M[i][j] = dot(L.g[S[i]], L.g[S[j]]);
  Mat Mi;
  if (!invert(M, &Mi)) return false;
  // rank check: M must be well conditioned relative to its scale
  double scale = 0;
  for (int i = 0; i < s; i++) scale = std::max(scale, M[i][i]);
  Vec lam(s, 0.0);
  for (int i = 0; i < s; i++)
    for (int j = 0; j < s; j++) lam[i] += Mi[i][j] * L.b[S[j]];
  for (int i = 0; i < s; i++)
    for (int k = 0; k < n; k++) (*d)[k] += lam[i] * L.g[S[i]][k];
  // verify G_S d = b_S (rejects nearly dependent rows)
  for (int i = 0; i < s; i++) {
    const double r = dot(L.g[S[i]], *d) - L.b[S[i]];
    if (std::fabs(r) > 1e-9 * (1.0 + std::fabs(L.b[S[i]])) || scale <= 0) return false;
  }
  *GGinv = Mi;
  return true;
}

bool feasible(const LinCons& L, const Vec& d) {
  for (size_t k = 0; k < L.g.size(); k++)
    if (dot(L.g[k], d) < L.b[k] - 1e-10 * (1.0 + std::fabs(L.b[k]))) return false;
  return true;
}

// Every subset of the constraints with at most n rows.
template <class F>
void for_subsets(int m, int n, F&& f) {
  std::vector<int> S;
  for (unsigned mask = 0; mask < (1u << m); mask++) {
    if (__builtin_popcount(mask) > n) continue;
    S.clear();
    for (int k = 0; k < m; k++)
      if (mask & (1u << k)) S.push_back(k);
    f(S);
  }
}

// Minimum-norm point of {d : g_k . d >= b_k}; false if the set is empty.
bool min_norm_point(const LinCons& L, int n, Vec* best) {
  double bn = std::numeric_limits<double>::infinity();
  bool found = false;
  for_subsets((int)L.g.size(), n, [&](const std::vector<int>& S) {
    Vec d;
    Mat Mi;
    if (!min_norm_on(L, S, n, &d, &Mi)) return;
    if (!feasible(L, d)) return;
    const double nd = norm(d);
    if (nd < bn) {
      bn = nd;
      *best = d;
      found = true;
    }
  });
  return found;
}

// The COBYLA trust-region subproblem: first the least achievable maximum
// violation t* of the linearised constraints within |d| <= rho, then the
// linearised objective minimised with every violation at most t*.  Both are
// convex in n (here 3) variables and solved exactly over active sets.
Vec trust_region_step(const Vec& gf, const Mat& gc, const Vec& c0, double rho, int n) {
  const int m = (int)gc.size();
  LinCons L;
  L.g = gc;
  L.b.resize(m);
  double v0 = 0;
  for (int k = 0; k < m; k++) v0 = std::max(v0, -c0[k]);
  auto set_t = [&](double t) {
    for (int k = 0; k < m; k++) L.b[k] = -c0[k] - t;
  };
  double t_star = 0.0;
  Vec d1(n, 0.0);
  if (v0 > 0) {
    double lo = 0.0, hi = v0;
    set_t(0.0);
    Vec d;
    if (min_norm_point(L, n, &d) && norm(d) <= rho) {
      hi = 0.0;
    } else {
      for (int it = 0; it < 60; it++) {
        const double mid = 0.5 * (lo + hi);
        set_t(mid);
        if (min_norm_point(L, n, &d) && norm(d) <= rho) hi = mid;
        else lo = mid;
      }
    }
    t_star = hi;
    set_t(t_star);
    if (!min_norm_point(L, n, &d1)) d1.assign(n, 0.0);
  } else {
    set_t(0.0);
  }
  // stage 2
  Vec best = d1;
  double bobj = dot(gf, d1), bnorm = norm(d1);
  for_subsets(m, n, [&](const std::vector<int>& S) {
    Vec dp;
    Mat Mi;
    if (!min_norm_on(L, S, n, &dp, &Mi)) return;
    const double np = norm(dp);
    if (np > rho * (1 + 1e-12)) return;
    // projection of gf on the null space of G_S
    Vec pg = gf;
    if (!S.empty()) {
      const int s = (int)S.size();
      Vec Gg(s);
      for (int i = 0; i < s; i++) Gg[i] = dot(L.g[S[i]], gf);
      for (int i = 0; i < s; i++) {
        double li = 0;
        for (int j = 0; j < s; j++) li += Mi[i][j] * Gg[j];
        for (int k = 0; k < n; k++) pg[k] -= li * L.g[S[i]][k];
      }
    }
    const double npg = norm(pg);
    Vec d = dp;
    if (npg > 1e-14 * (1.0 + norm(gf))) {
      const double a = std::sqrt(std::max(0.0, rho * rho - np * np));
      for (int k = 0; k < n; k++) d[k] -= a * pg[k] / npg;
    }
    if (!feasible(L, d)) return;
    const double obj = dot(gf, d), nd = norm(d);
    if (obj < bobj - 1e-15 * (1 + std::fabs(bobj)) || (obj <= bobj && nd < bnorm)) {
      best = d;
      bobj = obj;
      bnorm = nd;
    }
  });
  return best;
}

}  // namespace

int cobyla_minimize(int n, int m, std::vector<double>& x, const std::vector<double>& step, double rho_end,
                    int max_eval, const std::function<double(const double*, double*)>& fc) {
  const double alpha = 0.25, beta = 2.1, gamma = 0.5;
  double rho = 1.0;
  rho_end = std::min(rho_end, rho);
  int nfev = 0;
  Mat V(n + 1, Vec(n));            // vertices in scaled coordinates
  Vec fv(n + 1);
  Mat cv(n + 1, Vec(m));
  Vec xs(n);
  auto eval = [&](const Vec& u, double* f, double* c) {
    for (int i = 0; i < n; i++) xs[i] = u[i] * step[i];
    *f = fc(xs.data(), c);
    nfev++;
  };
  auto viol = [&](const Vec& c) {
    double v = 0;
    for (int k = 0; k < m; k++) v = std::max(v, -c[k]);
    return v;
  };
  for (int i = 0; i < n; i++) V[0][i] = x[i] / step[i];
  eval(V[0], &fv[0], cv[0].data());
  for (int j = 1; j <= n; j++) {
    V[j] = V[0];
    V[j][j - 1] += rho;
    eval(V[j], &fv[j], cv[j].data());
  }
  double mu = 0.0;
  bool need_geometry = false;
  while (nfev < max_eval) {
    // best vertex (least merit, then least violation) into slot 0
    int b = 0;
    for (int j = 1; j <= n; j++) {
      const double pj = fv[j] + mu * viol(cv[j]), pb = fv[b] + mu * viol(cv[b]);
      if (pj < pb || (pj == pb && viol(cv[j]) < viol(cv[b]))) b = j;
    }
    if (b != 0) {
      std::swap(V[0], V[b]);
      std::swap(fv[0], fv[b]);
      std::swap(cv[0], cv[b]);
    }
    // simplex edges and linear models
    Mat D(n, Vec(n)), Di;
    for (int j = 0; j < n; j++)
      for (int i = 0; i < n; i++) D[j][i] = V[j + 1][i] - V[0][i];
    if (!invert(D, &Di)) {  // degenerate simplex: rebuild it around the best vertex
      for (int j = 1; j <= n; j++) {
        V[j] = V[0];
        V[j][j - 1] += rho;
        eval(V[j], &fv[j], cv[j].data());
      }
      continue;
    }
    auto model_grad = [&](const Vec& vals) {  // g = D^-1 (vals_j - vals_0)
      Vec g(n, 0.0);
      for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) g[i] += Di[i][j] * (vals[j + 1] - vals[0]);
      return g;
    };
    const Vec gf = model_grad(fv);
    Mat gc(m);
    for (int k = 0; k < m; k++) {
      Vec ck(n + 1);
      for (int j = 0; j <= n; j++) ck[j] = cv[j][k];
      gc[k] = model_grad(ck);
    }
    // geometry: edge lengths and distances of each vertex from the opposite face
    int jlong = 0, jflat = 0;
    double lmax = 0, smin = std::numeric_limits<double>::infinity();
    for (int j = 0; j < n; j++) {
      const double lj = norm(D[j]);
      double w2 = 0;
      for (int i = 0; i < n; i++) w2 += Di[i][j] * Di[i][j];
      const double sj = 1.0 / std::sqrt(w2);
      if (lj > lmax) { lmax = lj; jlong = j; }
      if (sj < smin) { smin = sj; jflat = j; }
    }
    const bool acceptable = lmax <= beta * rho && smin >= alpha * rho;
    const double v0 = viol(cv[0]);
    auto lin_merit = [&](const Vec& d) {
      double v = 0;
      for (int k = 0; k < m; k++) v = std::max(v, -(cv[0][k] + dot(gc[k], d)));
      return dot(gf, d) + mu * v;
    };
    auto geometry_step = [&]() {
      const int j = lmax > beta * rho ? jlong : jflat;
      Vec w(n);
      for (int i = 0; i < n; i++) w[i] = Di[i][j];
      const double nw = norm(w);
      Vec dp(n), dm(n);
      for (int i = 0; i < n; i++) {
        dp[i] = gamma * rho * w[i] / nw;
        dm[i] = -dp[i];
      }
      const Vec& d = lin_merit(dp) <= lin_merit(dm) ? dp : dm;
      for (int i = 0; i < n; i++) V[j + 1][i] = V[0][i] + d[i];
      eval(V[j + 1], &fv[j + 1], cv[j + 1].data());
      need_geometry = false;
    };
    auto reduce_rho = [&]() {
      if (rho <= rho_end) return false;
      rho = 0.5 * rho;
      if (rho <= 1.5 * rho_end) rho = rho_end;
      need_geometry = false;
      return true;
    };
    if (need_geometry && !acceptable) {
      geometry_step();
      continue;
    }
    const Vec d = trust_region_step(gf, gc, cv[0], rho, n);
    if (norm(d) < 0.5 * rho) {
      if (!acceptable) {
        geometry_step();
        continue;
      }
      if (!reduce_rho()) break;
      continue;
    }
    // penalty parameter: the step must reduce the linearised merit function
    double vlin = 0;
    for (int k = 0; k < m; k++) vlin = std::max(vlin, -(cv[0][k] + dot(gc[k], d)));
    const double dfl = dot(gf, d);
    if (v0 - vlin > 0 && dfl > 0) {
      const double barmu = dfl / (v0 - vlin);
      if (mu < 1.5 * barmu) mu = 2.0 * barmu;
    }
    const double pred = -(dfl + mu * (vlin - v0));
    Vec un(n);
    for (int i = 0; i < n; i++) un[i] = V[0][i] + d[i];
    double fn;
    Vec cn(m);
    eval(un, &fn, cn.data());
    const double ared = (fv[0] + mu * v0) - (fn + mu * viol(cn));
    const double ratio = pred > 0 ? ared / pred : -1.0;
    // vertex to replace: barycentric weight of the new point times its distance
    Vec t(n, 0.0);
    double tsum = 0;
    for (int j = 0; j < n; j++) {
      for (int i = 0; i < n; i++) t[j] += Di[i][j] * d[i];
      tsum += t[j];
    }
    int jr = -1;
    double wbest = ared > 0 ? 0.0 : 1.0;
    for (int j = (ared > 0 ? -1 : 0); j < n; j++) {
      const Vec& vj = j < 0 ? V[0] : V[j + 1];
      const double tj = j < 0 ? 1.0 - tsum : t[j];
      double dist = 0;
      for (int i = 0; i < n; i++) dist += (vj[i] - un[i]) * (vj[i] - un[i]);
      const double w = std::fabs(tj) * std::max(1.0, dist / (rho * rho));
      if (w > wbest) {
        wbest = w;
        jr = j;
      }
    }
    if (jr != -1 || ared > 0) {
      const int slot = jr < 0 ? 0 : jr + 1;
      V[slot] = un;
      fv[slot] = fn;
      cv[slot] = cn;
    }
    if (ratio < 0.1) {
      need_geometry = true;
      if (acceptable && !reduce_rho()) break;
    }
  }
  // best point: feasible first, then least objective
  int b = 0;
  for (int j = 1; j <= n; j++) {
    const double vj = viol(cv[j]), vb = viol(cv[b]);
    if (vj < vb - 1e-12 || (std::fabs(vj - vb) <= 1e-12 && fv[j] < fv[b])) b = j;
  }
  for (int i = 0; i < n; i++) x[i] = V[b][i] * step[i];
  return nfev;
}

int fit_rbf_parameters(const float* distance, const float* covariance, const int* npairs, int n, double* theta,
                       std::string* err) {
  const double eps0 = 1e-5, xtol = 1e-5;
  if (n < 2) {
    *err = "too few offsets";
    return 1;
  }
  const double tau_max = (double)covariance[0];
  double lb[3] = {eps0, eps0, eps0};
  double ub[3] = {tau_max, HUGE_VAL, 2.0 - eps0};
  if (!(ub[0] > lb[0])) {
    *err = "compute_rbf_parameters: sample variance not above the lower bound";
    return 1;
  }
  if (theta[1] > theta[2]) {
    *err = "compute_rbf_parameters: requested constraint with bandwidth > exponent";
    return 1;
  }
  // data: offsets 1.. with pairs; weights 1 / sqrt(multiplicity of the distance value)
  std::vector<double> dx, dy;
  for (int i = 1; i < n; i++) {
    if (npairs[i] != 0 && distance[i] <= 1e6) {
      dx.push_back(std::fabs((double)distance[i]));
      dy.push_back((double)covariance[i]);
    }
  }
  if (dx.empty()) {
    *err = "no offset has voxel pairs";
    return 1;
  }
  // weights 1 / sqrt(multiplicity): the objective is evaluated once per distinct distance u with the
  // group sums S1 = sum y, S2 = sum y^2:  sum_i w_i^2 (y_i - a rho_u)^2 = (S2 - 2 a rho_u S1 + m a^2 rho_u^2) / m
  std::map<double, std::array<double, 3>> groups;  // distance -> (m, S1, S2)
  for (size_t i = 0; i < dx.size(); i++) {
    auto& g = groups[dx[i]];
    g[0] += 1.0;
    g[1] += dy[i];
    g[2] += dy[i] * dy[i];
  }
  std::vector<double> gd, gm, g1, g2;
  for (const auto& kv : groups) {
    gd.push_back(kv.first);
    gm.push_back(kv.second[0]);
    g1.push_back(kv.second[1]);
    g2.push_back(kv.second[2]);
  }
  const double N = (double)dx.size();
  auto fc = [&](const double* x, double* c) {
    // _rbf_least_squares (estimate_kernel_parameters.h:119-148)
    double obj = 0;
    for (size_t u = 0; u < gd.size(); u++) {
      const double rho = std::exp(-x[1] * std::pow(gd[u], x[2]));
      const double a = x[0] * rho;
      obj += (g2[u] - 2.0 * a * g1[u] + gm[u] * a * a) / gm[u];
    }
    obj /= N;
    // bounds and _rbf_constraint (x[1] - x[2] <= 0) as c >= 0
    c[0] = x[0] - lb[0];
    c[1] = x[1] - lb[1];
    c[2] = x[2] - lb[2];
    c[3] = ub[0] - x[0];
    c[4] = ub[2] - x[2];
    c[5] = x[2] - x[1];
    return obj;
  };
  std::vector<double> x(theta, theta + 3);
  // a start outside the bounds is projected into them
  for (int i = 0; i < 3; i++) x[i] = std::min(std::max(x[i], lb[i]), ub[i]);
  std::vector<double> step(3);
  for (int i = 0; i < 3; i++) {
    double s = std::max(0.25 * std::fabs(x[i]), 1e-4);
    if (std::isfinite(ub[i])) s = std::min(s, 0.25 * (ub[i] - lb[i]));
    step[i] = s;
  }
  // final radius: a relative change of xtol in every parameter
  double rho_end = 1.0;
  for (int i = 0; i < 3; i++) rho_end = std::min(rho_end, xtol * std::max(std::fabs(x[i]), 1e-3) / step[i]);
  cobyla_minimize(3, 6, x, step, rho_end, 20000, fc);
  for (int i = 0; i < 3; i++) {
    if (!std::isfinite(x[i])) {
      *err = "COBYLA did not return a finite point";
      return 1;
    }
    theta[i] = x[i];
  }
  return 0;
}

}  // namespace drb
