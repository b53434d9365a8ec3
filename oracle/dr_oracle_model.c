/*
 * dr_oracle_model.c -- precision-dependent part of the CPU oracle: a plain
 * restatement of MultiResParameters<T> (include/dualres/MultiResParameters.h)
 * and of the fit_model loop (include/dualres/gaussian_process_model.h).
 *
 * TEST INFRASTRUCTURE ONLY (see dr_oracle.h).  Parity unpinned: the reference
 * has no golden vectors and cannot be compiled in this image.
 *
 * Compiled twice: -DORC_DOUBLE (suffix _d, the `dualgpm` build) and without it
 * (suffix _f, the `dualgpmf` build).  It keeps the reference's operation order:
 * four unnormalised 3D FFTs per leapfrog step, complex lambda, Kahan sums in
 * double, and spectral zeroing of the set S = {Re lambda <= 0}.
 */
#include "dr_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORC_DOUBLE
typedef double real;
typedef double _Complex cplx;
#define SFX(n) n##_d
#define MODEL orc_model_d
#define CONJ conj
#define CRE creal
#define CIM cimag
#define CSQRT csqrt
#define RSQRT sqrt
#define REXP exp
#define RPOW pow
#define RABS fabs
#else
typedef float real;
typedef float _Complex cplx;
#define SFX(n) n##_f
#define MODEL orc_model_f
#define CONJ conjf
#define CRE crealf
#define CIM cimagf
#define CSQRT csqrtf
#define RSQRT sqrtf
#define REXP expf
#define RPOW powf
#define RABS fabsf
#endif

struct MODEL {
  int E[3];
  long N;
  cplx* lambda;
  cplx* lambda_mass;
  cplx* momentum;
  cplx* mu;
  cplx* mu_star;
  cplx* temp;
  cplx* tw[3];
  int* S;
  int nS;
  int n_h;
  int* D;
  real* Yh;
  int n_s;
  real* Ys;
  int* rowptr;
  int* col;
  real* val;
  real* real_mu;
  real* sub_grad;
  real* wmu;
  int n_o;
  int* O;
  int n_datasets;
  real sigma_sq_inv[2];
  double theta[3];
};

/* ------------------------------ FFT -------------------------------------- */
/* Unnormalised DFT, forward exp(-2 pi i jk/n), inverse exp(+2 pi i jk/n)
 * (FFTW convention, sized_fft.h:138-214), n a power of two.  Stockham
 * autosort (C. Van Loan, "Computational Frameworks for the Fast Fourier
 * Transform", 1992, sec. 1.7) in radix-4 stages, with one radix-2 stage first
 * when log2 n is odd: each stage reads one buffer and writes the other in
 * natural order, so no bit reversal is needed and the inner loops run over
 * contiguous elements.  tw[k] = exp(-2 pi i k / n), k < n/2. */
static inline cplx tw_at(const cplx* tw, int n, long k, int inverse) {
  /* exp(-+2 pi i k / n) for 0 <= k < n from the half table (W^(k + n/2) = -W^k) */
  const cplx w = k < n / 2 ? tw[k] : -tw[k - n / 2];
  return inverse ? CONJ(w) : w;
}

static cplx* make_twiddles(int n) {
  cplx* t = (cplx*)malloc(sizeof(cplx) * (n > 1 ? n / 2 : 1));
  for (int k = 0; k < n / 2; k++) {
    const double ang = -2.0 * M_PI * (double)k / (double)n;
    t[k] = (real)cos(ang) + (real)sin(ang) * I;
  }
  return t;
}

/* FFT_W lines at a time, stored split and line-fastest: element k of line v is
 * (re[k FFT_W + v], im[k FFT_W + v]).  Stage with m points per sub-transform
 * and l = n / (r m) groups (radix r = 2 or 4, W_r = exp(-+2 pi i / r)):
 *   y[k + r j m + q m] = W_(r l)^(j q) sum_p x[k + j m + p l m] W_r^(p q),
 * every butterfly applied to the FFT_W lines in one contiguous (vectorisable)
 * loop.  The result is in re/im; wre/wim are the other buffer. */
#define FFT_W 16
static void fft_lines_soa(real* re, real* im, real* wre, real* wim, int n, const cplx* tw, int inverse) {
  real *xr = re, *xi = im, *yr = wre, *yi = wim, *t;
  const real sgn = inverse ? (real)1 : (real)-1; /* W_4 = sgn i */
  int m = 1, lg = 0;
  while ((1 << lg) < n) lg++;
  if (lg & 1) {
    const int l = n / 2;
    for (int j = 0; j < l; j++) {
      const cplx w = tw_at(tw, n, j, inverse);
      const real wr = CRE(w), wi = CIM(w);
      const real *restrict ar = xr + (long)j * FFT_W, *restrict ai = xi + (long)j * FFT_W;
      const real *restrict br = ar + (long)l * FFT_W, *restrict bi = ai + (long)l * FFT_W;
      real *restrict o0r = yr + 2L * j * FFT_W, *restrict o0i = yi + 2L * j * FFT_W;
      real *restrict o1r = o0r + FFT_W, *restrict o1i = o0i + FFT_W;
      for (int v = 0; v < FFT_W; v++) {
        const real dr = ar[v] - br[v], di = ai[v] - bi[v];
        o0r[v] = ar[v] + br[v];
        o0i[v] = ai[v] + bi[v];
        o1r[v] = wr * dr - wi * di;
        o1i[v] = wr * di + wi * dr;
      }
    }
    t = xr; xr = yr; yr = t;
    t = xi; xi = yi; yi = t;
    m = 2;
  }
  for (; m < n; m *= 4) {
    const int l = n / (4 * m);
    const long lm = (long)l * m * FFT_W;
    for (int j = 0; j < l; j++) {
      const cplx w1 = tw_at(tw, n, (long)j * m, inverse), w2 = tw_at(tw, n, 2L * j * m, inverse),
                 w3 = tw_at(tw, n, 3L * j * m, inverse);
      const real w1r = CRE(w1), w1i = CIM(w1), w2r = CRE(w2), w2i = CIM(w2), w3r = CRE(w3), w3i = CIM(w3);
      for (int k = 0; k < m; k++) {
        const long in = ((long)j * m + k) * FFT_W, out = (4L * j * m + k) * FFT_W, om = (long)m * FFT_W;
        const real *restrict a0r = xr + in, *restrict a0i = xi + in;
        real *restrict y0r = yr + out, *restrict y0i = yi + out;
        for (int v = 0; v < FFT_W; v++) {
          const real a0x = a0r[v], a0y = a0i[v], a1x = a0r[v + lm], a1y = a0i[v + lm];
          const real a2x = a0r[v + 2 * lm], a2y = a0i[v + 2 * lm], a3x = a0r[v + 3 * lm], a3y = a0i[v + 3 * lm];
          const real b0x = a0x + a2x, b0y = a0y + a2y, b1x = a0x - a2x, b1y = a0y - a2y;
          const real b2x = a1x + a3x, b2y = a1y + a3y, dx = a1x - a3x, dy = a1y - a3y;
          const real b3x = -sgn * dy, b3y = sgn * dx;
          const real c1x = b1x + b3x, c1y = b1y + b3y, c2x = b0x - b2x, c2y = b0y - b2y;
          const real c3x = b1x - b3x, c3y = b1y - b3y;
          y0r[v] = b0x + b2x;
          y0i[v] = b0y + b2y;
          y0r[v + om] = w1r * c1x - w1i * c1y;
          y0i[v + om] = w1r * c1y + w1i * c1x;
          y0r[v + 2 * om] = w2r * c2x - w2i * c2y;
          y0i[v + 2 * om] = w2r * c2y + w2i * c2x;
          y0r[v + 3 * om] = w3r * c3x - w3i * c3y;
          y0i[v + 3 * om] = w3r * c3y + w3i * c3x;
        }
      }
    }
    t = xr; xr = yr; yr = t;
    t = xi; xi = yi; yi = t;
  }
  if (xr != re) {
    memcpy(re, xr, sizeof(real) * (size_t)n * FFT_W);
    memcpy(im, xi, sizeof(real) * (size_t)n * FFT_W);
  }
}

/* Transforms the lines a[o ostride + s sstride + k kstride], k < n, for
 * s < inner and o < outer, FFT_W values of s at a time. */
static void fft_pass(cplx* a, int n, long kstride, long sstride, long inner, long outer, long ostride,
                     const cplx* tw, int inverse) {
  const long nblk = (inner + FFT_W - 1) / FFT_W;
#pragma omp parallel
  {
    real* buf = (real*)malloc(sizeof(real) * 4 * (size_t)n * FFT_W);
    real *re = buf, *im = buf + (size_t)n * FFT_W, *wre = im + (size_t)n * FFT_W, *wim = wre + (size_t)n * FFT_W;
#pragma omp for schedule(static) collapse(2)
    for (long o = 0; o < outer; o++)
      for (long b = 0; b < nblk; b++) {
        const long s0 = b * FFT_W;
        const int w = (int)(inner - s0 < FFT_W ? inner - s0 : FFT_W);
        cplx* base = a + o * ostride + s0 * sstride;
        for (int k = 0; k < n; k++) {
          int v = 0;
          for (; v < w; v++) {
            const cplx c = base[v * sstride + (long)k * kstride];
            re[(long)k * FFT_W + v] = CRE(c);
            im[(long)k * FFT_W + v] = CIM(c);
          }
          for (; v < FFT_W; v++) re[(long)k * FFT_W + v] = im[(long)k * FFT_W + v] = 0;
        }
        fft_lines_soa(re, im, wre, wim, n, tw, inverse);
        for (int k = 0; k < n; k++)
          for (int v = 0; v < w; v++)
            base[v * sstride + (long)k * kstride] = re[(long)k * FFT_W + v] + im[(long)k * FFT_W + v] * I;
      }
    free(buf);
  }
}

static void fft3d_tw(cplx* a, const int* E, cplx* const* tw, int inverse) {
  const long E0 = E[0], E1 = E[1], E2 = E[2];
  /* x lines: start (z E1 + y) E0; y lines: start z E0 E1 + x, stride E0; z lines: start y E0 + x, stride E0 E1 */
  if (E0 > 1) fft_pass(a, (int)E0, 1, E0, E1 * E2, 1, 0, tw[0], inverse);
  if (E1 > 1) fft_pass(a, (int)E1, E0, 1, E0, E2, E0 * E1, tw[1], inverse);
  if (E2 > 1) fft_pass(a, (int)E2, E0 * E1, 1, E0 * E1, 1, 0, tw[2], inverse);
}

void SFX(orc_fft3d)(real* data, const int* E, int inverse) {
  cplx* tw[3];
  for (int d = 0; d < 3; d++) tw[d] = make_twiddles(E[d]);
  fft3d_tw((cplx*)data, E, tw, inverse);
  for (int d = 0; d < 3; d++) free(tw[d]);
}

void SFX(orc_set_threads)(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

static void fwd(const struct MODEL* m, cplx* a) { fft3d_tw(a, m->E, (cplx* const*)m->tw, 0); }
static void inv(const struct MODEL* m, cplx* a) { fft3d_tw(a, m->E, (cplx* const*)m->tw, 1); }

/* ---------------------------- model setup -------------------------------- */
static real cov_fn(int covfun, real d, real b, real e, real v) {
  /* kernels.inl:8-15 rbf(distance, bandwidth, exponent, variance);
   * kernels.inl:59-74 rational_quadratic(val, psi, nu, variance). */
  if (covfun == 0) return v * REXP(-b * RPOW(RABS(d), e));
  return v * RPOW((real)1 + b / e * d * d, -e);
}

/* MultiResParameters.h:173-300 (without _initialize_mu/_initialize_sigma) */
MODEL* SFX(orc_model_create)(int n_h, const int* D_ijk, const float* Yh,
                             int n_s, const float* Ys, const int* rowptr, const int* col, const real* val,
                             const float* Q, const double* theta, int covfun, int n_o, const int* O_ijk,
                             int* status) {
  *status = 0;
  if (n_h <= 0) { *status = -1; return NULL; }
  int g[3] = {0, 0, 0};
  for (int i = 0; i < n_h; i++)
    for (int d = 0; d < 3; d++)
      if (D_ijk[3 * i + d] > g[d]) g[d] = D_ijk[3 * i + d];
  for (int d = 0; d < 3; d++) g[d] += 1;
  struct MODEL* m = (struct MODEL*)calloc(1, sizeof(struct MODEL));
  if (orc_embedding_dims(g, m->E) != 0) { free(m); *status = -2; return NULL; }
  m->N = (long)m->E[0] * m->E[1] * m->E[2];
  const long N = m->N;
  m->lambda = (cplx*)calloc(N, sizeof(cplx));
  m->lambda_mass = (cplx*)calloc(N, sizeof(cplx));
  m->momentum = (cplx*)calloc(N, sizeof(cplx));
  m->mu = (cplx*)calloc(N, sizeof(cplx));
  m->mu_star = (cplx*)calloc(N, sizeof(cplx));
  m->temp = (cplx*)calloc(N, sizeof(cplx));
  for (int d = 0; d < 3; d++) m->tw[d] = make_twiddles(m->E[d]);

  /* circulant_base.inl:30-89: wrapped offsets 0..E/2, E/2-1..1; distance is the
   * float norm of Q (o, 0).  Then cov() in the model precision. */
  const real th_v = (real)theta[0], th_b = (real)theta[1], th_e = (real)theta[2];
  for (int n = 0; n < m->E[2]; n++)
    for (int mm = 0; mm < m->E[1]; mm++)
      for (int l = 0; l < m->E[0]; l++) {
        const float o[3] = {(float)(l <= m->E[0] / 2 ? l : m->E[0] - l),
                            (float)(mm <= m->E[1] / 2 ? mm : m->E[1] - mm),
                            (float)(n <= m->E[2] / 2 ? n : m->E[2] - n)};
        float s = 0.0f;
        for (int r = 0; r < 3; r++) {
          const float q = Q[4 * r + 0] * o[0] + Q[4 * r + 1] * o[1] + Q[4 * r + 2] * o[2];
          s += q * q;
        }
        const real dist = (real)sqrtf(s);
        m->lambda[(long)n * m->E[0] * m->E[1] + (long)mm * m->E[0] + l] =
            cov_fn(covfun, dist, th_b, th_e, th_v);
      }
  fwd(m, m->lambda);

  /* MultiResParameters.h:258-284 */
  m->S = (int*)malloc(sizeof(int) * N);
  m->nS = 0;
  for (long i = 0; i < N; i++)
    if (CRE(m->lambda[i]) <= 0) m->S[m->nS++] = (int)i;
  if ((long)m->nS >= N / 2) { *status = -3; SFX(orc_model_free)(m); return NULL; }

  /* MultiResParameters.h:287-289 */
  m->n_h = n_h;
  m->D = (int*)malloc(sizeof(int) * n_h);
  for (int i = 0; i < n_h; i++)
    m->D[i] = D_ijk[3 * i + 2] * m->E[0] * m->E[1] + D_ijk[3 * i + 1] * m->E[0] + D_ijk[3 * i];
  m->Yh = (real*)malloc(sizeof(real) * n_h);
  for (int i = 0; i < n_h; i++) m->Yh[i] = (real)Yh[i];
  m->n_s = n_s;
  m->n_datasets = n_s > 0 ? 2 : 1;
  if (n_s > 0) {
    m->Ys = (real*)malloc(sizeof(real) * n_s);
    for (int i = 0; i < n_s; i++) m->Ys[i] = (real)Ys[i];
    m->rowptr = (int*)malloc(sizeof(int) * (n_s + 1));
    memcpy(m->rowptr, rowptr, sizeof(int) * (n_s + 1));
    const int nnz = rowptr[n_s];
    m->col = (int*)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    m->val = (real*)malloc(sizeof(real) * (nnz > 0 ? nnz : 1));
    memcpy(m->col, col, sizeof(int) * nnz);
    memcpy(m->val, val, sizeof(real) * nnz);
    m->wmu = (real*)malloc(sizeof(real) * n_s);
  }
  m->real_mu = (real*)calloc(n_h, sizeof(real));
  m->sub_grad = (real*)calloc(n_h, sizeof(real));

  /* MultiResParameters.h:647-667 (output indices; indices >= E are rejected
   * here because the reference would read past the field). */
  m->n_o = n_o;
  m->O = (int*)malloc(sizeof(int) * (n_o > 0 ? n_o : 1));
  for (int i = 0; i < n_o; i++) {
    for (int d = 0; d < 3; d++)
      if (O_ijk[3 * i + d] < 0 || O_ijk[3 * i + d] >= m->E[d]) { *status = -4; SFX(orc_model_free)(m); return NULL; }
    m->O[i] = O_ijk[3 * i + 2] * m->E[0] * m->E[1] + O_ijk[3 * i + 1] * m->E[0] + O_ijk[3 * i];
  }
  m->sigma_sq_inv[0] = 1;
  m->sigma_sq_inv[1] = 1;
  for (int d = 0; d < 3; d++) m->theta[d] = theta[d];
  return m;
}

void SFX(orc_model_free)(MODEL* m) {
  if (!m) return;
  free(m->lambda); free(m->lambda_mass); free(m->momentum); free(m->mu); free(m->mu_star);
  free(m->temp); free(m->S); free(m->D); free(m->Yh); free(m->Ys); free(m->rowptr);
  free(m->col); free(m->val); free(m->real_mu); free(m->sub_grad); free(m->wmu); free(m->O);
  for (int d = 0; d < 3; d++) free(m->tw[d]);
  free(m);
}

void SFX(orc_model_info)(const MODEL* m, int* E, int64_t* N, int* n_S) {
  for (int d = 0; d < 3; d++) E[d] = m->E[d];
  *N = m->N;
  *n_S = m->nS;
}

void SFX(orc_model_lambda)(const MODEL* m, double* out) {
  for (long i = 0; i < m->N; i++) { out[2 * i] = CRE(m->lambda[i]); out[2 * i + 1] = CIM(m->lambda[i]); }
}

void SFX(orc_model_set_sigma)(MODEL* m, real sh, real ss) { m->sigma_sq_inv[0] = sh; m->sigma_sq_inv[1] = ss; }
void SFX(orc_model_get_sigma)(const MODEL* m, real* s) { s[0] = m->sigma_sq_inv[0]; s[1] = m->sigma_sq_inv[1]; }
void SFX(orc_model_set_mu)(MODEL* m, const real* mu) { memcpy(m->mu, mu, sizeof(cplx) * m->N); }
void SFX(orc_model_get_mu)(const MODEL* m, real* mu) { memcpy(mu, m->mu, sizeof(cplx) * m->N); }

/* MultiResParameters.h:310-319 */
static void low_rank_adjust(const MODEL* m, cplx* A) {
  for (int i = 0; i < m->nS; i++) A[m->S[i]] = 0;
}

/* ------------------------------ energies --------------------------------- */
typedef struct { double re, im, cre, cim; } kahan_c;
static void kahan_add(kahan_c* k, double re, double im) {
  double a = re - k->cre, b = k->re + a;
  k->cre = (b - k->re) - a; k->re = b;
  a = im - k->cim; b = k->im + a;
  k->cim = (b - k->im) - a; k->im = b;
}

/* MultiResParameters.h:429-476 (Kahan branch, :436-448) */
static double log_prior_impl(MODEL* m, const cplx* mu) {
  memcpy(m->temp, mu, sizeof(cplx) * m->N);
  inv(m, m->temp);
  kahan_c k = {0, 0, 0, 0};
  for (long i = 0; i < m->N; i++) {
    if (CRE(m->lambda[i]) > 0) {
      const double _Complex t = (double)CRE(m->temp[i]) + (double)CIM(m->temp[i]) * I;
      const double _Complex l = (double)CRE(m->lambda[i]) + (double)CIM(m->lambda[i]) * I;
      const double _Complex a = conj(t) * t / l;
      kahan_add(&k, creal(a), cimag(a));
    }
  }
  return -0.5 * (k.re + k.im) / (double)m->N;
}

static void set_real_mu(MODEL* m, const cplx* mu) {
  for (int i = 0; i < m->n_h; i++) m->real_mu[i] = CRE(mu[m->D[i]]);
}

static void w_times(const MODEL* m, const real* x, real* y) {
  for (int r = 0; r < m->n_s; r++) {
    real s = 0;
    for (int k = m->rowptr[r]; k < m->rowptr[r + 1]; k++) s += m->val[k] * x[m->col[k]];
    y[r] = s;
  }
}

/* MultiResParameters.h:488-514 */
static double log_lik_impl(MODEL* m, const cplx* mu, double* norms) {
  set_real_mu(m, mu);
  double nh = 0.0;
  for (int i = 0; i < m->n_h; i++) { const double r = (double)(m->Yh[i] - m->real_mu[i]); nh += r * r; }
  double ll = (double)m->sigma_sq_inv[0] * nh, ns = 0.0;
  if (m->n_datasets == 2) {
    w_times(m, m->real_mu, m->wmu);
    for (int i = 0; i < m->n_s; i++) { const double r = (double)(m->Ys[i] - m->wmu[i]); ns += r * r; }
    ll += (double)m->sigma_sq_inv[1] * ns;
  }
  if (norms) { norms[0] = nh; norms[1] = ns; }
  return -0.5 * ll;
}

/* MultiResParameters.h:337-376; result left in m->temp */
static void gradient_impl(MODEL* m, const cplx* mu_star) {
  memcpy(m->temp, mu_star, sizeof(cplx) * m->N);
  inv(m, m->temp);
  const real negN = -(real)m->N;
  for (long i = 0; i < m->N; i++) m->temp[i] /= negN * m->lambda[i];
  low_rank_adjust(m, m->temp);
  fwd(m, m->temp);
  set_real_mu(m, mu_star);
  for (int i = 0; i < m->n_h; i++) m->sub_grad[i] = m->sigma_sq_inv[0] * (m->Yh[i] - m->real_mu[i]);
  if (m->n_datasets == 2) {
    w_times(m, m->real_mu, m->wmu);
    for (int r = 0; r < m->n_s; r++) m->wmu[r] = m->Ys[r] - m->wmu[r];
    /* ((Ys - W mu)^T W)^T accumulated column by column */
    real* acc = (real*)calloc(m->n_h, sizeof(real));
    for (int r = 0; r < m->n_s; r++)
      for (int k = m->rowptr[r]; k < m->rowptr[r + 1]; k++) acc[m->col[k]] += m->wmu[r] * m->val[k];
    for (int i = 0; i < m->n_h; i++) m->sub_grad[i] += m->sigma_sq_inv[1] * acc[i];
    free(acc);
  }
  /* the scatter runs in parallel, as MultiResParameters.h:370 does (D holds distinct indices) */
#pragma omp parallel for schedule(static)
  for (int i = 0; i < m->n_h; i++) m->temp[m->D[i]] += m->sub_grad[i];
}

/* MultiResParameters.h:735-738 */
static void mass_matrix(MODEL* m) {
  for (long i = 0; i < m->N; i++) m->lambda_mass[i] = (real)1 / m->lambda[i] + m->sigma_sq_inv[0];
  low_rank_adjust(m, m->lambda_mass);
}

/* MultiResParameters.h:551-603 (Kahan branch, :558-572) */
static double kinetic_impl(MODEL* m, const cplx* p) {
  memcpy(m->temp, p, sizeof(cplx) * m->N);
  inv(m, m->temp);
  kahan_c k = {0, 0, 0, 0};
  for (long i = 0; i < m->N; i++) {
    if (CRE(m->lambda_mass[i]) != 0 || CIM(m->lambda_mass[i]) != 0) {
      const double _Complex t = (double)CRE(m->temp[i]) + (double)CIM(m->temp[i]) * I;
      const double _Complex l = (double)CRE(m->lambda_mass[i]) + (double)CIM(m->lambda_mass[i]) * I;
      const double _Complex a = conj(t) * t / l;
      kahan_add(&k, creal(a), cimag(a));
    }
  }
  return -0.5 * (k.re + k.im) / (double)m->N;
}

double SFX(orc_log_prior)(MODEL* m, const real* mu) { return log_prior_impl(m, (const cplx*)mu); }
double SFX(orc_log_likelihood)(MODEL* m, const real* mu) { return log_lik_impl(m, (const cplx*)mu, NULL); }
void SFX(orc_gradient)(MODEL* m, const real* mu, real* grad) {
  gradient_impl(m, (const cplx*)mu);
  memcpy(grad, m->temp, sizeof(cplx) * m->N);
}
double SFX(orc_kinetic)(MODEL* m, const real* p) {
  mass_matrix(m);
  return kinetic_impl(m, (const cplx*)p);
}

/* The leapfrog loop of MultiResParameters.h:689-700 (momentum given). */
static void leapfrog_impl(MODEL* m, cplx* mu_star, cplx* p, real eps, int L) {
  real k = 0.5;
  gradient_impl(m, mu_star);
  for (long i = 0; i < m->N; i++) p[i] += (k * eps) * m->temp[i];
  const real scale = (real)m->N / eps;
  for (int step = 0; step < L; step++) {
    k = (step == (L - 1)) ? (real)0.5 : (real)1;
    memcpy(m->temp, p, sizeof(cplx) * m->N);
    inv(m, m->temp);
    for (long i = 0; i < m->N; i++) m->temp[i] /= m->lambda_mass[i] * scale;
    low_rank_adjust(m, m->temp);
    fwd(m, m->temp);
    for (long i = 0; i < m->N; i++) mu_star[i] += m->temp[i];
    gradient_impl(m, mu_star);
    for (long i = 0; i < m->N; i++) p[i] += (k * eps) * m->temp[i];
  }
}

void SFX(orc_leapfrog)(MODEL* m, real* mu, real* p, real eps, int L) {
  mass_matrix(m);
  leapfrog_impl(m, (cplx*)mu, (cplx*)p, eps, L);
}

/* MultiResParameters.h:784-815 with injected normals (z[2i] = re, z[2i+1] = im). */
static double sample_momentum_injected(MODEL* m, const real* z) {
  double E0 = 0.0, A, B, c = 0.0;
  for (long i = 0; i < m->N; i++) {
    m->momentum[i] = z[2 * i] + z[2 * i + 1] * I;
    A = ((double)z[2 * i] * z[2 * i] + (double)z[2 * i + 1] * z[2 * i + 1]) - c;
    B = E0 + A;
    c = (B - E0) - A;
    E0 = B;
  }
  E0 *= -0.5;
  inv(m, m->momentum);
  const real Nr = (real)m->N;
  for (long i = 0; i < m->N; i++) m->momentum[i] *= CSQRT(m->lambda_mass[i]) / Nr;
  low_rank_adjust(m, m->momentum);
  fwd(m, m->momentum);
  return E0;
}

/* MultiResParameters.h:674-727 without the Gibbs step. */
static double transition_impl(MODEL* m, const real* z, double u, real eps, int L, double* out, double* norms) {
  memcpy(m->mu_star, m->mu, sizeof(cplx) * m->N);
  mass_matrix(m);
  double E0 = sample_momentum_injected(m, z);
  double nrm0[2], nrm1[2];
  const double lp_initial = log_prior_impl(m, m->mu) + log_lik_impl(m, m->mu, nrm0);
  E0 += lp_initial;
  leapfrog_impl(m, m->mu_star, m->momentum, eps, L);
  const double lp_proposal = log_prior_impl(m, m->mu_star) + log_lik_impl(m, m->mu_star, nrm1);
  const double proposed = lp_proposal + kinetic_impl(m, m->momentum);
  double R = exp(proposed - E0);
  if (isnan(R)) R = 0;
  const int accept = u < R;
  if (accept) memcpy(m->mu, m->mu_star, sizeof(cplx) * m->N);
  set_real_mu(m, m->mu);
  if (out) { out[0] = R; out[1] = accept; out[2] = lp_initial; out[3] = E0; out[4] = proposed; out[5] = 0; }
  if (norms) { norms[0] = accept ? nrm1[0] : nrm0[0]; norms[1] = accept ? nrm1[1] : nrm0[1]; }
  return R < 1.0 ? R : 1.0;
}

double SFX(orc_transition)(MODEL* m, const real* z, double u, real eps, int L, double* out, double* norms) {
  return transition_impl(m, z, u, eps, L, out, norms);
}

double SFX(orc_momentum)(MODEL* m, const real* z, real* p) {
  mass_matrix(m);
  const double E0 = sample_momentum_injected(m, z);
  memcpy(p, m->momentum, sizeof(cplx) * m->N);
  return E0;
}

/* --------------------------- oracle RNG ---------------------------------- */
/* xoshiro256** seeded by splitmix64; Box-Muller normals; Marsaglia-Tsang gamma. */
typedef struct { uint64_t s[4]; int have; double cached; } orng;
static uint64_t splitmix(uint64_t* x) {
  uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static void orng_seed(orng* r, uint64_t seed) {
  for (int i = 0; i < 4; i++) r->s[i] = splitmix(&seed);
  r->have = 0;
}
static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t orng_next(orng* r) {
  const uint64_t res = rotl(r->s[1] * 5, 7) * 9, t = r->s[1] << 17;
  r->s[2] ^= r->s[0]; r->s[3] ^= r->s[1]; r->s[1] ^= r->s[2]; r->s[0] ^= r->s[3];
  r->s[2] ^= t; r->s[3] = rotl(r->s[3], 45);
  return res;
}
static double orng_u01(orng* r) { return ((double)(orng_next(r) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
static double orng_normal(orng* r) {
  if (r->have) { r->have = 0; return r->cached; }
  const double u1 = orng_u01(r), u2 = orng_u01(r);
  const double rad = sqrt(-2.0 * log(u1));
  r->cached = rad * sin(2.0 * M_PI * u2);
  r->have = 1;
  return rad * cos(2.0 * M_PI * u2);
}
static double orng_gamma(orng* r, double shape, double scale) {
  if (shape < 1.0) {
    const double g = orng_gamma(r, shape + 1.0, 1.0);
    return g * pow(orng_u01(r), 1.0 / shape) * scale;
  }
  const double d = shape - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
  for (;;) {
    double x, v;
    do { x = orng_normal(r); v = 1.0 + c * x; } while (v <= 0.0);
    v = v * v * v;
    const double u = orng_u01(r);
    if (log(u) < 0.5 * x * x + d - d * v + d * log(v)) return d * v * scale;
  }
}

/* MultiResParameters.h:744-759 */
static void initialize_mu(MODEL* m, orng* r) {
  for (long i = 0; i < m->N; i++) {
    const real b = (real)orng_normal(r), a = (real)orng_normal(r);
    m->mu[i] = a + b * I;
  }
  fwd(m, m->mu);
  const real k = 10 * (real)m->N;
  for (long i = 0; i < m->N; i++) m->mu[i] *= CSQRT(m->lambda[i]) / k;
  low_rank_adjust(m, m->mu);
  inv(m, m->mu);
  set_real_mu(m, m->mu);
}

/* MultiResParameters.h:764-778 */
static void initialize_sigma(MODEL* m, orng* r, double shape) {
  m->sigma_sq_inv[0] = (real)orng_gamma(r, shape, 1.0);
  if (m->n_datasets == 2) m->sigma_sq_inv[1] = m->sigma_sq_inv[0] / (real)orng_u01(r);
}

/* MultiResParameters.h:821-838 */
static void update_sigma(MODEL* m, orng* r, const double* norms) {
  const real shape_h = (real)(0.5 * m->n_h + 1);
  const real rate_h = (real)(0.5 * norms[0]);
  m->sigma_sq_inv[0] = (real)orng_gamma(r, shape_h, 1.0 / rate_h);
  if (m->n_datasets == 2) {
    const real shape_s = (real)(0.5 * m->n_s + 1);
    const real rate_s = (real)(0.5 * norms[1]);
    m->sigma_sq_inv[1] = (real)orng_gamma(r, shape_s, 1.0 / rate_s);
  }
}

static double one_update(MODEL* m, orng* r, real eps, int L, real* z) {
  for (long i = 0; i < 2 * m->N; i++) z[i] = (real)orng_normal(r);
  double norms[2];
  const double u = orng_u01(r);
  const double rate = transition_impl(m, z, u, eps, L, NULL, norms);
  update_sigma(m, r, norms);
  return rate;
}

/* gaussian_process_model.h:88-177 + mcmc_summary (:191-316) */
int SFX(orc_fit)(MODEL* m, int burnin, int n_save, int thin, int L, double mh_target, uint64_t seed,
                 double* mean, double* var, double* activation, double* stats) {
  orng r;
  orng_seed(&r, seed);
  initialize_mu(m, &r);
  initialize_sigma(m, &r, m->theta[0]);
  /* add_data_to_mu (MultiResParameters.h:632-641) */
  for (int i = 0; i < m->n_h; i++) m->mu[m->D[i]] += m->Yh[i];
  orc_hmc h;
  if (orc_hmc_init(&h, burnin, n_save, thin, L, 1.0 / L, mh_target) != 0) return -1;
  real* z = (real*)malloc(sizeof(real) * 2 * m->N);
  double* s1 = (double*)calloc(m->n_o, sizeof(double));
  double* s2 = (double*)calloc(m->n_o, sizeof(double));
  double* sa = (double*)calloc(m->n_o, sizeof(double));
  int save_count = 0, samples = 0;
  double grads = 0, iters = 0;
  while (save_count < h.n_save && h.iteration <= orc_hmc_max_iterations(&h)) {
    const real eps = (real)orc_hmc_eps(&h, h.warmup ? 0.5 : orng_u01(&r));
    const int Li = orc_hmc_integrator_steps(&h);
    const double rate = one_update(m, &r, eps, Li, z);
    grads += Li + 1; iters += 1;
    orc_hmc_update(&h, rate);
    if (orc_hmc_save_iteration(&h)) {
      double mx = 0;
      for (int i = 0; i < m->n_o; i++) { const double v = fabs((double)CRE(m->mu[m->O[i]])); if (v > mx) mx = v; }
      if (mx < 1e-6) mx = 1e-6;
      for (int i = 0; i < m->n_o; i++) {
        const double v = (double)CRE(m->mu[m->O[i]]);
        s1[i] += v; s2[i] += v * v; sa[i] += fabs(v) / mx;
      }
      samples++;
      save_count++;
    }
  }
  const double n = samples > 0 ? samples : 1;
  double amax = -1e300;
  for (int i = 0; i < m->n_o; i++) {
    mean[i] = s1[i] / n;
    var[i] = (s2[i] - s1[i] * s1[i] / n) / n;
    activation[i] = sa[i] / (n * sqrt(var[i]));
    if (activation[i] > amax) amax = activation[i];
  }
  for (int i = 0; i < m->n_o; i++) activation[i] /= amax;
  stats[0] = orc_hmc_mh_rate(&h);
  stats[1] = h.eps;
  stats[2] = grads;
  stats[3] = iters;
  free(z); free(s1); free(s2); free(sa);
  return samples;
}

int64_t SFX(orc_run_iterations)(MODEL* m, int iters, int L, real eps, uint64_t seed) {
  orng r;
  orng_seed(&r, seed);
  real* z = (real*)malloc(sizeof(real) * 2 * m->N);
  int64_t grads = 0;
  for (int it = 0; it < iters; it++) {
    one_update(m, &r, eps, L, z);
    grads += L + 1;
  }
  free(z);
  return grads;
}
