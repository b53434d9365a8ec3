/*
 * dr_oracle.h -- CPU oracle for the dual-resolution GP-HMC sampler path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links, loads or
 * calls this code.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may use it, and only as the checker or as the timed CPU
 * restatement of the reference path.
 *
 * Parity status: UNPINNED.  The reference (asw221/dualres) ships no tests,
 * golden vectors or fixtures for this path, and it cannot be compiled in this
 * image (it needs Eigen >= 3.3, FFTW3 with threads, Boost.filesystem and
 * NLopt, none of which are installed).  The oracle is therefore a restatement
 * of the reference's algorithm, cross-checked against an independent numpy
 * restatement (tests/golden/gen_golden.py) and analytic known-answer tests.
 *
 * Every function cites the reference file:line it restates (paths relative
 * to the reference project root).
 *
 * Precision-dependent entry points exist twice: suffix _d (double, restating
 * the `dualgpm` build) and _f (float, restating the `dualgpmf` build with
 * DUALRES_SINGLE_PRECISION).  The float build keeps the reference's
 * double-precision Kahan sums and double likelihood norms.
 */
#ifndef DR_ORACLE_H
#define DR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- precision independent (dr_oracle_common.c) ------------- */

/* Nonzero = not NaN and != 0 (include/dualres/impl/nifti_manipulation.inl:335-360).
 * Writes column-major (i fastest) ijk triples; returns the count. */
int orc_nonzero_indices(const float* img, int nx, int ny, int nz, int* ijk, int max_out);

/* Bounding box of the nonzero voxels (nifti_manipulation.inl:210-219).
 * Returns nnz; bbmin/bbmax get 3 ints each.  nnz == 0 leaves them untouched. */
int orc_bounding_box(const float* img, int nx, int ny, int nz, int* bbmin, int* bbmax);

/* Embedding dims E_d = 2^ceil(log2(2 (g_d - 1))) (MultiResParameters.h:191-206,
 * circulant_base.inl:44-57).  Returns 0, or -1 if some g_d <= 1. */
int orc_embedding_dims(const int* g, int* E);

/* Neighbourhood offsets within `radius` mm (kriging_matrix.h:41-56, 63-106).
 * Q is the 4x4 row-major qform.  Offsets are written as ijk triples, i fastest.
 * Returns the number of offsets, or -1 when max_out is too small. */
int orc_neighborhood(const float* Q, float radius, int* P, int max_out);

/* Preprocessing of dualgpm.cpp:125-155, 288 and gaussian_process_model.h:104-117:
 *  - hr is masked in place by hmask (zero where mask == 0 or hr is NaN),
 *  - union = hmask + omask, input bbox = bbox(union nonzeros),
 *  - D = nonzero hr ijk inside that bbox, relative to its min corner,
 *  - O = nonzero omask ijk inside that bbox, relative to its min corner,
 *  - Yh = nonzero hr values (column-major).
 * hmask / omask may be NULL (the reference defaults both to the hr image,
 * GPMCommandParser.inl:532-540).  Returns n_h, or a negative error code.
 * *n_o receives the output count. */
int orc_prepare_highres(float* hr, const float* hmask, const float* omask,
                        int nx, int ny, int nz,
                        int* D_ijk, float* Yh, int* O_ijk, int* n_o, int max_out);

/* Kriging CSR (kriging_matrix.h:148-343).  theta = (variance, bandwidth,
 * exponent).  Weights are solved in double by column-pivoted Householder QR
 * (the reference uses Eigen's colPivHouseholderQr in float).  solve == 0
 * builds the sparsity pattern only (val untouched).  Returns nnz, -1 when a
 * buffer is too small, -2 for more than 5000 offsets, -3 for an index that
 * would read outside the bounded index map (undefined behaviour in the
 * reference).  rowptr has n_std_nonzero + 1 entries. */
int64_t orc_kriging_build(const float* hr, int nx, int ny, int nz, const float* Qhr,
                          const float* sr, int sx, int sy, int sz, const float* Qsr,
                          const float* theta, float radius, int solve,
                          int* rowptr, int max_rows, int* col, double* val,
                          int64_t max_nnz, int* n_rows_out);

/* Covariance functions (kernels.inl:8-15, 59-74). covfun 0 = rbf, 1 = rational quadratic. */
double orc_cov(int covfun, double d, const double* theta);

/* Minimum contrast estimation summary (estimate_kernel_parameters.h:50-101):
 * the lattice offsets of perturbation_matrix_3d (perturbation_matrix.h:19-109),
 * in its order, deduplicated keeping first occurrences; returns the count
 * (25348) and fills P (3 ints per offset) when P is not NULL. */
int orc_mce_offsets(int* P, int max_out);
/* For every offset: distance |Q_3x3 p| (float), the covariance of the pairs of
 * non-zero, non-NaN voxels (x, x + p) inside the grid (double sums, stored as
 * float) and the pair counts.  Also returns the raw double sums (3 per offset)
 * when sums is not NULL. */
int orc_mce_summary(const float* img, int nx, int ny, int nz, const float* Q, const int* P, int n_off,
                    float* distance, float* covariance, int* npairs, double* sums);

/* HMCParameters (HMCParameters.h:97-297), double state. */
typedef struct {
  int warmup, eps_start_found, burnin, integrator_steps, iteration, n_save, thin;
  double A, eps, eps0, eps_bar, eps_target, gamma, h_bar, mh_running_sum, mh_target, t0, kappa;
} orc_hmc;
int orc_hmc_init(orc_hmc* h, int burnin, int n_save, int thin, int L,
                 double starting_eps, double mh_target);
double orc_hmc_eps(const orc_hmc* h, double jitter_u01);   /* jitter_u01 = U(0,1) draw, used post-warmup */
int orc_hmc_integrator_steps(const orc_hmc* h);
void orc_hmc_update(orc_hmc* h, double mh_rate);
int orc_hmc_save_iteration(const orc_hmc* h);
int orc_hmc_max_iterations(const orc_hmc* h);
double orc_hmc_mh_rate(const orc_hmc* h);

/* ---------------- precision dependent (dr_oracle_model.c) ---------------- */

/* Opaque model state (MultiResParameters<T> + MultiResData<T>). */
typedef struct orc_model_d orc_model_d;
typedef struct orc_model_f orc_model_f;

#define ORC_DECLARE(SFX, REAL)                                                       \
  /* Unnormalised 3D DFT, FFTW sign convention, x fastest (sized_fft.h:138-159). */ \
  void orc_fft3d##SFX(REAL* data_interleaved, const int* E, int inverse);           \
  /* MultiResParameters ctor (MultiResParameters.h:173-300) without the random    \
   * initialisation: embedding, circulant base, lambda, S, data indices.         \
   * W is n_s x n_h CSR (may be NULL with n_s = 0 for single resolution). */     \
  orc_model##SFX* orc_model_create##SFX(int n_h, const int* D_ijk, const float* Yh,  \
      int n_s, const float* Ys, const int* rowptr, const int* col, const REAL* val, \
      const float* Q, const double* theta, int covfun, int n_o, const int* O_ijk,   \
      int* status);                                                                 \
  void orc_model_free##SFX(orc_model##SFX* m);                                      \
  void orc_model_info##SFX(const orc_model##SFX* m, int* E, int64_t* N, int* n_S);  \
  /* lambda as interleaved complex (re, im), N entries. */                         \
  void orc_model_lambda##SFX(const orc_model##SFX* m, double* out);                 \
  void orc_model_set_sigma##SFX(orc_model##SFX* m, REAL sh, REAL ss);               \
  void orc_model_get_sigma##SFX(const orc_model##SFX* m, REAL* s2inv);              \
  void orc_model_set_mu##SFX(orc_model##SFX* m, const REAL* mu);                    \
  void orc_model_get_mu##SFX(const orc_model##SFX* m, REAL* mu);                    \
  double orc_log_prior##SFX(orc_model##SFX* m, const REAL* mu);                     \
  double orc_log_likelihood##SFX(orc_model##SFX* m, const REAL* mu);                \
  void orc_gradient##SFX(orc_model##SFX* m, const REAL* mu, REAL* grad);            \
  double orc_kinetic##SFX(orc_model##SFX* m, const REAL* p);                        \
  /* Fixed-momentum leapfrog of MultiResParameters.h:689-700.  mu and p are      \
   * updated in place.  Returns nothing; energies via orc_log_prior etc. */       \
  void orc_leapfrog##SFX(orc_model##SFX* m, REAL* mu, REAL* p, REAL eps, int L);    \
  /* One HMC transition (MultiResParameters.h:674-727) with injected randomness:  \
   * z = 2N standard normals (re, im interleaved), u = accept uniform.  The        \
   * Gibbs draws are skipped; out[0..5] = {R, accepted, lp_initial, E0,            \
   * proposed_energy, 0}; norms[0..1] = squared residual norms at the kept mu. */  \
  double orc_transition##SFX(orc_model##SFX* m, const REAL* z, double u, REAL eps,  \
                             int L, double* out, double* norms);                    \
  /* The momentum draw alone (MultiResParameters.h:784-815) from injected       \
   * normals z (as orc_transition): writes p (N complex, re/im interleaved) and   \
   * returns E0 = -1/2 sum |z|^2.  Uses the current sigma for the mass matrix. */ \
  double orc_momentum##SFX(orc_model##SFX* m, const REAL* z, REAL* p);              \
  /* Full fit_model loop (gaussian_process_model.h:88-177) with the oracle's own  \
   * RNG.  Outputs (n_o each): mean, var, activation; stats[0..3] = {mh rate,    \
   * final eps, gradient evaluations, iterations}. */                            \
  int orc_fit##SFX(orc_model##SFX* m, int burnin, int n_save, int thin, int L,      \
                   double mh_target, uint64_t seed, double* mean, double* var,      \
                   double* activation, double* stats);                               \
  /* Runs `iters` transitions from the current state (timing helper for the CPU  \
   * baseline).  Returns gradient evaluations performed. */                      \
  int64_t orc_run_iterations##SFX(orc_model##SFX* m, int iters, int L, REAL eps,    \
                                  uint64_t seed);                                     \
  void orc_set_threads##SFX(int n);

ORC_DECLARE(_d, double)
ORC_DECLARE(_f, float)

#ifdef __cplusplus
}
#endif
#endif
