/*
 * dualres_b200.h -- C ABI of the B200-native dual-resolution GP-HMC sampler.
 *
 * This is the drop-in boundary for the `dualgpmf` path of asw221/dualres.  The
 * reference has no C ABI of its own; its boundary is the C++ template API
 * (MultiResData<T>, MultiResParameters<T>, HMCParameters<T>, fit_model) plus
 * the `dualgpmf` command line.  Each entry point below names the reference
 * interface it replaces (paths relative to the reference project root).
 *
 * Conventions
 *  - Every function returns DR_OK (0) or a negative DR_ERR_* code;
 *    dr_last_error() returns a message for the calling thread.  No C++
 *    exception crosses this boundary (the reference throws std::domain_error /
 *    std::logic_error, which dualgpm.cpp:382-405 turns into exit code 1).
 *  - Images are float32, x fastest (NIfTI column-major), 0 or NaN = no data.
 *  - Qforms are 4x4 float32 row-major (nifti_manipulation.h:34).
 *  - Complex fields are interleaved float32 (re, im), x fastest, on the
 *    embedding grid E0 x E1 x E2.
 *  - Unless a parameter says "device", pointers are host pointers.
 *  - Handles are not thread-safe; use one handle per thread.
 *  - The library runs only on a CUDA GPU (sm_100a).  There is no CPU path.
 */
#ifndef DUALRES_B200_H
#define DUALRES_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DR_OK 0
#define DR_ERR_INVALID (-1)     /* bad argument: NULL, size, range */
#define DR_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define DR_ERR_NOMEM (-3)       /* device memory exhausted or budget exceeded */
#define DR_ERR_DOMAIN (-4)      /* model domain error (std::domain_error in the reference) */
#define DR_ERR_UNSUPPORTED (-5) /* a size outside the supported range */
#define DR_ERR_STATE (-6)       /* call not valid in the current state */
#define DR_ERR_TIMEOUT (-7)     /* a bounded device wait gave up */

#define DR_COV_RBF 0 /* v exp(-b |d|^e)            (include/dualres/impl/kernels.inl:8-15)  */
#define DR_COV_RQ 1  /* v (1 + psi/nu d^2)^(-nu)   (include/dualres/impl/kernels.inl:59-74) */

typedef struct dr_volume dr_volume;
typedef struct dr_chainset dr_chainset;

/* One dual-resolution problem: the inputs `dualgpmf` reads
 * (src/dualgpm.cpp:84-245, GPMCommandParser.inl:196-545). */
typedef struct {
  int nx, ny, nz;          /* high-res image grid (voxels) */
  const float* highres;    /* nx*ny*nz, required (--highres) */
  const float* qform_hr;   /* 16 floats */
  const float* hmask;      /* optional (--hmask); NULL = the high-res image itself */
  const float* omask;      /* optional (--omask); NULL = the high-res image itself */
  int sx, sy, sz;          /* std-res grid; ignored when stdres == NULL */
  const float* stdres;     /* optional (--stdres); NULL = single resolution */
  const float* qform_sr;   /* 16 floats, required with stdres */
  const float* smask;      /* optional (--smask) */
  float covariance[3];     /* --covariance: variance, bandwidth, exponent */
  int covfun;              /* DR_COV_RBF (default) or DR_COV_RQ (--rational-quadratic) */
  float neighborhood;      /* --neighborhood mm; <= 0 = 3 x largest voxel dimension */
  int device;              /* CUDA device ordinal */
} dr_volume_desc;

typedef struct {
  int E[3];                   /* embedding grid */
  int64_t N;                  /* E0*E1*E2 */
  int box[3];                 /* real-space region covering data and output voxels */
  int n_highres;              /* data voxels (rows of Yh) */
  int n_stdres;               /* std-res voxels (rows of W) */
  int n_output;               /* output voxels */
  int64_t kriging_nnz;        /* nnz(W) */
  int n_nonpositive;          /* |S|, eigenvalues with Re <= 0 */
  double max_eigenvalue;      /* lambda[0] / N */
  double setup_seconds;       /* host + device set-up time */
  double kriging_seconds;     /* of which the kriging build */
  float neighborhood;         /* radius used (mm) */
  int64_t device_bytes;       /* device memory held by the volume */
  double kriging_plan_seconds;   /* of the kriging build: sparsity, covariances and K^-1 */
  double kriging_solve_seconds;  /* ... the per-row solves (device, or host) */
  int kriging_device_rows;    /* rows solved on the device (complete rows with equal k' once) */
  int kriging_host_rows;      /* rows left to the host (not numerically positive definite) */
} dr_volume_info;

/* Replaces MultiResData<T>(h_res, s_res, theta, r) (MultiResData.h:96-127), the
 * kriging build (kriging_matrix.h:148-343) and the one-time part of the
 * MultiResParameters<T> constructor (MultiResParameters.h:173-300): masks,
 * bounding box, data/output indices, circulant eigenvalues (FP64) and S.
 * Errors: DR_ERR_DOMAIN for |S| >= N/2 (MultiResParameters.h:283-284), invalid
 * covariance (dualgpm.cpp:447-464) or > 5000 neighbourhood offsets
 * (kriging_matrix.h:172-174). */
int dr_volume_create(const dr_volume_desc* desc, dr_volume** out);
int dr_volume_info_get(const dr_volume* v, dr_volume_info* info);
/* W as CSR (host buffers of n_stdres+1, kriging_nnz, kriging_nnz entries). */
int dr_volume_kriging_get(const dr_volume* v, int* rowptr, int* col, float* val);
/* Re lambda in FP64 (N entries); MultiResParameters::lambda() (:411-415). */
int dr_volume_lambda_get(const dr_volume* v, double* lambda_re);
/* Flat embedding-grid indices of the data (n_highres) and output (n_output)
 * voxels; MultiResParameters::data_indices() (:419-422). Either may be NULL. */
int dr_volume_indices_get(const dr_volume* v, int* data_idx, int* out_idx);
/* Observed data vectors; MultiResData::Yh()/Ys() (MultiResData.h:139-150). */
int dr_volume_data_get(const dr_volume* v, float* Yh, float* Ys);
/* Releases the handle.  Device memory is freed now, or when the last chain set
 * created on the volume is destroyed. */
void dr_volume_destroy(dr_volume* v);

/* HMC settings: HMCParameters<T>(burnin, nsave, thin, L, eps0, mhtarget)
 * (HMCParameters.h:97-149) plus the --seed option. */
typedef struct {
  int burnin;              /* --burnin (default 1000) */
  int nsave;               /* --nsave (default 1000) */
  int thin;                /* --thin (default 3) */
  int leapfrog;            /* --leapfrog (default 25) */
  float mhtarget;          /* --mhtarget (default 0.65) */
  float starting_eps;      /* <= 0: 1 / leapfrog (dualgpm.cpp:253-258) */
  uint64_t seed;           /* --seed */
  int store_samples;       /* keep every saved output-voxel sample on the device (--samples) */
} dr_hmc_opts;

typedef struct {
  int iteration;           /* HMCParameters::iteration() */
  int saved;               /* samples accumulated in the summary */
  int integrator_steps;    /* HMCParameters::integrator_steps() for the next iteration */
  float eps;               /* HMCParameters::eps_value() */
  float mh_rate;           /* HMCParameters::metropolis_hastings_rate() */
  float sigma_hr;          /* MultiResParameters::sigma(0) */
  float sigma_sr;          /* MultiResParameters::sigma(1) */
  double last_log_ratio;   /* log R of the last transition (proposed - initial energy) */
  int64_t accepted;        /* accepted transitions */
  int64_t grad_evals;      /* gradient evaluations so far (sum of L + 1) */
  int done;                /* nsave samples saved */
  float last_eps;          /* step size of the last transition (the eps argument of update) */
  double initial_energy;   /* initial and proposed energy of the last transition, as */
  double proposed_energy;  /* --monitor prints them (MultiResParameters.h:700-713) */
} dr_chain_stats;

/* n_chains independent chains on one volume, advanced together.  Each chain
 * is initialised as MultiResParameters<T> does (_initialize_mu / _initialize_sigma,
 * MultiResParameters.h:744-778) followed by add_data_to_mu (:632-641). */
int dr_chainset_create(dr_volume* v, int n_chains, const dr_hmc_opts* opts, dr_chainset** out);
/* One MultiResParameters::update + HMCParameters::update per chain and per
 * iteration (the loop body of gaussian_process_model.h:134-171), `iterations`
 * times.  Chains that have saved nsave samples stop changing. */
int dr_step(dr_chainset* cs, int iterations);
/* dr_step, also returning the device time of the iterations in ms, measured
 * with CUDA events on the chainset's stream around the launches. */
int dr_step_timed(dr_chainset* cs, int iterations, double* device_ms);
/* Runs until every chain has saved nsave samples (fit_model's loop). */
int dr_run(dr_chainset* cs);
int dr_chain_stats_get(dr_chainset* cs, dr_chain_stats* stats /* n_chains entries */);
/* Posterior summary of mcmc_summary<T> (gaussian_process_model.h:191-316):
 * mean, variance and activation over the output voxels (n_output each, any
 * may be NULL).  chain = -1 pools every chain. */
int dr_summary_get(dr_chainset* cs, int chain, float* mean, float* var, float* activation);
/* Saved samples of one chain at the output voxels: n_saved x n_output floats
 * (requires store_samples). */
int dr_samples_get(dr_chainset* cs, int chain, float* samples, int max_saved, int* n_saved);
/* Per saved iteration of one chain: sigma_hr, sigma_sr (0 in single-resolution
 * mode) and the log likelihood, n_saved x 3 doubles (requires store_samples);
 * the columns after mu in the --samples stream (gaussian_process_model.h:149-163). */
int dr_sample_records_get(dr_chainset* cs, int chain, double* rec, int max_saved, int* n_saved);
void dr_chainset_destroy(dr_chainset* cs);
/* The configuration the chain set runs (no reference counterpart): update path
 * (0 fused x/y plane kernel, 1 the same with bulk prefetch of the state planes,
 * 2 x-line kernel with separate y passes), kriging-product blocks per SM, the
 * iteration time measured when the shape was tuned (0 when it was not), and
 * whether the kriging products run on the tensor cores (1; 2 when W^T's chain
 * vectors arrive by TMA row gathers) or as CSR products (0).  At creation the update paths are timed on a scratch chain set of the
 * same shape (with the tensor-core products where available), then the other
 * product choices on the fastest path, and the fastest is kept for the process;
 * DRB_AUTOTUNE=0 turns this off, DRB_NO_PLANE / DRB_PLANE_PREFETCH force a
 * path, DRB_TC_PRODUCTS=0 / 1 the products.  Any output may be NULL. */
int dr_chainset_config_get(const dr_chainset* cs, int* path, int* blocks_per_sm, double* tuned_ms,
                           int* tensor_products);
/* The tile shape of the chain set's z passes, chosen by the same tuning (DRB_ZTILE=1 / 8 forces it): chains per tile,
 * 8 for tiles of 4 lines x 8 chains, 1 for tiles of 32 lines of one chain (always 1 below 8 chains).  No reference
 * counterpart: the reference's FFTW plans have no tiles. */
int dr_chainset_ztile_get(const dr_chainset* cs, int* z_tile_chains);
/* The radix plans of the chain set's transforms of length 64, 128 and 256, chosen by the same tuning
 * (DRB_FFT_PLAN=<bits> forces them): *plan has bit 1 set when the inverse z pass uses the second plan, bit 2 the
 * forward z pass, bit 4 the x transforms of the x-line kernel (first plan: 8 x 8, 16 x 8, 16 x 16 radices; second:
 * 16 x 4, 8 x 16, 8 x 8 x 4).  Replaces the per-size plans FFTW chooses when the reference plans its transforms
 * (sized_fft.h:63-68). */
int dr_chainset_fft_plan_get(const dr_chainset* cs, int* plan);

/* ---- fixed-input evaluation (MultiResParameters public API) ------------- */
/* Sets chain `chain` to mu (2N floats) and sigma^-2 = (s_hr, s_sr). */
int dr_set_state(dr_chainset* cs, int chain, const float* mu, float s_hr, float s_sr);
/* mu (2N floats) and sigma^-2 of a chain (MultiResParameters::mu_ / sigma). */
int dr_get_state(dr_chainset* cs, int chain, float* mu, float* s2inv);
/* Checkpoint of a chain set's sampler state into a host buffer: every chain's accepted spectral state, mu at the
 * data and output voxels, the chain states (iteration, step size and dual averaging, sigma, accept bookkeeping; the
 * counter-based RNG needs nothing else), the posterior-summary sums and any stored samples.  A chain set created on
 * the same volume with the same options and chain count and restored from it continues bit for bit as the saved
 * one would have (DR_ERR_INVALID when the shapes differ).  _size gives the bytes of the buffer.  No reference
 * counterpart (the reference's fits run to completion in one process). */
int dr_chainset_checkpoint_size(const dr_chainset* cs, int64_t* bytes);
int dr_chainset_checkpoint_save(dr_chainset* cs, void* buf, int64_t bytes);
int dr_chainset_checkpoint_restore(dr_chainset* cs, const void* buf, int64_t bytes);
/* log prior (MultiResParameters.h:429-476) and log likelihood (:488-514) at mu
 * with the chain's sigma: out[0] = prior, out[1] = likelihood. */
int dr_log_posterior(dr_chainset* cs, int chain, const float* mu, double* out);
/* Gradient of the log posterior at mu (MultiResParameters.h:337-376), 2N floats. */
int dr_gradient(dr_chainset* cs, int chain, const float* mu, float* grad);
/* The leapfrog integrator of MultiResParameters::update (:689-700) from
 * (mu0, p0) with a fixed momentum, through the same device kernels that run
 * the sampler.  energies[0..5] = {log prior(mu0), log lik(mu0), kinetic(p0),
 * log prior(muL), log lik(muL), kinetic(pL)} with kinetic as in :551-603. */
int dr_leapfrog_fixed(dr_chainset* cs, int chain, const float* mu0, const float* p0, float eps,
                      int L, float* mu_out, float* p_out, double* energies);

/* Same result as dr_log_posterior, but the call allocates no device memory.
 * It is meant for callers that cannot call cudaMalloc or cudaFree at this
 * point: code whose device memory belongs to another allocator (a framework's
 * caching allocator or a fixed arena), or a serving loop that has stopped
 * allocating after start-up, since cudaFree synchronises the whole device and
 * allocations fragment a shared pool.  No reference counterpart: the reference
 * runs on the CPU only.
 *   v          volume (created beforehand; its creation does allocate)
 *   mu_device  real-space field on the device, 2N floats (re, im), x fastest
 *   s_hr, s_sr sigma^-2 of the high-res and std-res data
 *   out        host, out[0] = log prior, out[1] = log likelihood
 * Scratch is one library-owned array of ~32 MiB that every GPU loading the
 * library holds until the process exits.  Limits: N <= 2^21 (e.g. 128^3),
 * n_highres <= 2^20, n_stdres <= 2^20; larger volumes get DR_ERR_UNSUPPORTED.
 * The first call on a device looks up the array's device address; make that
 * first call before any stream capture.  All calls share the array: calls
 * that overlap on the GPU (several host threads, or several devices sharing a
 * context) race, so serialise them.  The call runs on the legacy default
 * stream and returns when the result is on the host.  The legacy stream is
 * not ordered after work on streams created with cudaStreamNonBlocking, so
 * the writes that produce mu_device must be finished before the call
 * (synchronise the producing stream, or produce mu_device on the legacy
 * stream).  The caller's current device is the same after the call. */
int dr_log_posterior_noalloc(const dr_volume* v, const float* mu_device, float s_hr, float s_sr, double* out);

/* ---- serving: continuous batching of denoising jobs --------------------- */
/* A request loop that the reference does not have (it fits one volume per
 * process).  Each job is one dualgpmf fit (volume + n_chains chains).  Host
 * set-up (masks, indices, kriging) runs on worker threads; a scheduler thread
 * admits prepared jobs while their device footprint fits the HBM budget, keeps
 * each job's chain state resident, and advances every admitted job a few
 * iterations per round on its own stream, so jobs that arrive while others run
 * overlap with them on the device.  Results are identical to running the job
 * alone: every job's random streams depend only on its seed. */
typedef struct dr_server dr_server;

typedef struct {
  int device;
  int64_t hbm_budget_bytes;    /* admission budget; <= 0: 80 % of the device memory free at creation */
  int max_active;              /* jobs resident on the device at once; <= 0: 64 */
  int iterations_per_round;    /* iterations each admitted job advances per round; <= 0: 8 */
  int host_threads;            /* set-up workers; <= 0: 4 */
  int max_chains_in_flight;    /* chains of the resident jobs advanced at once, earliest admitted first (a job of
                                  more chains runs when it is the only one); <= 0: 128 */
} dr_server_opts;

#define DR_JOB_QUEUED 0   /* waiting for host set-up */
#define DR_JOB_READY 1    /* set up on the host, waiting for device memory */
#define DR_JOB_RUNNING 2  /* resident on the device */
#define DR_JOB_DONE 3
#define DR_JOB_FAILED 4
#define DR_JOB_PREEMPTED 5 /* checkpointed and released from the device; dr_server_resume continues it */

typedef struct {
  int state;                   /* DR_JOB_* */
  int error;                   /* DR_ERR_* when failed */
  double submit_s;             /* server clock (s) at submission */
  double admit_s;              /* ... when admitted to the device */
  double finish_s;             /* ... when the summary was read back */
  int64_t grad_evals;          /* sum over chains of L + 1 per iteration */
  float mh_rate;               /* mean over chains */
  int n_output;                /* output voxels */
  int64_t device_bytes;        /* footprint while resident */
} dr_job_status;

typedef struct {
  int64_t submitted, done, failed, running;
  int64_t grad_evals;          /* over finished jobs */
  int64_t peak_device_bytes;   /* largest resident footprint */
  int peak_running;            /* largest number of resident jobs */
  double busy_s;               /* server clock of the last finish */
  int64_t kernel_launches;     /* kernels the scheduler enqueued (graph nodes counted) */
} dr_server_stats;

int dr_server_create(const dr_server_opts* opts, dr_server** out);
/* Copies the images; returns immediately with the job id. */
int dr_server_submit(dr_server* sv, const dr_volume_desc* desc, const dr_hmc_opts* opts, int n_chains,
                     uint64_t* job_id);
int dr_server_status(dr_server* sv, uint64_t job_id, dr_job_status* out);
/* Posterior mean / variance / activation of a finished job (n_output each, any may be NULL). */
int dr_server_result(dr_server* sv, uint64_t job_id, float* mean, float* var, float* activation);
/* Waits (host side) until the job finished or failed, or timeout_s passed (DR_ERR_TIMEOUT). */
int dr_server_wait(dr_server* sv, uint64_t job_id, double timeout_s);
/* Preempts a resident job: at its next round boundary the scheduler saves its chain set's checkpoint
 * (dr_chainset_checkpoint_save) in host memory, releases its device memory (the host set-up, kriging matrix
 * included, is kept) and marks it DR_JOB_PREEMPTED; the call waits up to timeout_s for that.  DR_ERR_STATE when the
 * job is not admitted yet or has ended.  No reference counterpart (the reference runs one fit per process). */
int dr_server_preempt(dr_server* sv, uint64_t job_id, double timeout_s);
/* Re-admits a preempted job like a new submission (same id); once rebuilt on the device it continues from its
 * checkpoint, so its result equals that of an uninterrupted run bit for bit. */
int dr_server_resume(dr_server* sv, uint64_t job_id);
/* Waits until every submitted job finished or failed. */
int dr_server_drain(dr_server* sv, double timeout_s);
int dr_server_stats_get(dr_server* sv, dr_server_stats* out);
/* Releases a finished job's host record (results are no longer available). */
int dr_server_forget(dr_server* sv, uint64_t job_id);
void dr_server_destroy(dr_server* sv);

/* ---- covariance estimation (dualgpmf without --covariance) -------------- */
/* Lattice offsets of the minimum-contrast summary, perturbation_matrix_3d
 * (perturbation_matrix.h:62-109): *n = 25348; offsets (3 ints each, at most
 * max_out) may be NULL. */
int dr_mce_offsets(int* offsets, int max_out, int* n);
/* compute_mce_summary_data (estimate_kernel_parameters.h:50-115) on the GPU:
 * for every offset p, the distance |Q p| (mm), the covariance of the pairs of
 * non-zero, non-NaN voxels (x, x + p) and their count.  img is nx*ny*nz
 * floats, x fastest; qform row-major 4x4.  sums (3 doubles per offset: sum xy,
 * sum x, sum y) may be NULL. */
int dr_mce_summary(const float* img, int nx, int ny, int nz, const float* qform, int device, float* distance,
                   float* covariance, int* npairs, double* sums);
/* compute_rbf_parameters (estimate_kernel_parameters.h:267-390) with the
 * defaults dualgpm.cpp uses: bounded least squares of the RBF model to the
 * summary, bandwidth <= exponent, minimised by COBYLA.  theta: start values in
 * (dualgpm.cpp starts from 1, 0.6, 1.5), estimate out.  Host only. */
int dr_fit_rbf_parameters(const float* distance, const float* covariance, const int* npairs, int n, double* theta);
/* Both steps: compute_covar_parameters_if_needed (src/dualgpm.cpp:375-404). */
int dr_estimate_covariance(const float* img, int nx, int ny, int nz, const float* qform, int device, double* theta);

/* ---- host-side set-up --------------------------------------------------- */
/* The kriging matrix of get_sparse_kriging_matrix_data (kriging_matrix.h:
 * 148-343), built on the host (no GPU needed).  `highres` must already be
 * masked (the reference masks it first, dualgpm.cpp:126-137).  The CSR arrays
 * are allocated by the library; release them with dr_free. */
int dr_kriging_matrix(const float* highres, int nx, int ny, int nz, const float* qform_hr, const float* stdres, int sx,
                      int sy, int sz, const float* qform_sr, const float* covariance, float neighborhood, int* n_rows,
                      int64_t* nnz, int** rowptr, int** col, float** val);
void dr_free(void* p);

/* ---- diagnostics -------------------------------------------------------- */
/* Runs the device implementation of HMCParameters::update (HMCParameters.h:
 * 259-297) over n given MH rates and returns eps_value() and integrator_steps()
 * after each update; for parity checks of the step-size adaptation. */
int dr_debug_dual_averaging(int burnin, int nsave, int thin, int L, float starting_eps, float mhtarget,
                            int n, const float* mh_rates, double* eps_out, int* steps_out, int device);
/* Times `reps` back-to-back launches of one kernel of the leapfrog step at
 * step index `step` (>= 1) on the chainset's stream with CUDA events and
 * returns the mean duration in ms.  which: 0 x-line update, 1 forward y pass,
 * 2 forward z pass + gather, 3 W product, 4 W^T product, 5 inverse z pass,
 * 6 inverse y pass.  The kernels run on the live chain state, which they
 * change: call it only when the chains are no longer needed.  algo_bytes
 * receives the kernel's algorithmic bytes per launch (may be NULL). */
/* Runs one bounded mbarrier wait that nothing completes (the time-out path of
 * the library's bulk-copy and tensor-core pipelines): *gave_up = 1 when the
 * wait returned after about limit_ms (0 < limit_ms <= 10000) with the time it
 * waited in *waited_ms; the device stays usable. */
int dr_debug_bounded_wait(int device, double limit_ms, int* gave_up, double* waited_ms);

/* Host-only check of the dense-tile layout of the tensor-core kriging products
 * (no GPU): plans the n_rows x n_cols CSR matrix with the given row keys
 * (Z-order keys of 3 x 10-bit coordinates) for at most g_max CTAs, fills the
 * FP32 blob as the device does, and writes back the dense matrix read out of
 * the blob through the tiles' row and column maps (dense: n_rows x n_cols
 * floats; dense[0] is NaN if a padding position of the blob is not zero) and stats[0..6] = tiles, chunks,
 * segments, CTAs, chunks covered by the segments exactly once, matrix rows in
 * the tiles exactly once, and 1 if the segment index tables are consistent. */
int dr_debug_tc_layout(int n_rows, int n_cols, const int* rowptr, const int* col, const float* val,
                       const uint32_t* keys, int g_max, float* dense, int64_t* stats);
int dr_debug_time_kernel(dr_chainset* cs, int which, int step, int reps, double* avg_ms, double* algo_bytes);
/* Bytes in use and the high-water mark of the library's device memory pool (every stream-ordered allocation of
 * the library comes from it; it keeps freed memory for reuse).  reset_high != 0 first resets the high-water mark
 * to the bytes in use.  No reference counterpart (allocation accounting for tests). */
int dr_debug_pool_usage(int device, int reset_high, uint64_t* used, uint64_t* high);
/* Device kernel launches made by this thread since the last call (for launch accounting). */
int64_t dr_kernel_launches(int reset);
const char* dr_last_error(void);
const char* dr_version(void);

#ifdef __cplusplus
}
#endif
#endif
