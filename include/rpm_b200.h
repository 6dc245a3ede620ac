/*
 * rpm_b200.h -- C ABI of librpm_b200.so, the B200 (sm_100a) engine for the
 * radical-pair hot path of sam-not-smart/RPM.
 *
 * Reference files are cited relative to "Realistic system size/code/":
 *   ENG  = rpm_statevector_engine.py
 *   CORE = poster_reproduction/core.py
 *   JD   = rpm_quantum_needle_jd_sweeps.py
 *
 * Conventions
 *   - Every function returns an int status: RPM_OK (0) or one of RPM_E_*.
 *     rpm_last_error() returns a thread-local message for the last failure.
 *     No C++ exception crosses this boundary.
 *   - Complex numbers are interleaved (re, im): complex128 = 2 x double,
 *     complex64 = 2 x float.  State vectors are C-order over the tensor
 *     dimensions (the first axis slowest), as NumPy's reshape(dims).
 *   - Pointers named *_dev are device pointers owned by the caller (e.g.
 *     torch tensors); *_host are host pointers.  `stream` is a cudaStream_t
 *     (NULL = legacy default stream).  Calls on one rpm_system are not
 *     re-entrant: the system owns internal scratch buffers.
 */
#ifndef RPM_B200_H
#define RPM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define RPM_OK 0
#define RPM_E_INVALID 1      /* bad argument; the host raises ValueError      */
#define RPM_E_CUDA 2         /* CUDA runtime failure                          */
#define RPM_E_NOMEM 3        /* device or host allocation failed              */
#define RPM_E_UNSUPPORTED 4  /* size or shape outside the compiled limits     */
#define RPM_E_NOT_HERMITIAN 5 /* a local term fails the Hermiticity check     */
#define RPM_E_NUMERIC 6      /* eigen-solver did not converge / non-finite    */
#define RPM_E_TIMEOUT 7      /* a bounded device wait gave up                 */

#define RPM_MAX_AXES 32      /* tensor axes of one system                     */
#define RPM_MAX_TERM_AXES 4  /* axes one local term may act on                */
#define RPM_MAX_LOCAL_DIM 64 /* local operator side                           */
#define RPM_MAX_KRYLOV 128   /* Krylov dimension                              */

#define RPM_PREC_C64 64      /* complex64 state arithmetic (FP32)             */
#define RPM_PREC_C128 128    /* complex128 state arithmetic (FP64)            */

typedef struct rpm_system rpm_system;

/* One local term: `naxes` distinct tensor axes and a row-major complex128
 * operator of side prod(dims[axes]) -- ENG:28-34 (LocalTerm). */
typedef struct rpm_term {
  int naxes;
  int axes[RPM_MAX_TERM_AXES];
  const double* op;
} rpm_term;

const char* rpm_last_error(void);
int rpm_version(void);
/* Number of CUDA devices visible; 0 when no driver or device. */
int rpm_device_count(int* count);

/* Build a Hamiltonian system.  Replaces ENG:46-93 (MatrixFreeHamiltonian.__init__,
 * _compile_term: axis/shape/Hermiticity checks with `hermitian_tolerance`) and,
 * when nleft > 0, ENG:142-219 (CompiledFullPairHamiltonian.__init__: radical
 * split into left/right CSR blocks and the 4x4 electron-pair operator; the
 * first left and first right axis are the electron pair).  With nleft == 0
 * the generic per-term kernel is used.  host_only != 0 builds the host tables
 * without touching the GPU (for inspection). */
int rpm_system_create(const int* dims, int ndims, const rpm_term* terms, int nterms,
                      const int* left_axes, int nleft, const int* right_axes, int nright,
                      double hermitian_tolerance, int host_only, rpm_system** out);
int rpm_system_destroy(rpm_system* sys);
/* dimension N, split flag, left/right group sizes and CSR nonzero counts. */
int rpm_system_info(const rpm_system* sys, long long* dimension, int* split,
                    int* nl, int* nr, int* nnz_left, int* nnz_right);
/* Copy the host CSR tables of a split system (arrays sized from rpm_system_info):
 * row pointers (n+1), columns, complex128 values, memory offsets of each
 * left/right group index, and the 4x4 pair operator (16 complex128). */
int rpm_system_split_tables(const rpm_system* sys, int* lptr, int* lcol, double* lval,
                            int* rptr, int* rcol, double* rval, long long* offl,
                            long long* offr, double* pair);

/* out = H psi for `batch` vectors spaced `ld` elements apart.
 * Replaces ENG:95-108 (MatrixFreeHamiltonian.matvec), ENG:110-114 (matmat)
 * and ENG:221-253 (CompiledFullPairHamiltonian.matvec/matmat). */
int rpm_hpsi(rpm_system* sys, int precision, const void* psi_dev, void* out_dev,
             int batch, long long ld, void* stream);

/* Select the cube-kernel variant used by every later H psi launch (process
 * wide; 0 = built-in heuristic): inner spin-1/2 digits per radical cube
 * (ni_l, ni_r in {1, 2}), pass-L column tile tr in {1, 2, 4, 8} and pass-R
 * row tile tl in {1, ..., 16}.  A choice that cannot run for a system falls
 * back to the heuristic.  Used by the autotuner; no reference counterpart. */
int rpm_set_cube_tuning(int ni_l, int ni_r, int tr, int tl);

/* Haberkorn recombination with singlet / triplet rates (1/us) on a radical-
 * split system, for the batched propagator: the state evolves under
 * H - (i/2)(kS P_S + kT P_T); the common decay exp(-min(kS, kT) t / 2) is
 * factored out and the remaining -(i/2)|kS - kT| Q (Q = P_S or P_T, an
 * electron-pair operator) is added to the pair operator.  Unequal rates make
 * the system non-Hermitian: the plain Lanczos path refuses it and the batched
 * path runs Arnoldi.  Set the rates before creating a batch from the system.
 * The reference has equal rates only (its yield weight exp(-t/tau)/tau);
 * unequal rates have no reference counterpart. */
int rpm_system_set_recombination(rpm_system* sys, double singlet_rate, double triplet_rate);
int rpm_system_recombination(const rpm_system* sys, double* singlet_rate, double* triplet_rate, int* non_hermitian);

/* *usable = 1 when complex64 H psi of this system runs on the shape-
 * specialised kernels (axes ordered electron A, electron B, left nuclei,
 * right nuclei; each radical's spin-1 nuclei before its spin-1/2 nuclei;
 * a compiled digit pattern), else 0.  Diagnostic; no reference counterpart. */
int rpm_system_fast_hpsi(const rpm_system* sys, int* usable);

/* Reduced density matrices of a bipartition for `nstates` states spaced `ld`
 * elements apart (complex128): rho[s][a][b] = sum_c psi_s[offa[a] + offc[c]]
 * conj(psi_s[offa[b] + offc[c]]), a, b < da, c < dc; offa_dev/offc_dev are
 * device int64 offset tables of the kept and traced axes.  Its eigenvalues
 * are the squared Schmidt coefficients behind CORE:311-328
 * (pure_log_negativity) and CORE:331-334 (reduced_electron_density). */
int rpm_reduced_density(const void* states_dev, long long nstates, long long ld, const long long* offa_dev, int da,
                        const long long* offc_dev, long long dc, void* rho_dev, void* stream);

/* Squared Schmidt coefficients from the eigenvectors of rho_A (u_dev: per
 * state da x da complex128, column i = eigenvector i):
 * sigma2[s][i] = sum_c |sum_a conj(U[a][i]) psi_s[offa[a] + offc[c]]|^2,
 * accurate for small Schmidt values, for CORE:311-328 (pure_log_negativity). */
int rpm_schmidt_norms(const void* states_dev, long long nstates, long long ld, const long long* offa_dev, int da,
                      const long long* offc_dev, long long dc, const void* u_dev, double* sigma2_dev, void* stream);

/* Transition lines of one radical for the factorized ensemble yield
 * (rpm_quantum_needle_reproduction.py:128-170): line (i, j) of the d
 * eigenvalues lam_dev has frequency lam[i] - lam[j] and weight
 * sp[i][j] sq[j][i] * scale (sp, sq: d x d complex128 electron-spin operators
 * in the eigenbasis, row-major) and is deposited with linear interpolation
 * onto grid_dev (2 * half_width + 1 complex128 bins of width delta, centred);
 * a line outside the grid sets *bad_dev = 1. */
int rpm_bin_transition_lines(const double* lam_dev, const void* sp_dev, const void* sq_dev, int d, double scale,
                             double delta, long long half_width, void* grid_dev, int* bad_dev, void* stream);

/* rpm_hpsi without any device allocation.  It has no counterpart in the
 * reference.  It serves callers that may not call cudaMalloc while they run
 * (run loops of frameworks that own all device memory through a pool or
 * arena, where a cudaMalloc would synchronise the device and escape their
 * accounting; fixed-budget embedded runtimes).  It picks the same kernels as
 * rpm_hpsi for the same arguments.  Its only scratch, batch x ld elements of
 * the partial result between the two radical passes, lives in a 4 MiB array
 * compiled into the library, which every GPU that loads the library keeps
 * until process exit; larger batch x ld x element-size requests fail with
 * RPM_E_UNSUPPORTED (systems without a radical split need no scratch).
 * The first call on each device looks up that array's device address (and
 * sets kernel attributes); make it before any stream capture.  The address
 * is cached for the device's primary context: do not call it again on a
 * device after cudaDeviceReset.  All calls
 * share the one array: calls that overlap on the GPU (concurrent streams or
 * threads) race and must be serialised by the caller.  Nothing in the array
 * needs to start at zero; each call overwrites what it reads. */
int rpm_hpsi_noalloc(rpm_system* sys, int precision, const void* psi_dev, void* out_dev,
                     int batch, long long ld, void* stream);

/* FP64 Hermitian Lanczos with two classical Gram-Schmidt passes, replacing
 * ENG:651-688 (AdaptiveLanczosPropagator._basis).  basis_dev holds max_dim
 * complex128 columns of length N (column j at basis_dev + j*N); alpha_dev
 * (max_dim) and beta_dev (max_dim-1) receive the tridiagonal.  On return
 * *actual_host is the basis size (smaller than max_dim after a breakdown
 * with beta <= breakdown_tol) and *norm_host = ||state||.  Raises
 * RPM_E_INVALID for the zero vector (ENG:656-658).  Synchronises `stream`. */
int rpm_lanczos_basis(rpm_system* sys, const void* state_dev, int max_dim,
                      double breakdown_tol, void* basis_dev, double* alpha_dev,
                      double* beta_dev, int* actual_host, double* norm_host, void* stream);

/* Spectral data of the leading d x d block of the tridiagonal (alpha, beta)
 * for each of `ndims` sizes: eigenvalues and eigenvectors by implicit QR with
 * Wilkinson shifts in FP64 (replaces scipy.linalg.eigh_tridiagonal in
 * ENG:569-609).  spectra_dev holds ndims records of RPM_SPECTRUM_DOUBLES. */
#define RPM_SPECTRUM_DOUBLES (RPM_MAX_KRYLOV + RPM_MAX_KRYLOV * RPM_MAX_KRYLOV + 2)
int rpm_tridiag_spectra(const double* alpha_dev, const double* beta_dev, int ndims,
                        const int* dims_host, double* spectra_dev, void* stream);

/* One evaluation request against spectra records: coefficients
 * c = exp(-i T_hi t) e1, the embedded error
 * safety*state_norm*||c - [c_lo; 0]|| (ENG:690-715, 876-888; lo < 0: zero)
 * and, when gram_dev != NULL, state_norm^2 c^H G c (ENG:532-538). */
typedef struct rpm_krylov_req {
  int hi;       /* spectra record of the propagating dimension */
  int lo;       /* spectra record of the embedded dimension, or -1 */
  double time;  /* time offset in us */
} rpm_krylov_req;
int rpm_krylov_eval(const double* spectra_dev, int nreq, const rpm_krylov_req* reqs_host,
                    double safety, double state_norm, const void* gram_dev, int gram_ld,
                    void* coef_dev, int coef_ld, double* err_host, double* value_host,
                    void* stream);

/* G = A^H A for the singlet amplitudes A = (V[0,1,:] - V[1,0,:])/sqrt 2 of the
 * first m complex128 basis columns (ENG:521-529); gram_dev is m x m complex128,
 * Hermitian-symmetrised. */
int rpm_singlet_gram(rpm_system* sys, const void* basis_dev, int m, void* gram_dev, void* stream);

/* out = scale * V[:, :m] c (complex128), and *norm_host = ||out|| when
 * norm_host != NULL (ENG:895, 904, 909).  Synchronises when norm_host != NULL. */
int rpm_combine(rpm_system* sys, const void* basis_dev, int m, const void* coef_dev,
                double scale, void* out_dev, double* norm_host, void* stream);

/* Whole plain propagation of one complex128 state with the singlet
 * population observable, the reference controller's steps
 * (ENG:717-933: minimum dimension first, the maximum basis and its ladder
 * when the minimum misses the step budget, halving on rejection, growth by
 * 1.5 below a tenth of the budget) decided on the device: per Krylov step
 * one fixed launch sequence (basis, singlet Gram, candidate spectra and
 * errors, observation points, new state) and one host read.  The state
 * (length N, device) is propagated in place to the last completed time;
 * values_host / state_errors_host (ntimes) receive the populations and the
 * accumulated state-error estimates at times_host[cursor0 .. points_done).
 * result->status = 1 when the step fell below minimum_step_us (the caller
 * raises the reference's error).  Needs maximum_dimension <= 64 and at most
 * 15 ladder dimensions.  Synchronises `stream`. */
typedef struct rpm_plain_knobs {
  int minimum_dimension, maximum_dimension, dimension_increment, embedded_offset;
  double safety_factor, state_error_budget, initial_step_us, maximum_step_us, minimum_step_us,
      breakdown_tolerance;
} rpm_plain_knobs;
typedef struct rpm_plain_result {
  int accepted_steps, rejected_steps;
  long long matvecs;
  int maximum_krylov_dimension, status;
  int points_done, pad;
  double minimum_step_us, maximum_step_us, accumulated_state_error, maximum_norm_error;
} rpm_plain_result;
int rpm_plain_propagate(rpm_system* sys, const rpm_plain_knobs* knobs, void* state_dev,
                        const double* times_host, int ntimes, int cursor0, double norm_error0,
                        double* values_host, double* state_errors_host, rpm_plain_result* result,
                        void* stream);

/* Singlet population ||(psi[0,1,:] - psi[1,0,:])/sqrt2||^2 of `batch`
 * complex128 vectors of length n (n divisible by 4, electrons first) spaced
 * `ld` apart (ENG:492-497) into values_host.  Synchronises. */
int rpm_singlet_population(const void* psi_dev, long long n, int batch, long long ld,
                           double* values_host, void* stream);

/* ||psi|| (complex128) into *norm_host.  Synchronises. */
int rpm_norm(rpm_system* sys, const void* psi_dev, double* norm_host, void* stream);

/* Composite Simpson yield  sum_k w_k exp(-t_k/tau) P_k / tau  in FP64 with
 * compensated summation, for `batch` population rows of length n spaced
 * `ld` apart (JD:418-420, scipy.integrate.simpson odd/even rules). */
int rpm_simpson_yield(const double* times_dev, const double* pops_dev, int n, int batch,
                      long long ld, double lifetime_us, double* yields_dev, void* stream);

/* out = (1 (x) .. (x) U (x) .. (x) 1) in for a d x d complex128 operator U
 * (row-major, host) acting on tensor axis `axis`, for `batch` complex128
 * vectors spaced `ld` apart.  Replaces poster_reproduction/core.py:285-292
 * (local_unitary_apply), the instantaneous nuclear pulse between segments of
 * rpm_nuclear_spin_rotation_control.py:281-308. */
int rpm_apply_local_operator(const int* dims, int ndims, int axis, const double* op_host,
                             const void* in_dev, void* out_dev, int batch, long long ld, void* stream);

/* ---------------------------------------------------------------------------
 * Batched mixed-precision propagation: many trajectories (state vectors of
 * one or more systems, e.g. field orientations or bath sizes) advanced
 * together.  complex64 Lanczos basis and H psi; FP64 alpha/beta, state,
 * tridiagonal exponential, error control and singlet populations.  The
 * batched counterpart of ENG:717-933 (AdaptiveLanczosPropagator.propagate
 * with SingletPopulationObservable) with a fixed Krylov dimension and the
 * largest step meeting the embedded error budget (no rejected steps).
 * ------------------------------------------------------------------------- */
typedef struct rpm_batch rpm_batch;

typedef struct rpm_batch_config {
  int krylov_dim;              /* fixed Krylov dimension, 2..64              */
  int embedded_offset;         /* error estimate from dims (m, m - offset)   */
  double safety_factor;        /* multiplies the embedded estimate           */
  double state_error_budget;   /* total over [0, T], allotted per dt/T       */
  double initial_step_us;      /* first trial step                           */
  double maximum_step_us;
  double minimum_step_us;      /* below this a trajectory fails (status 3)   */
  double breakdown_relative;   /* beta_j <= rel*(|alpha_j|+beta_{j-1}): stop */
  int use_graph;               /* replay each Krylov step from a CUDA graph   */
  long long max_steps;         /* safety limit on Krylov steps (<=0: 1e7)    */
  int lanczos_kernel;          /* RPM_LANCZOS_PERSISTENT (0): one persistent
                                  launch per Krylov step where the shape has
                                  one; RPM_LANCZOS_PASSES (1): two pass
                                  launches per Lanczos iteration             */
  int wavefront;               /* persistent kernel: vectors that advance
                                  together through the iterations (<=0:
                                  equal groups of at most 16) */
  int reorth_policy;           /* RPM_REORTH_NONE (0): three-term recurrence
                                  only; RPM_REORTH_PERIODIC (1): after every
                                  `reorth_period` iterations the next Lanczos
                                  vector is reorthogonalised against the whole
                                  basis (two classical Gram-Schmidt passes,
                                  FP64 sums over the complex64 basis)        */
  int reorth_period;           /* iterations between reorthogonalisations    */
  int persistent_ctas;         /* CTAs of a persistent launch (<=0: one per
                                  SM); fewer leave SMs free for the other
                                  kernels of a batch running concurrently on
                                  another stream                             */
} rpm_batch_config;

#define RPM_LANCZOS_PERSISTENT 0
#define RPM_LANCZOS_PASSES 1
#define RPM_REORTH_NONE 0
#define RPM_REORTH_PERIODIC 1

typedef struct rpm_batch_stats {
  int accepted_steps;
  int rejected_steps;
  long long matvecs;
  int maximum_krylov_dimension;
  int status;                  /* 0 ok, 1 zero/non-finite input, 2 eigen-solver,
                                  3 step underflow, 4 non-finite state        */
  double minimum_step_us;
  double maximum_step_us;
  double accumulated_state_error;
  double maximum_norm_error;
} rpm_batch_stats;

/* Prepare a batch over `nsys` radical-split systems (each must have the cube
 * form: terms on {e}, {n_k} or {e, n_k} per radical). */
int rpm_batch_create(rpm_system* const* systems, int nsys, const rpm_batch_config* cfg, rpm_batch** out);
/* Per-trajectory stride (elements) of the state buffer passed to propagate. */
int rpm_batch_leading_dimension(const rpm_batch* batch, long long* ld);
/* Propagate `ntraj` trajectories; trajectory b uses system sys_of_host[b] and
 * starts from psi_dev + b*ld (complex128, overwritten with the final state).
 * values_dev / state_errors_dev (ntraj x ntimes, FP64, device) receive the
 * singlet population and the accumulated state-error estimate at each time;
 * stats_host (ntraj entries, host) receives each trajectory's statistics and
 * status. */
int rpm_batch_propagate(rpm_batch* batch, int ntraj, const int* sys_of_host, void* psi_dev,
                        const double* times_host, int ntimes, double* values_dev,
                        double* state_errors_dev, rpm_batch_stats* stats_host, void* stream);
/* Measurement counters since creation or the last reset: kernels launched,
 * Krylov-step replays, and the mean duration (ms) of one batched Lanczos
 * iteration (H psi with the fused recurrence, all trajectories) sampled inside
 * the graph while no trajectory had finished: one pass pair, or the persistent
 * launches of a step divided by its iterations. */
int rpm_batch_counters(rpm_batch* batch, int reset, long long* kernel_launches, long long* step_replays,
                       double* hpsi_ms_mean, long long* hpsi_samples);
/* How the last recorded Krylov step ran its Lanczos iterations (replaces the
 * per-vector loop of ENG:651-688): 0 one persistent launch per shape group
 * (per segment between reorthogonalisations), 1 shape-specialised pass pairs
 * per iteration, 2 general cube kernels (or Arnoldi). */
int rpm_batch_lanczos_kind(const rpm_batch* batch, int* kind);
/* Factorized exact oracle (rpm_quantum_needle_reproduction.py:127-240):
 * batched Hermitian eigen-decomposition of n x n complex matrices (replaces
 * the per-radical numpy.linalg.eigh of diagonalize_radical, :127): a_dev
 * holds `batch` row-major matrices (overwritten), w_dev receives the
 * eigenvalues in ascending order (batch x n), v_dev the eigenvectors as
 * columns (v[i * n + j] = component i of eigenvector j); Householder
 * tridiagonalisation, implicit tridiagonal QR, back-transformation, all FP64.
 * work_dev: rpm_he_eigh_workspace bytes.  Synchronises the stream. */
int rpm_he_eigh_workspace(int n, int batch, long long* bytes);
int rpm_he_eigh(int n, int batch, void* a_dev, double* w_dev, void* v_dev, void* work_dev, cudaStream_t stream);
/* C = A^H B for `batch` square complex128 matrices (row-major): the
 * eigenbasis spin operators of diagonalize_radical (:127-170). */
int rpm_zgemm_hn(int n, int batch, const void* a_dev, const void* b_dev, void* c_dev, cudaStream_t stream);
/* Radix-2 complex128 FFT of `batch` rows of power-of-two length n in place
 * (scratch: n x batch complex); inverse = 1 gives the unscaled inverse
 * transform.  With rpm_spectrum_mac (acc += x * y element-wise) it forms the
 * convolution of binned transition spectra (convolved_correlation_spectrum,
 * :175-201). */
int rpm_fft_pow2(int n, int batch, void* data_dev, void* scratch_dev, int inverse, cudaStream_t stream);
int rpm_spectrum_mac(long long count, void* acc_dev, const void* x_dev, const void* y_dev, cudaStream_t stream);
/* Kernel of the batched singlet Gram V^H P_S V (replaces the per-basis
 * projection of ENG:521-529): 0 the CUDA-core kernel, 1 (default) the
 * tensor-core kernel (tcgen05, TF32 split into high and low parts, FP32 sums
 * over 32 rows in tensor memory, FP64 across them) wherever the batch allows
 * it (every state dimension a multiple of 8, Krylov dimension <= 63).  Read
 * when a batch's step is set up. */
int rpm_set_gram_kernel(int kernel);
/* Consumer warps per CTA of the persistent Lanczos kernel, 8, 9 or 10
 * (default 8); a tuning knob for measurements, no counterpart in the
 * reference. */
int rpm_set_persistent_warps(int consumer_warps);
/* Per-system Krylov dimensions (caps[k] for the batch's system k, 0: the
 * batch's krylov_dim; otherwise 2 <= cap <= krylov_dim): a trajectory's
 * basis ends after cap Lanczos / Arnoldi iterations, so systems of uneven
 * size in one batch each run at their own dimension.  nsys = 0 clears them.
 * No counterpart in the reference, whose dimension is per propagator. */
int rpm_batch_set_krylov_caps(rpm_batch* batch, const int* caps, int nsys);
/* Replace the configured state-error budget for later propagate calls (the
 * knob ENG:620-649 exposes as a mutable attribute). */
int rpm_batch_set_budget(rpm_batch* batch, double state_error_budget);
int rpm_batch_destroy(rpm_batch* batch);

/* -------------------------------------------------------------------------
 * Adjoint sweep for gradients of the singlet yield.  No reference
 * counterpart: the reference's only derivatives are finite differences of
 * yields over angle grids (np.gradient over theta,
 * rpm_quantum_needle_reproduction.py and rpm_three_nitrogen_quadrupole.py:153);
 * this replaces central differences through ENG:717-933.
 * The yield is Phi = sum_k w_k <psi_k|P_S|psi_k> on a uniform grid
 * t_k = t_0 + k dt, psi_{k+1} = exp(-i H_k dt) psi_k (equal recombination
 * rates, decay folded into w_k).  The adjoint lambda_k = U_k^dag lambda_{k+1}
 * + w_k P_S psi_k is marched backwards and, per interval,
 *   M_ab += int <lambda| (|a><b| (x) 1) |psi> dt   (a, b = 2 eA + eB),
 *   S_r  += int <lambda| D_r |psi> dt            (derivative systems D_r),
 *   W    += int <lambda| H |psi> dt              (FP64, optional),
 * so that dPhi/dp = 2 Im( sum_ab E_ab M_ab + sum_r c_r S_r + c_H W ) for
 * dH/dp = E (x) 1 + sum_r c_r D_r + c_H H.  The first two state axes must be
 * the electrons; systems must be Hermitian radical-split cube-form systems.
 * ------------------------------------------------------------------------- */
typedef struct rpm_adjoint rpm_adjoint;

/* Workspace for ntraj trajectories of dimension n (states spaced ld
 * elements, ld even); `degree` Taylor terms per interval (1..24),
 * `nodes` Gauss-Legendre nodes (1..4) and the basis precision
 * (RPM_PREC_C64 or RPM_PREC_C128; states stay FP64). */
int rpm_adjoint_create(int ntraj, long long n, long long ld, int degree, int nodes, int precision,
                       rpm_adjoint** out);
int rpm_adjoint_destroy(rpm_adjoint* adj);
/* lambda += weight * P_S psi for every trajectory (complex128 device buffers). */
int rpm_adjoint_source(rpm_adjoint* adj, const void* psi_dev, void* lambda_dev, double weight, void* stream);
/* Walk intervals j = nintervals-1 .. 0 backwards.  On entry lambda_dev /
 * psi_dev (ntraj x ld complex128) hold lambda and psi at the end of interval
 * nintervals-1 (lambda including its source there); on return they hold them
 * at the start of interval 0, lambda including source_weights[0].  Interval
 * j evolves under systems[segment_of_interval[j]] (host arrays).
 * density_dev: ntraj x nseg x 16 complex (FP64, accumulated);
 * derivative_dev: ntraj x nseg x nder complex (accumulated), with
 * derivative_systems[s * nder + r] (NULL: none) applied in segment s;
 * energy_dev (optional): ntraj x nseg complex, accumulated W.
 * *max_tail (optional; synchronises the stream) receives the largest
 * ||last Taylor term|| / ||psi|| over all intervals and trajectories. */
int rpm_adjoint_sweep(rpm_adjoint* adj, rpm_system* const* systems, int nseg,
                      rpm_system* const* derivative_systems, int nder, const int* segment_of_interval,
                      const double* source_weights, double dt, int nintervals, void* lambda_dev,
                      void* psi_dev, double* density_dev, double* derivative_dev, double* energy_dev,
                      double* max_tail, void* stream);
/* Forward Taylor stepping with the same basis: psi_dev (ntraj x ld
 * complex128) advances over `nintervals` intervals of length dt (interval j
 * under systems[segment_of_interval[j]]); populations_dev[b * pop_ld + j]
 * receives the singlet population at the end of interval j (ENG:492-497).
 * A fixed schedule, so yields are smooth in the Hamiltonian's parameters
 * (finite differences through it need no frozen step controller). */
int rpm_adjoint_forward(rpm_adjoint* adj, rpm_system* const* systems, int nseg, const int* segment_of_interval,
                        double dt, int nintervals, void* psi_dev, double* populations_dev, long long pop_ld,
                        double* max_tail, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RPM_B200_H */
