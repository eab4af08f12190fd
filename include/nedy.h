/*
 * nedy.h -- C ABI of the B200-native GF2 Kadanoff-Baym hot path.
 *
 * Drop-in boundary for the per-timestep work of tblommel/NEdyson: the
 * second-Born self-energy (density-fitted, spin-unrestricted and full-U), the
 * Hartree-Fock mean field, the Dyson time step with its Gregory-weighted history
 * integrals and Legendre mixed-component convolutions, the polynomial predictor,
 * the bootstrap and the correlation energy.  Plain C: opaque handles, raw
 * pointers and sizes; every function returns an nedy_status code and never
 * throws or exits across the boundary.
 *
 * Storage: Green's functions keep the reference's packed layout (reference
 * src/greens.cpp:34-195), with nao x nao row-major complex128 blocks:
 *   NEDY_LES  block (i,j), i <= j, at j*(j+1)/2 + i      (column G^<(.,T) contiguous)
 *   NEDY_RET  block (i,j), j <= i, at i*(i+1)/2 + j      (row G^R(T,.) contiguous)
 *   NEDY_TV   block (t,m) at t*(ntau+1) + m
 *   NEDY_MAT  block m
 * Block indices are 64-bit.  The imaginary-time grid is the ntau+1
 * Legendre-Gauss-Lobatto nodes tau_m = beta (x_m + 1) / 2 (nedy_collocation_nodes).
 *
 * Threading: a context owns one CUDA stream; calls on one context must come from
 * one host thread at a time (the reference objects are not re-entrant either,
 * src/dyson.h:26-37).
 */
#ifndef NEDY_H
#define NEDY_H

#ifdef __cplusplus
extern "C" {
#endif

#define NEDY_ABI_VERSION 1

enum nedy_status {
  NEDY_OK = 0,
  NEDY_ERR_ARG = 1,      /* bad argument or size (the reference asserts) */
  NEDY_ERR_CUDA = 2,     /* CUDA runtime error */
  NEDY_ERR_NOCONV = 3,   /* iteration did not reach its tolerance */
  NEDY_ERR_TIMEOUT = 4,  /* a bounded device wait gave up */
  NEDY_ERR_OOM = 5,      /* device allocation failed */
  NEDY_ERR_STATE = 6,    /* call out of order (e.g. tensor not set) */
  NEDY_ERR_SINGULAR = 7  /* zero pivot in a Dyson solve */
};

enum nedy_component { NEDY_LES = 0, NEDY_RET = 1, NEDY_TV = 2, NEDY_MAT = 3 };
/* Arithmetic of the self-energy contractions (nedy_ctx_set_precision).
 * FP64: every product in FP64 on the DMMA tensor cores (the reference's arithmetic).
 * SPLIT_BF16X3: the density-fitted self-energy contractions as BF16 piece products on
 *   tcgen05: each operand is split into three BF16 pieces, the six piece products with
 *   combined weight >= 2^-16 are accumulated in FP32.
 * SPLIT_BF16X2: the same with two pieces per operand (hi, lo) and the three products
 *   hi*hi + hi*lo + lo*hi (about 2^-17 relative per product instead of FP32 rounding):
 *   half the tensor work of SPLIT_BF16X3.
 * In every mode the Dyson solves, the mean field, the density matrix and the residuals
 * stay FP64; the full-U self-energy is always FP64. */
enum nedy_precision { NEDY_PREC_FP64 = 0, NEDY_PREC_SPLIT_BF16X3 = 1, NEDY_PREC_SPLIT_BF16X2 = 2 };

typedef struct nedy_ctx nedy_ctx;
typedef struct nedy_gf nedy_gf;
typedef struct nedy_buf nedy_buf;

/* Sizes of one simulation: dyson(nt, ntau, nao, k) (reference src/dyson.cpp:25-43),
 * beta and dt as passed to dyson_step (src/dyson.h:86). */
typedef struct {
  int nt, ntau, nao, k;
  double beta, dt;
  int device;                 /* CUDA device ordinal */
  long long workspace_bytes;  /* self-energy chunk budget; 0 = default (8 GiB) */
} nedy_config;

int nedy_abi_version(void);
const char *nedy_status_string(int status);
/* Message of the last failing call on this host thread. */
const char *nedy_last_error(void);

int nedy_ctx_create(const nedy_config *cfg, nedy_ctx **out);
int nedy_ctx_destroy(nedy_ctx *ctx);
int nedy_ctx_synchronize(nedy_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), e.g. to record events around calls. */
int nedy_ctx_stream(nedy_ctx *ctx, void **stream);
/* Per-phase device timing of nedy_decomp_tstp / nedy_decomp_spin_tstp (CUDA events):
 * ms4 = accumulated milliseconds of predictor, mean field, self-energy, Dyson step. */
int nedy_ctx_set_timing(nedy_ctx *ctx, int on);
/* Self-energy arithmetic for this context (nedy_precision); FP64 by default.  The
 * reference computes in FP64 only; the split modes are this engine's addition. */
int nedy_ctx_set_precision(nedy_ctx *ctx, int mode);
/* Accounting of the split-precision tensor-core GEMMs of this process: returns their
 * algorithmic BF16 tensor-pipe FLOPs (2 M N K per piece product) and summed device time
 * (CUDA events around each launch) since the previous call, then switches the
 * accounting on (on != 0) or off. */
int nedy_split_stats(int on, double *pipe_flops, double *ms);
/* Autotuner of the split GEMM tile shapes (on by default): each problem class (operand
 * kinds, output kind, M, N, padded K) times its candidate shapes (64/128/256-wide tiles,
 * 2-4 pipeline stages) on its first launches and keeps the fastest; every candidate
 * computes the same result.  The report lists classes, candidate times and choices. */
int nedy_split_autotune(int on);
int nedy_split_tune_report(char *buf, int len);
/* *classes = problem classes still timing their candidates (0: every class has chosen;
 * from then on no launch runs a trial shape).  No reference counterpart. */
int nedy_split_tune_pending(int *classes);
/* Work partition of the density-fitted self-energy for a workspace budget (bytes):
 * *chunk slices per chunk and *sub exchange units per launch, as the solver chooses them
 * (planning helper, no reference counterpart; host arithmetic, no device access).
 * precision: nedy_precision; real_symmetric: every B^Q real symmetric; sms: streaming
 * multiprocessors of the device (148 on a B200). */
int nedy_sigma_chunk_plan(int nao, int naux, long long budget, int precision, int real_symmetric, int sms, int *chunk,
                          int *sub);
/* Check of one split GEMM kernel instance (test hook, no reference counterpart):
 * C (nb x M x N) = 0.75 * op(A) op(B)^T (+ C when accumulate is 1; accumulate 2: the product
 * replaces a C filled with values that must not be read) on seeded uniform operands
 * (complex when *_cplx, conjugated when conj_*), split into npieces BF16 pieces, with the
 * given instance: tile_n 64/128/256 output columns per CTA, stages, k_block 0 for the
 * per-product kernel or 32/64 for the one-load kernel, kdiv the K-split divisor, persistent
 * 1 the persistent one-load kernel (one CTA per SM over a tile list, two TMEM
 * accumulators; tile_n 64 or 128, out_pieces only), persistent 2 the CTA-pair one-load kernel
 * (clusters of two CTAs, 256-row tiles by tcgen05.mma.cta_group::2; complex x complex),
 * persistent 3 the persistent CTA-pair kernel (tile_n 128, out_pieces only).  *rel_err = max |C - C_fp64| / max |C_fp64|; NEDY_ERR_ARG for
 * an instance that does not exist or does not fit in shared memory. */
int nedy_split_gemm_check(int device, int M, int N, int K, int nb, int a_cplx, int b_cplx, int conj_a, int conj_b,
                          int npieces, int out_pieces, int accumulate, int tile_n, int stages, int k_block, int kdiv,
                          int persistent, unsigned long long seed, double *rel_err);
int nedy_ctx_phase_times(const nedy_ctx *ctx, double *ms4);
/* Test hook of the bounded device waits (no reference counterpart): presets the error
 * word of the context's split-precision GEMMs as a wait that gave up would set it
 * (code != 0).  The CTAs of the next split launches then skip their work and the call
 * that launched them returns NEDY_ERR_TIMEOUT; reporting clears the word, so the call
 * after that runs normally.  Lets a test drive the timeout path without a device fault. */
int nedy_ctx_inject_split_error(nedy_ctx *ctx, int code);
/* Dense solve X = A^-1 B of nb independent complex systems, A n x n and B n x nrhs each,
 * row-major, interleaved (re, im) doubles in HOST memory; B is overwritten by X, A is left as
 * it was.  The engine's replacement for the partial-pivot LU solves of the Dyson step and the
 * bootstrap (Eigen PartialPivLU::solve at src/dyson_step.h:65, :163, :252 and
 * src/dyson_boot.h:61, :170): Gauss-Jordan with partial pivoting on the context's stream, the
 * same routine those steps use.  NEDY_ERR_SINGULAR on a zero pivot. */
int nedy_dense_solve(nedy_ctx *ctx, int n, int nrhs, int nb, const double *A, double *B);
/* Number of engine kernel launches issued by this process so far. */
unsigned long long nedy_launch_count(void);
/* Collocation nodes x_m in [-1,1] and weights (ntau+1 values each). */
int nedy_collocation_nodes(const nedy_ctx *ctx, double *x, double *w);

/* --- Green's functions: green_func(nt, ntau, size1, sig) (src/greens.cpp:34-55) --- */
int nedy_gf_create(nedy_ctx *ctx, int nt, int ntau, int nao, int sig, nedy_gf **out);
/* The same with only the last `window` time steps of G^R (rows) and G^< (columns) on the
 * device (no reference counterpart: the reference holds every triangle, src/greens.cpp:44-45).
 * A time step of G reads nothing older (its own row, the k+1 rows of the extrapolation,
 * the learned predictor's history), while Sigma must keep its whole triangles for the Dyson
 * integrals; so a windowed G and a full Sigma halve the history the device holds, and the
 * caller streams every finished row out (nedy_gf_download of one row or column, while it is
 * within the window).  window >= NEDY_GF_MIN_WINDOW; G^tv and G^M stay whole.  Block ranges
 * of the lesser / retarded components must then lie in one row (column). */
#define NEDY_GF_MIN_WINDOW 12
int nedy_gf_create_windowed(nedy_ctx *ctx, int nt, int ntau, int nao, int sig, int window, nedy_gf **out);
/* The same as nedy_gf_create with the lesser and retarded triangles in pinned host memory
 * mapped into the device's address space (no reference counterpart: the reference holds
 * every triangle in host memory, src/greens.cpp:44-45, and runs on the host).  For Sigma of
 * runs whose two-time history exceeds the device: the kernels read and write it in place
 * over the host link, so a Dyson step, which reads both of Sigma's triangles whole, then
 * moves them across that link every step.  G^tv and G^M stay on the device; transfers and
 * every entry point take it like any green_func. */
int nedy_gf_create_host_history(nedy_ctx *ctx, int nt, int ntau, int nao, int sig, nedy_gf **out);
/* *host = 1 when the lesser and retarded triangles of g live in mapped host memory */
int nedy_gf_host_history(const nedy_gf *g, int *host);
int nedy_gf_window(const nedy_gf *g, int *window);
/* Waits for the device; may be called before or after nedy_ctx_destroy of its context
 * (every other call on the handle needs a live context). */
int nedy_gf_destroy(nedy_gf *g);
/* Copy nblocks nao x nao blocks starting at block first_block of a component. */
int nedy_gf_upload(nedy_gf *g, int component, long long first_block, long long nblocks, const void *host);
int nedy_gf_download(const nedy_gf *g, int component, long long first_block, long long nblocks, void *host);
int nedy_gf_device_pointer(const nedy_gf *g, int component, void **dev);
/* green_func::set_tstp_zero (src/greens.h:76-86) */
int nedy_gf_set_tstp_zero(nedy_gf *g, int tstp);

/* --- Device buffers (mean-field hmf, density matrices, ...) --- */
int nedy_buf_create(nedy_ctx *ctx, long long bytes, nedy_buf **out);
/* Waits for the device; may be called before or after nedy_ctx_destroy. */
int nedy_buf_destroy(nedy_buf *b);
int nedy_buf_upload(nedy_buf *b, long long offset, long long bytes, const void *host);
int nedy_buf_download(const nedy_buf *b, long long offset, long long bytes, void *host);
int nedy_buf_device_pointer(const nedy_buf *b, void **dev);

/* --- Interaction tensors --- */
/* Vija: nao x nao x naux row-major real (B^Q_ij).  Replaces the tensors handed to
 * molGF2SolverDecomp(Vija, Viaj) (src/mol2bSolver.h:103); Viaj is derived. */
int nedy_set_df_tensor(nedy_ctx *ctx, const double *Vija, int nao, int naux);
/* U, Uexch: nao^4 row-major real; Uexch(j,l,n,q) = 2 U(j,n,l,q) - U(j,l,n,q).
 * Replaces molGF2Solver(U, Uexch) (src/mol2bSolver.h:194). */
int nedy_set_full_tensor(nedy_ctx *ctx, const double *U, const double *Uexch, int nao);

/* --- Self-energy of time row tstp (Sigma is zeroed first, like the reference) --- */
/* molGF2SolverDecomp::solve(int, GREEN&, GREEN&)          src/mol2bSolver.h:125 */
int nedy_gf2_decomp_solve(nedy_ctx *ctx, int tstp, nedy_gf *Sigma, const nedy_gf *G);
/* molGF2SolverSpinDecomp::solve(int, vector<GREEN>&, ...) src/mol2bSolver.h:67 */
int nedy_gf2_spin_decomp_solve(nedy_ctx *ctx, int tstp, nedy_gf *Sigma_up, nedy_gf *Sigma_dn,
                               const nedy_gf *G_up, const nedy_gf *G_dn);
/* molGF2Solver::solve(int, GREEN&, GREEN&)                 src/mol2bSolver.h:204 */
int nedy_gf2_full_solve(nedy_ctx *ctx, int tstp, nedy_gf *Sigma, const nedy_gf *G);

/* --- Mean field; hmf buffers hold (nt+1) x nao x nao complex blocks --- */
/* rho = i*sig*G^<(t,t) written at rho_offset (bytes) of a buffer; green_func::get_dm (src/greens.h:68-74) */
int nedy_get_dm(nedy_ctx *ctx, const nedy_gf *G, int tstp, nedy_buf *rho, long long rho_offset);
/* molHFSolverDecomp::solve_HF(tstp, hmf, rho)              src/molHFSolver.h:64 */
int nedy_hf_decomp(nedy_ctx *ctx, int tstp, nedy_buf *hmf, const nedy_buf *rho);
/* molHFSolverSpinDecomp::solve_HF; rho2 holds the two spin densities back to back  src/molHFSolver.h:125 */
int nedy_hf_spin_decomp(nedy_ctx *ctx, int tstp, nedy_buf *hmf_up, nedy_buf *hmf_dn, const nedy_buf *rho2);
/* molHFSolver::solve_HF                                    src/molHFSolver.h:31 */
int nedy_hf_full(nedy_ctx *ctx, int tstp, nedy_buf *hmf, const nedy_buf *rho);
/* Same result as nedy_hf_decomp, but the call allocates no device memory.  No
 * counterpart in the reference.  For callers that cannot call cudaMalloc once the
 * simulation runs: a host program whose own pool allocator has reserved the free
 * device memory, or a driver loop that must not stall the device, which the
 * implicit synchronisation of cudaMalloc/cudaFree would do.  (nedy_hf_decomp may
 * grow or merge the context's workspace, which allocates.)  Its intermediates
 * live in one static device array of NEDY_NOALLOC_SCRATCH_BYTES, held by every
 * GPU that loads the library until the process exits.  A call needs
 * 16*naux bytes (rounded up to 256) + 16*nao*nao*naux bytes of it (nao=64,
 * naux=256 fits); larger sizes are rejected with NEDY_ERR_ARG.
 * The first call on a device looks up that array's device address (set-up);
 * make that first call before any stream capture starts.  All calls on a device
 * share the array and find the previous call's values in it (nothing there is
 * read before it is written): calls that overlap on the GPU (other host threads,
 * other contexts on the same device) race.  Each call synchronises the context's
 * stream and returns after the update has finished, like nedy_hf_decomp. */
#define NEDY_NOALLOC_SCRATCH_BYTES (24LL << 20)
int nedy_hf_decomp_noalloc(nedy_ctx *ctx, int tstp, nedy_buf *hmf, const nedy_buf *rho);

/* --- Dyson equation --- */
/* dyson::Extrapolate(int, GREEN&)                          src/dyson.h:114 */
int nedy_extrapolate(nedy_ctx *ctx, int tstp, nedy_gf *G);
/* dyson::dyson_step(int, GREEN&, const GREEN&, const cplx*, mu, beta, dt)  src/dyson.h:86.
 * err3 (optional) receives the ret, tv and les residual norms. */
int nedy_dyson_step(nedy_ctx *ctx, int tstp, nedy_gf *G, const nedy_gf *Sigma, const nedy_buf *hmf, double mu,
                    double *err3);
/* dyson::dyson_start(GREEN&, const GREEN&, const cplx*, mu, beta, dt)   src/dyson.h:58 */
int nedy_dyson_start(nedy_ctx *ctx, nedy_gf *G, const nedy_gf *Sigma, const nedy_buf *hmf, double mu, double *err);
/* dyson::energy_conv(int, const GREEN&, const GREEN&, beta, dt)         src/dyson.h:137 */
int nedy_energy_conv(nedy_ctx *ctx, int tstp, const nedy_gf *Sigma, const nedy_gf *G, double *energy);

/* --- One whole time step of the restricted density-fitted simulation
 * (DecompSimulation::do_tstp, src/molNEsim_decomp_impl.h:85-104): predictor,
 * then corr_steps x [rho, hmf(tstp) = h_t + HF(rho), Sigma, dyson_step].
 * h_t: nao x nao complex one-body Hamiltonian at tstp (h0 plus the drive).
 * err: residual of the last dyson_step (sum of the three components). */
int nedy_decomp_tstp(nedy_ctx *ctx, int tstp, nedy_gf *G, nedy_gf *Sigma, nedy_buf *hmf, const nedy_buf *h_t,
                     double mu, int corr_steps, double *err);
/* One whole time step of the full-U simulation (Simulation::do_tstp,
 * src/molNEsim_impl.h:89-124): predictor, then corr_steps x [rho, hmf(tstp) = h_t +
 * HF(rho) with U (molHFSolver::solve_HF), the GF2 self-energy row with U and Uexch
 * (molGF2Solver::solve), dyson_step].  nedy_set_full_tensor must have been called.
 * h_t: nao x nao complex one-body Hamiltonian at tstp (h0 plus the drive, which the
 * reference adds through Ed_contractions, :56-61).  err: residual of the last dyson_step. */
int nedy_full_tstp(nedy_ctx *ctx, int tstp, nedy_gf *G, nedy_gf *Sigma, nedy_buf *hmf, const nedy_buf *h_t,
                   double mu, int corr_steps, double *err);
/* The same step with a residual exit (the reference always runs CorrSteps iterations;
 * the exit is the engine's addition).  After iteration k the change d_k = max |G_k - G_{k-1}|
 * over the new row (les column, ret row, tv row) is measured; the iterations stop once
 * d_k times the corrector's contraction factor is <= tol, i.e. once the row is estimated
 * to be within tol of the converged one, or after max_corr iterations.  The contraction
 * is measured (4 x the ratio of successive changes) on steps that run two or more
 * iterations: the first step on a context, and every 8th step after, run at least two.
 * iters: iterations run; err_hist (optional, max_corr entries): d_k per iteration. */
int nedy_decomp_tstp_tol(nedy_ctx *ctx, int tstp, nedy_gf *G, nedy_gf *Sigma, nedy_buf *hmf, const nedy_buf *h_t,
                         double mu, int max_corr, double tol, int *iters, double *err_hist);
/* --- Learned next-step predictor (no counterpart in the reference, whose predictor is the
 * polynomial extrapolation dyson::Extrapolate, src/dyson.cpp:47-117).  A 2-layer MLP of
 * width 256 (BF16 operands, FP32 accumulation, FP32 master weights, Adam) corrects the
 * k = 5 extrapolation of every element of the new row that has 9 history points and
 * oscillates smoothly, from the three previous sixth differences of its time series.
 * It is trained on the GPU on rows the engine converged (collect) and used by
 * nedy_decomp_tstp_tol: after the first corrector iteration the step compares the
 * learned and the polynomial prediction with the corrected row; once 8 steps are judged,
 * fewer than 3 wins among the last 8 switch the context back to the polynomial predictor. */
typedef struct nedy_predictor nedy_predictor;
int nedy_predictor_create(nedy_ctx *ctx, long long capacity, unsigned long long seed, nedy_predictor **out);
int nedy_predictor_destroy(nedy_predictor *p);
/* training samples from the converged row tstp of G (every stride-th eligible element) */
int nedy_predictor_collect(nedy_predictor *p, const nedy_gf *G, int tstp, int stride);
int nedy_predictor_samples(nedy_predictor *p, long long *n);
int nedy_predictor_clear(nedy_predictor *p);
/* iters Adam steps on random minibatches of the collected samples; loss: last minibatch */
int nedy_predictor_train(nedy_predictor *p, int iters, int batch, double lr, double *loss);
/* number of parameters; copy them out (get != 0) or in (FP32: W1 256x12, b1, W2 256x256, b2, W3 2x256, b3) */
long long nedy_predictor_nparams(void);
int nedy_predictor_params(nedy_predictor *p, float *host, int get);
/* forward pass on n host feature rows (n x 12) -> y (n x 2); loss 0.5 sum|y-t|^2 / n and
 * its gradient (nparams floats) on host rows, for checks against a CPU restatement */
int nedy_predictor_forward(nedy_predictor *p, const float *x, int n, float *y);
/* the same network through the inference kernel the steps use (tcgen05 tensor cores,
 * 128 rows per CTA, W1/W2 resident in shared memory), on n host rows -> y (n x 2) */
int nedy_predictor_infer(nedy_predictor *p, const float *x, int n, float *y);
int nedy_predictor_loss_grad(nedy_predictor *p, const float *x, const float *t, int n, double *loss, float *grad);
/* the prediction of row tstp alone: dyson::Extrapolate, plus the learned correction of
 * the context's predictor when learned != 0 */
int nedy_predict(nedy_ctx *ctx, int tstp, nedy_gf *G, int learned);
/* use p in nedy_decomp_tstp_tol / nedy_decomp_spin_tstp_tol of ctx (NULL: polynomial
 * extrapolation only) */
int nedy_ctx_set_predictor(nedy_ctx *ctx, nedy_predictor *p);
/* active: learned predictor in use; judged / better: steps judged and won by it;
 * last2: the last judged max changes from the learned and from the polynomial prediction */
int nedy_ctx_predictor_stats(const nedy_ctx *ctx, int *active, long long *judged, long long *better, double *last2);

/* DecompSpinSimulation::do_tstp (src/molNEsim_decomp_spin_impl.h:86-108) with the residual
 * exit of nedy_decomp_tstp_tol in place of the fixed CorrSteps loop: the change d_k is the
 * max over both spins' new rows; h_t_up / h_t_dn are the one-body Hamiltonians of each spin
 * at tstp (the reference uses one hcore for both), mu_up / mu_dn the chemical potentials.
 * Both G rows get the learned correction when a predictor is set (use in context). */
int nedy_decomp_spin_tstp_tol(nedy_ctx *ctx, int tstp, nedy_gf *G_up, nedy_gf *G_dn, nedy_gf *S_up, nedy_gf *S_dn,
                              nedy_buf *hmf_up, nedy_buf *hmf_dn, const nedy_buf *h_t_up, const nedy_buf *h_t_dn,
                              double mu_up, double mu_dn, int max_corr, double tol, int *iters, double *err_hist);
/* Spin-unrestricted step (DecompSpinSimulation::do_tstp, src/molNEsim_decomp_spin_impl.h:97-122).
 * In this and in nedy_decomp_spin_tstp_tol the two spins' Dyson steps run side by side: the
 * second on a stream of the context's own (created on first use, with its own workspace)
 * from a short-lived helper thread; the call returns once both are done, and the context's
 * stream is ordered after both. */
int nedy_decomp_spin_tstp(nedy_ctx *ctx, int tstp, nedy_gf *G_up, nedy_gf *G_dn, nedy_gf *S_up, nedy_gf *S_dn,
                          nedy_buf *hmf_up, nedy_buf *hmf_dn, const nedy_buf *h_t_up, const nedy_buf *h_t_dn,
                          double mu_up, double mu_dn, int corr_steps, double *err);

/* --- Equilibrium (Matsubara) GF2 state on the collocation grid: the state the reference
 * takes from the external gfmol solver (src/molNEsim_decomp_impl.h:23-33, L_to_Tau :146-167).
 * Restricted (nspin = 1) or unrestricted (nspin = 2, the mean field and self-energy of
 * both spins as in molHFSolverSpinDecomp / molGF2SolverSpinDecomp) density-fitted GF2:
 * iterates Sigma^M[G^M] (the GF2 contraction of the t = 0 mixed row, G^tv(0,tau) =
 * -i G^M(beta - tau)), F = h0 + HF(-G^M(beta)) and the Dyson equation
 * G = G_ref + G_ref * (F - F_ref + Sigma^M) * G (Matsubara convolutions evaluated exactly
 * on the degree-ntau interpolants), with G <- G + mixing (G_new - G), until
 * max |G_new - G| <= tol or max_iter iterations.
 * On entry G[s]->mat holds G_ref, the free G^M of the Fock matrix F_ref[s] at the chemical
 * potential of the run (which stays fixed); on return G[s]->mat holds the GF2 equilibrium,
 * Sigma[s]->mat its self-energy and F_out[s] its mean field (nao x nao complex buffers).
 * nedy_set_df_tensor must have been called; the context's ntau and beta are the grid.
 * iters / diff (optional): iterations run and the last change. */
int nedy_matsubara_gf2(nedy_ctx *ctx, int nspin, nedy_gf *const *G, nedy_gf *const *Sigma, const nedy_buf *const *h0,
                       const nedy_buf *const *F_ref, nedy_buf *const *F_out, double mixing, int max_iter, double tol,
                       int *iters, double *diff);

/* --- Batched independent simulations (many molecules or fields of uneven nao; no
 * counterpart in the reference, which steps one DecompSimulation at a time,
 * src/molNEsim_decomp_impl.h:85-104).  Each instance keeps its own context (stream,
 * workspace), G, Sigma, mean-field buffer and the one-body Hamiltonians h(t) of all steps
 * (h_all: (nt+1) x nao x nao complex; hmf the same size).  nedy_batch_tstp runs the step
 * of every instance: a pool of native worker threads (workers <= 0: up to 16) takes the
 * instances largest nao first and issues each step on its instance's stream, so the
 * instances' kernels run concurrently.  tol = 0: corr_steps iterations per instance
 * (nedy_decomp_tstp); tol > 0: the residual exit of nedy_decomp_tstp_tol with at most
 * corr_steps.  iters (optional, n entries) receives the iterations of each instance.
 * On an error the remaining instances are not started and the first failing instance
 * is named in nedy_last_error. */
typedef struct nedy_batch nedy_batch;
typedef struct {
  nedy_ctx *ctx;
  nedy_gf *G, *Sigma;
  nedy_buf *hmf;
  const nedy_buf *h_all;
  double mu;
} nedy_batch_instance;
int nedy_batch_create(const nedy_batch_instance *inst, int n, int workers, nedy_batch **out);
int nedy_batch_destroy(nedy_batch *b);
int nedy_batch_tstp(nedy_batch *b, int tstp, int corr_steps, double tol, int *iters);

#ifdef __cplusplus
}
#endif
#endif /* NEDY_H */
