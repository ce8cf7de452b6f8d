/*
 * nqs.h — C ABI of libnqs.so, the B200 (sm_100a) kernels of one VMC iteration over persistent
 * walkers for the continuum spinor Psiformer of wenqin-chen/continuum-nqs.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and returns an int status
 * (NQS_OK == 0). All array arguments are CALLER-OWNED DEVICE memory unless a name ends in _host.
 * The library allocates no device memory per call: scratch memory is a caller-provided workspace
 * whose size the matching *_workspace_size function reports. (The first Cholesky on a device creates
 * one high-priority side stream and two events, kept for the process, for its look-ahead.) Work is enqueued on the given cudaStream_t
 * (passed as void*) and is asynchronous; no entry point synchronises the device except
 * nqs_model_create / nqs_ewald_create (one-time uploads of constants).
 *
 * Layouts
 *   theta   : float64[P]   the real ravel of the flax parameter tree (complex leaf -> re block,
 *                          im block), leaf order = sorted dict keys (reference src/nqs/minsr.py:30-53)
 *   R       : float64[W][N][2]  Cartesian positions;   S : int32[W][N] spins in {0,1}
 *   complex : interleaved (re, im) float64 pairs
 *
 * Reference interfaces replaced (paths inside wenqin-chen/continuum-nqs):
 *   nqs_logpsi          <- ContinuumSpinorPsiformer.__call__ / make_logpsi   src/nqs/psiformer.py:118-196
 *   nqs_local_energy    <- make_local_energy(...)(R,S) under jax.vmap        src/nqs/local_energy.py:40-117
 *   nqs_ewald_*         <- make_ewald_lattice / make_ewald                   src/nqs/ewald.py:26-73
 *   nqs_mcmc_sweeps     <- make_mcmc sweep scanned over sweeps, vmapped      src/nqs/sampler.py:25-91,
 *                                                                            src/nqs/minsr.py:107-118
 *   nqs_per_sample_O    <- per_sample_O                                      src/nqs/minsr.py:56-65
 *   nqs_logpsi_vjp      <- jax.grad of the surrogate loss in make_train_step src/nqs/train.py:53-59
 *   nqs_minsr_direction <- _otil_etil + minsr_direction                      src/nqs/minsr.py:68-81
 *   nqs_clip_energies   <- the median-MAD clip inside train_minsr            src/nqs/minsr.py:142-150
 */
#ifndef NQS_H_
#define NQS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------- */
#define NQS_OK                0
#define NQS_ERR_INVALID_ARG   1   /* null pointer, negative size, inconsistent descriptor       */
#define NQS_ERR_UNSUPPORTED   2   /* shape outside the compiled limits (N, d, heads, K, ...)    */
#define NQS_ERR_WORKSPACE     3   /* workspace smaller than *_workspace_size reported           */
#define NQS_ERR_CUDA          4   /* a CUDA runtime call or kernel launch failed                */
#define NQS_ERR_NONFINITE     5   /* non-finite value where the algorithm cannot recover        */
#define NQS_ERR_TIMEOUT       6   /* a bounded device wait ran out                              */
#define NQS_ERR_NOT_SPD       7   /* Cholesky met a non-positive pivot                          */

/* ---- precision of the wavefunction network ------------------------------------------------ */
#define NQS_PREC_FP64   0   /* every stage in float64                                         */
#define NQS_PREC_MIXED  1   /* network in float32 with its Dense GEMMs on the tcgen05 tensor
                               cores (TF32 operands, float32 accumulation) where the shapes
                               allow; determinants, LU pivots, log-space sums, energies float64 */
#define NQS_PREC_MIXED_SIMT 2  /* as NQS_PREC_MIXED with every GEMM on the float32 SIMT cores  */
#define NQS_PREC_MIXED_BF16 3  /* as NQS_PREC_MIXED with BF16 operands (kind::f16, float32
                                  accumulation) for the Dense layers whose K is a multiple of
                                  64 (the rest TF32); activations stay float32 in memory    */

/* ---- compiled limits ---------------------------------------------------------------------- */
#define NQS_MAX_DEPTH     16
#define NQS_MAX_ELEC      64
#define NQS_MAX_EMBED     128
#define NQS_MAX_DETS      16
#define NQS_MAX_FREQ      16
#define NQS_MAX_KNOTS     64

/* index of each per-block tensor inside NqsModelDesc.off_block[b][.] (flax names) */
enum NqsBlockParam {
  NQS_B_DENSE0_BIAS = 0, NQS_B_DENSE0_KERNEL, NQS_B_DENSE1_BIAS, NQS_B_DENSE1_KERNEL,
  NQS_B_LN0_BIAS, NQS_B_LN0_SCALE, NQS_B_LN1_BIAS, NQS_B_LN1_SCALE,
  NQS_B_K_BIAS, NQS_B_K_KERNEL, NQS_B_O_BIAS, NQS_B_O_KERNEL,
  NQS_B_Q_BIAS, NQS_B_Q_KERNEL, NQS_B_V_BIAS, NQS_B_V_KERNEL,
  NQS_B_NPARAM
};

/* Wavefunction description: the fields of ContinuumSpinorPsiformer (src/nqs/psiformer.py:100-116)
 * plus the offset of every parameter tensor inside theta (-1 = absent). */
typedef struct NqsModelDesc {
  int32_t n_elec, embed_dim, depth, n_heads, ff_mult, n_freq, n_dets, n_g;
  int32_t learnable_env, use_jastrow, jastrow_kind /* 0 = rbf, 1 = cusp */, n_knots;
  double cusp;
  double A[4];                 /* cell matrix, row-major, columns are lattice vectors          */
  const double* Gs_host;       /* [n_g][2] envelope plane waves                                */
  const double* W_host;        /* [n_elec][n_g][2 spins] complex (interleaved re, im)          */
  const double* knots_host;    /* [n_knots] rbf centres (numpy linspace(0, r_c, n_knots))      */
  int64_t n_params;            /* P                                                            */
  int64_t off_final_ln_bias, off_final_ln_scale;
  int64_t off_embed_bias, off_embed_kernel;
  int64_t off_backflow_bias, off_backflow_kernel;          /* complex leaves                   */
  int64_t off_dW, off_det_logw, off_jas_c_opp, off_jas_c_same, off_jastrow_loga;
  int64_t off_block[NQS_MAX_DEPTH][NQS_B_NPARAM];
} NqsModelDesc;

typedef struct NqsModel NqsModel;
typedef struct NqsEwald NqsEwald;

/* Library / device information. */
int nqs_version(void);
const char* nqs_status_string(int status);
/* Last error detail (thread-local, human readable). */
const char* nqs_last_error(void);
/* Number of kernels this library has launched since it was loaded (process-wide). */
unsigned long long nqs_kernel_launches(void);
/* Optional cudaEvent_t pair (NULL to clear) recorded on the caller's stream immediately before and
 * after the Gram kernel inside nqs_minsr_direction, for timing it in isolation. */
int nqs_profile_events(void* start_event, void* stop_event);
/* Bound of every device-side wait of the library, in polls (no reference counterpart; failure
 * detection, process-wide): the tensor-core kernels' mbarrier waits (default 2^22 polls) and the
 * triangular solves' flag waits (default 2^21 polls, with back-off). 0 restores the defaults. A
 * wait that runs out aborts its kernel without hanging: a tensor-core Gram reports it through
 * nqs_minsr_direction's status; a network pass (nqs_logpsi, nqs_local_energy, nqs_mcmc_sweeps,
 * ...) sets its log psi / gradient / Laplacian outputs to NaN; a triangular solve publishes NaN. */
int nqs_set_wait_limit(unsigned polls);
/* Implementation selection (no reference counterpart; process-wide, default off): with it on,
 * the float64 Cholesky of the MinSR / Gram solves runs as one persistent kernel over a task graph
 * of 128 x 128 tiles (factor, panel solve and trailing-update tasks dealt in a look-ahead
 * order, bounded waits on per-tile counters); off, one launch per 64-column panel. Same pivot
 * floor and status flags. Off by default: its fixed dealing order hands out a step's trailing
 * updates before the next step's factor, so the critical path waits behind them (27.3 ms
 * against 22.9 ms at n = 8192 on a B200). */
int nqs_set_cholesky_dag(int enable);
/* Implementation selection (no reference counterpart; process-wide, default on): the K = 256
 * trailing updates of the preconditioner Cholesky in the mixed-precision MinSR solves
 * (gram_prec 1 / 2) run on the tensor cores, each float64 operand split into a TF32 part and a
 * float32 remainder (three TF32 products, float32 accumulation over 256 terms: ~1e-6 relative to
 * the float64 update, against the 1e-4 mean(T_ii) shift the preconditioner already carries).
 * Off: float64 CUDA-core updates. The float64 solve (gram_prec 0) always uses the latter. */
int nqs_set_cholesky_tc(int enable);
/* Implementation selection (no reference counterpart; process-wide, default on): the tensor-core
 * Gram (nqs_gram and the mixed-precision MinSR solves) computes 256 x 256 tiles per CTA, two
 * M = 128 accumulators in tensor memory against one shared B panel; off, 128 x 256 tiles. Same
 * float32 accumulation order per entry, so the same results. */
int nqs_set_gram_wide(int enable);
/* Shift of the preconditioner factor in the mixed-precision MinSR solves (gram_prec 1 / 2), relative
 * to mean(T_ii) of the tensor-core Gram (no reference counterpart; process-wide): the factor is
 * that of T_tc + (lam + rel mean(T_ii)) I, covering the Gram's float32-accumulation indefiniteness;
 * the conjugate gradients still solve at lam. Default 1e-4; rel = 0 restores it. */
int nqs_set_preconditioner_shift(double rel);
/* Self-test of the flag waits (no reference counterpart; used by the failure-detection test):
 * solves L x = v in place (L: float64 [n][n] lower triangular, device; n <= 64 x 255) with the
 * wavefront triangular solve whose 64-row block `dead_block` never publishes its result (-1: all
 * publish), so the blocks after it wait at most wait_limit polls, give up and publish NaN.
 * status_dev (device int) receives 1 when a wait ran out, else 0. Workspace: (2 x 64 + 64 x 64 x
 * ceil(n / 64)) doubles. */
int nqs_selftest_bounded_wait(const double* L, int n, int dead_block, unsigned wait_limit,
                              double* v, void* workspace, size_t workspace_bytes, int* status_dev,
                              void* stream);
/* Per-launch timing of the tensor-core row GEMMs of the float32 network (profiling aid, no
 * reference counterpart): while enabled, every launch is bracketed by a pair of CUDA events (up to
 * 16384 launches are kept) and its algorithmic bytes (operand rows, weights, output, residual)
 * are summed. nqs_profile_gemm_read waits for the recorded events, returns the summed kernel time
 * (ms), bytes and launch count since the last read, and clears them. */
int nqs_profile_gemm(int enable);
int nqs_profile_gemm_read(double* ms, double* bytes, long long* launches);
/* Implementation selection (no reference counterpart; process-wide, default on): with fusion on,
 * each transformer block of a single-channel (value) pass of the float32 path runs as one fused
 * tensor-core launch when N <= 16, embed_dim is 32 or 64 and ff_mult is 2; off, the same block
 * runs as separate LayerNorm / GEMM / attention / GEMM launches. Both compute the same function
 * with the same TF32 products; the switch exists so that the two can be compared. */
int nqs_set_block_fusion(int enable);
/* Implementation selection (no reference counterpart; process-wide, default on): with it on,
 * the kernels of more than 16 electrons run one 256-thread CTA per job (determinant head: every
 * elimination step and tangent product spread over the CTA; up to 64 electrons, 48 with the
 * Laplacian) and per (job, head) (attention: up to 64 tokens, head width 8 or 16); off, one
 * warp per (job, determinant) and per (job, head). Same functions, same pivot rule; the switch
 * exists so that the two can be compared. */
int nqs_set_large_n_kernels(int enable);
/* Implementation selection (no reference counterpart; process-wide, default off): with it on,
 * attention over 16 tokens or fewer also runs one 256-thread CTA per (job, head) instead of one
 * warp per (job, head). Same function; the switch exists so that the two can be compared (at
 * configuration 2 on a B200 the local energies took 59.5 ms with it, 48.2 ms without). */
int nqs_set_attention_cta_small(int enable);
/* Implementation selection (no reference counterpart; process-wide, default off): with it on,
 * the float32 per-sample Jacobian and log-psi VJP passes run their Dense layers on the tensor
 * cores (TF32, or BF16 with NQS_PREC_MIXED_BF16) like the forward passes: the recomputed
 * forward as row GEMMs, the reverse X W^T products reading the stored kernels. Off, those
 * layers stay float32 on the CUDA cores. On a B200 at configuration 2 it saves 2.2 ms of a
 * 14.1 ms Jacobian and moves the MinSR update from 8.4e-4 to 5.2e-3 of the float64 one. */
int nqs_set_jacobian_tc(int enable);
/* Implementation selection (no reference counterpart; process-wide, default on): with it on, the
 * attention of the float32 multi-channel batches (forward-Laplacian local energies, spin-flip
 * gradients; head width 16, up to 64 tokens) of the tensor-core network precisions (mixed,
 * mixed_bf16; not mixed_simt) runs on the tensor cores: every product of every
 * channel as mma.sync m16n8k8 TF32 chains, the probabilities and the Laplacian accumulators held
 * in accumulator fragments. Value-only passes (sampling, the Jacobian's forward) keep the float32
 * CUDA-core kernels. On a B200 it takes the local energies of configuration 2 from 48.3 to
 * 45.4 ms and of configuration 5 (512 walkers) from 454 to 365 ms at unchanged error against the
 * float64 path; off restores the float32 kernels. */
int nqs_set_attention_mma(int enable);
/* Pipeline depth cap of the tensor-core row GEMMs (no reference counterpart; process-wide,
 * read when a launch is enqueued): at most max_stages (2..4) operand tiles in flight per CTA;
 * 0 restores the default (4). A tuning knob of the multi-instance autotuner. */
int nqs_set_rowgemm_stages(int max_stages);
/* Per-launch timing of the fused value-pass blocks (profiling aid, no reference counterpart),
 * recorded while nqs_profile_gemm(1) is in force: summed kernel time (ms), algorithmic HBM bytes
 * (rows in and out, weights once), tensor-core and attention flops, and the launch count since
 * the last read, which clears them. */
int nqs_profile_block_read(double* ms, double* bytes, double* flops, long long* launches);

/* Model handle: validates the descriptor and uploads the immutable constants (Gs, W, knots).
 * Replaces the flax module construction in src/nqs/psiformer.py:100-116. */
int nqs_model_create(const NqsModelDesc* desc, NqsModel** out);
int nqs_model_destroy(NqsModel* model);
int64_t nqs_model_n_params(const NqsModel* model);

/* Workspace bytes for an operation on n_walkers walkers.  op: */
#define NQS_OP_LOGPSI      0
#define NQS_OP_LOCAL_E     1
#define NQS_OP_MCMC        2
#define NQS_OP_PER_SAMPLE_O 3
#define NQS_OP_PER_SAMPLE_O_CKPT 4   /* nqs_per_sample_O_ex with checkpoint_blocks != 0       */
#define NQS_OP_LOGPSI_VJP  5         /* nqs_logpsi_vjp, every block's activations kept        */
#define NQS_OP_LOGPSI_VJP_CKPT 6     /* nqs_logpsi_vjp with checkpoint_blocks != 0            */
int nqs_workspace_size(const NqsModel* model, int op, int n_walkers, int precision,
                       size_t* bytes);

/* log psi for W configurations.  out_logpsi: complex[W].
 * Replaces model.apply(params, R, S) vmapped over walkers (src/nqs/psiformer.py:118-196). */
int nqs_logpsi(NqsModel* model, const double* theta, const double* R, const int32_t* S,
               int n_walkers, double* out_logpsi, int precision,
               void* workspace, size_t workspace_bytes, void* stream);

/* Local energy E_loc = kinetic + Zeeman + Rashba SOC (+ Coulomb if ewald != NULL) per walker,
 * with the kinetic Laplacian from the forward Laplacian. out_eloc: complex[W];
 * out_logpsi (nullable): complex[W]. Replaces make_local_energy (src/nqs/local_energy.py:40-117)
 * and the `e + coulomb(R)` of src/nqs/minsr.py:124-126. */
int nqs_local_energy(NqsModel* model, const double* theta, const double* R, const int32_t* S,
                     int n_walkers, double m_star, double lambda_r, double h_z,
                     const NqsEwald* ewald, double* out_eloc, double* out_logpsi,
                     int precision, void* workspace, size_t workspace_bytes, void* stream);
/* nqs_local_energy with an external spin field (the ext_field of make_local_energy,
 * src/nqs/local_energy.py:41-42,86-88,109-111): field = f(r_i) evaluated by the caller at the
 * walkers' positions, float64[W][N][3] (f_x, f_y, f_z), adding
 *   - sum_i f_z(r_i) (sigma_z)_{s_i s_i}  -  sum_i [f_x sigma_x + f_y sigma_y]_{s_i s'} Psi(s')/Psi. */
int nqs_local_energy_field(NqsModel* model, const double* theta, const double* R,
                           const int32_t* S, int n_walkers, double m_star, double lambda_r,
                           double h_z, const NqsEwald* ewald, const double* field,
                           double* out_eloc, double* out_logpsi, int precision, void* workspace,
                           size_t workspace_bytes, void* stream);

/* Single-particle spin estimators of W configurations from the N spin-flip ratios
 * ratio_i = Psi(s_i -> 1 - s_i) / Psi (src/nqs/observables.py:31-45): out_sx = ratio (complex
 * [W][N]), out_sy = -i sz ratio (complex [W][N]), out_sz = 1 - 2 s_i (float64 [W][N]); a
 * non-finite ratio (exactly singular flipped determinant) gives 0. Workspace: NQS_OP_LOCAL_E. */
int nqs_spin_estimators(NqsModel* model, const double* theta, const double* R, const int32_t* S,
                        int n_walkers, double* out_sx, double* out_sy, double* out_sz,
                        int precision, void* workspace, size_t workspace_bytes, void* stream);

/* Gradient and Laplacian of log psi (forward Laplacian): out_grad complex[W][2N],
 * out_lap complex[W], out_logpsi complex[W] (each nullable). */
int nqs_grad_laplacian(NqsModel* model, const double* theta, const double* R, const int32_t* S,
                       int n_walkers, double* out_logpsi, double* out_grad, double* out_lap,
                       int precision, void* workspace, size_t workspace_bytes, void* stream);

/* Metropolis sweeps (src/nqs/sampler.py:36-57): per sweep one joint Gaussian move of all
 * electrons (PBC wrapped) and n_spin_flips single-spin flips, each accepted iff
 * u < exp(min(0, 2 Re dlogpsi)). R_io, S_io, logpsi_io (complex[W], the cached current value)
 * are updated in place. Randomness: counter-based Philox4x32-10 keyed by (seed, counter) and
 * (walker, sweep, draw), unless the inj_* buffers are given, in which case they are used
 * verbatim: inj_normals f64[n_sweeps][W][N][2], inj_u_pos f64[n_sweeps][W],
 * inj_flip_idx i32[n_sweeps][n_spin_flips][W], inj_u_flip f64[n_sweeps][n_spin_flips][W].
 * out_acc_pos / out_acc_spin: f64[W] accepted fraction over the sweeps (nullable).
 * out_d (nullable): f64[n_sweeps][1 + n_spin_flips][W] every log-ratio d that was tested. */
int nqs_mcmc_sweeps(NqsModel* model, const double* theta, double* R_io, int32_t* S_io,
                    double* logpsi_io, int n_walkers, int n_sweeps, int n_spin_flips,
                    double step, uint64_t seed, uint64_t counter,
                    const double* inj_normals, const double* inj_u_pos,
                    const int32_t* inj_flip_idx, const double* inj_u_flip,
                    double* out_acc_pos, double* out_acc_spin, double* out_d,
                    int precision, void* workspace, size_t workspace_bytes, void* stream);

/* nqs_mcmc_sweeps with the random stream's sweep counter in device memory (uint64, read when
 * the kernels run and advanced by n_sweeps on the device at the end), for a sequence of calls
 * captured once in a CUDA graph and replayed: each replay draws fresh proposals. No injected
 * randomness. */
int nqs_mcmc_sweeps_devctr(NqsModel* model, const double* theta, double* R_io, int32_t* S_io,
                           double* logpsi_io, int n_walkers, int n_sweeps, int n_spin_flips,
                           double step, uint64_t seed, uint64_t* counter_dev,
                           double* out_acc_pos, double* out_acc_spin, int precision,
                           void* workspace, size_t workspace_bytes, void* stream);

/* Per-sample Jacobian O[w][k] = d log psi(R_w,S_w) / d theta_k written as two real rows:
 * out_O is [2W][P] with rows 0..W-1 = Re O and rows W..2W-1 = Im O, dtype f64 (out_dtype 0)
 * or f32 (out_dtype 1). Hand-written reverse mode (src/nqs/minsr.py:56-65). */
int nqs_per_sample_O(NqsModel* model, const double* theta, const double* R, const int32_t* S,
                     int n_walkers, void* out_O, int out_dtype, int precision,
                     void* workspace, size_t workspace_bytes, void* stream);
/* nqs_per_sample_O with activation checkpointing (the same per_sample_O, src/nqs/minsr.py:56-65):
 * checkpoint_blocks != 0 keeps only each transformer block's input during the forward and
 * recomputes the block's activations (LayerNorms, q/k/v, attention output, MLP) just before its
 * reverse step. O is bit-identical to the stored-activation pass; the activation memory per
 * walker drops from depth x (block intermediates) to one block's, so a workspace of the same size
 * holds more walkers per chunk. Workspace: NQS_OP_PER_SAMPLE_O_CKPT (NQS_OP_PER_SAMPLE_O when
 * checkpoint_blocks == 0). */
int nqs_per_sample_O_ex(NqsModel* model, const double* theta, const double* R, const int32_t* S,
                        int n_walkers, void* out_O, int out_dtype, int precision,
                        int checkpoint_blocks, void* workspace, size_t workspace_bytes,
                        void* stream);
/* Vector-Jacobian product of log psi over W configurations without forming O:
 *   out_grad[k] = sum_w Re(cotangent_w * d log psi(R_w, S_w) / d theta_k)     (float64[P])
 * cotangent: complex[W]. This is jax.vjp of the vmapped log psi (JAX's convention for a complex
 * output of real parameters), the derivative train.py takes of its surrogate loss
 * 2 mean_w Re[conj(e_w - mean e) log psi_w] (src/nqs/train.py:53-59) with
 * cotangent_w = (2/W) conj(e_w - mean e). Hand-written reverse mode; the weight gradients are
 * reduced over walkers on the device (float64 atomics, so the last bits depend on the order).
 * checkpoint_blocks as in nqs_per_sample_O_ex. Workspace: NQS_OP_LOGPSI_VJP or
 * NQS_OP_LOGPSI_VJP_CKPT. */
int nqs_logpsi_vjp(NqsModel* model, const double* theta, const double* R, const int32_t* S,
                   int n_walkers, const double* cotangent, double* out_grad, int precision,
                   int checkpoint_blocks, void* workspace, size_t workspace_bytes, void* stream);

/* MinSR direction (src/nqs/minsr.py:68-81): O is the [2W][P] output of nqs_per_sample_O
 * (o_dtype 0 = f64, 1 = f32), eps complex[W] the (clipped) local energies.
 *   Otil = O - column mean (per half), etil = [Re; Im](eps - mean eps),
 *   y = (Otil Otil^T + lam I)^-1 etil,  dtheta = Otil^T y;  out_dtheta (nullable) receives
 *   dtheta, theta_io (nullable) is updated theta -= lr dtheta in the same pass.
 * gram_prec 0: float64 SIMT Gram T = Otil Otil^T (a float64 O is centred IN PLACE), float64
 *   Cholesky of T + lam I, then max_iters (0..64) steps of iterative refinement against the
 *   exact operator.
 * gram_prec 1 (BF16) / 2 (TF32): the Gram runs on the tcgen05 tensor cores (float32
 *   accumulation); the float64 Cholesky factor of T + (lam + delta) I, delta = 1e-4 mean(T_ii),
 *   preconditions conjugate gradients on the EXACT system (Otil Otil^T + lam I) y = etil, whose
 *   operator is applied from O itself with float64 accumulation: the solve is at the caller's
 *   lam. CG stops after max_iters iterations or when the preconditioned residual has fallen by
 *   tol (sqrt(r.z / r0.z0) <= tol); the iterations left are skipped on the device.
 * damping_out (nullable, device double) receives delta (0 for the float64 Gram).
 * info_dev (nullable, device int[5]): [0] non-zero when a Cholesky pivot was not positive,
 * [1] a tensor-core Gram CTA hit its bounded-wait limit, [2] pivots raised to the floor
 * u max T_ii (u = 2^-16 BF16, 2^-20 TF32) in the preconditioner's factor, [3] CG iterations done,
 * [4] why CG stopped (0 iteration limit, 1 converged, 2 loss of positivity). */
int nqs_minsr_workspace_size(int n_walkers, int64_t n_params, int o_dtype, int gram_prec,
                             size_t* bytes);
int nqs_minsr_direction_ex(void* O, int o_dtype, const double* eps, int n_walkers,
                           int64_t n_params, double lam, int gram_prec, int max_iters, double tol,
                           double* out_dtheta, double* theta_io, double lr, int* info_dev,
                           double* damping_out, void* workspace, size_t workspace_bytes,
                           void* stream);
/* The same with tol = 1e-2, max_iters = n_refine and status_dev (nullable, device int[3]) =
 * info_dev[0..2]. */
int nqs_minsr_direction(void* O, int o_dtype, const double* eps, int n_walkers,
                        int64_t n_params, double lam, int gram_prec, int n_refine,
                        double* out_dtheta, double* theta_io, double lr, int* status_dev,
                        double* damping_out, void* workspace, size_t workspace_bytes,
                        void* stream);

/* Lower triangle of T = A A^T on the tcgen05 tensor cores (float32 accumulation, float64 out):
 * A row-major [M][lda] of BF16 (a_dtype 1) or float32 read as TF32 (a_dtype 2); lda * elem size
 * a multiple of 16 bytes; err_dev (device int, nullable) set to 1 if a bounded wait ran out. */
int nqs_gram(const void* A, int a_dtype, int M, int64_t K, int64_t lda, double* T, int64_t ldt,
             int* err_dev, void* stream);

/* x = (A A^T + lam I)^-1 rhs for a float64 row-major A [M][K] (float64 Gram + Cholesky); used
 * for the explicit parameter-space SR of src/nqs/minsr.py:84-88 (A = Otil^T). */
int nqs_gram_solve_workspace_size(int M, int64_t K, size_t* bytes);
int nqs_gram_solve(const double* A, int M, int64_t K, double lam, const double* rhs, double* x,
                   void* workspace, size_t workspace_bytes, void* stream);

/* Energy gradient of the surrogate 2 mean_w Re[conj(e_w - mean e) log psi_theta(x_w)]
 * (src/nqs/train.py:53-59): grad = (2/W) sum_w Re(conj(e_w - mean e) O_w), with O the [2W][P]
 * rows of nqs_per_sample_O. The workspace needs 2W doubles. */
int nqs_energy_gradient(const void* O, int o_dtype, const double* e, int n_walkers,
                        int64_t n_params, double* out_grad, void* workspace,
                        size_t workspace_bytes, void* stream);
/* nqs_energy_gradient for callers that hold no workspace and must not allocate device memory.
 * No counterpart in the reference: it exists for callers such as a framework's custom-call
 * handler whose allocator owns the device memory. Same result as nqs_energy_gradient; its 2W
 * doubles of scratch are a file-scope device array inside libnqs (512 KiB per device), so it
 * allocates nothing and n_walkers is limited to NQS_NOALLOC_MAX_WALKERS (larger: returns
 * NQS_ERR_UNSUPPORTED with the reason in nqs_last_error). The first call on each device resolves
 * that array's address with the device current; make it before any stream capture. All calls on
 * a device share the array: calls that overlap in time (other streams, other host threads) race
 * and must be serialised by the caller. The resolved address is cached per device ordinal for the
 * life of the process: resetting a device (cudaDeviceReset, or tearing down its primary context)
 * while libnqs is loaded is not supported for this entry point. */
#define NQS_NOALLOC_MAX_WALKERS 32768
int nqs_energy_gradient_noalloc(const void* O, int o_dtype, const double* e, int n_walkers,
                                int64_t n_params, double* out_grad, void* stream);
/* Adam step (optax.adam defaults b1 0.9, b2 0.999, eps 1e-8) on the real ravel theta; t >= 1 is
 * the step count used for bias correction. m, v: float64[P] moment buffers (start at 0). */
int nqs_adam_update(double* theta, const double* grad, double* m, double* v, int64_t n_params,
                    double lr, double b1, double b2, double eps, int t, void* stream);
/* The Adam step of optax.adam applied to the tree gradient that jax.grad gives train.py
 * (src/nqs/train.py:53-61): a complex leaf element c = a + i b is updated as one complex number
 * with JAX's gradient G = dL/da - i dL/db, one complex first moment and the real second moment of
 * |G|^2. grad is the real-ravel gradient (dL/da, dL/db) that nqs_logpsi_vjp returns; partner
 * (int64[P], device) gives for each component of a complex element the index of the other one
 * (re block k <-> im block k + n) and -1 for a real parameter. */
int nqs_adam_update_complex(double* theta, const double* grad, double* m, double* v,
                            const int64_t* partner, int64_t n_params, double lr, double b1,
                            double b2, double eps, int t, void* stream);

/* Median-MAD clip of Re e (src/nqs/minsr.py:145-148): med = median(Re e),
 * mad = median(|Re e - med|) + 1e-12, Re e clipped to med +- clip_k mad, Im kept.
 * stats (nullable, f64[5]): mean Re e, std(Re e)/sqrt(W), var(Re e), med, mad. W <= 16384. */
int nqs_clip_energies(const double* e, int n_walkers, double clip_k, double* out_eclip,
                      double* stats, void* stream);

/* Ewald (src/nqs/ewald.py:26-73): eta = ewald_alpha, or sqrt(pi/area) when ewald_alpha <= 0. */
int nqs_ewald_create(const double A[4], double alpha, double ewald_alpha, int n_real,
                     int n_recip, NqsEwald** out);
int nqs_ewald_destroy(NqsEwald* ewald);
int nqs_ewald_zeta(const NqsEwald* ewald, double* zeta_M);
/* ewald_pair(r) for M displacement vectors r f64[M][2] -> out f64[M]. */
int nqs_ewald_pair(const NqsEwald* ewald, const double* r, int M, double* out, void* stream);
/* coulomb_energy(R) for W walkers of N electrons -> out f64[W]. */
int nqs_ewald_energy(const NqsEwald* ewald, const double* R, int n_walkers, int n_elec,
                     double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* NQS_H_ */
