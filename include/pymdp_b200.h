/*
 * pymdp_b200 — C-ABI of the B200-native (sm_100a) FPI and EFE hot paths.
 *
 * Every entry point takes plain pointers and sizes (no framework types), runs
 * on the caller's CUDA stream, never synchronises the stream and never copies
 * to the host, and returns an int32 status (0 = success). On failure the
 * thread-local message from b2_last_error() names the entry point and the
 * offending argument, in the style of the reference's
 * `ffi::Error(kInvalidArgument, "fpi_ffi: ...")` (pymdp/ffi/common/error_helpers.h:24-49).
 *
 * Device pointers must be CUDA device (or managed) memory on the current
 * device. Unless stated otherwise, float buffers are float32, integer buffers
 * int32, attribute arrays (shapes, offsets, dependency lists) are HOST int64
 * arrays, exactly like the reference's XLA FFI attributes.
 */
#ifndef PYMDP_B200_H_
#define PYMDP_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum {
  B2_OK = 0,
  B2_ERR_INVALID_ARGUMENT = 1, /* shape / offset / dependency inconsistency   */
  B2_ERR_UNSUPPORTED = 2,      /* valid input outside this build's limits     */
  B2_ERR_CUDA = 3,             /* CUDA runtime error (launch, allocation ...) */
  B2_ERR_NO_DEVICE = 4         /* no sm_100 device / kernel image unavailable */
};

/* Limits of this build. Rank cap matches the reference's
 * kMaxFfiDependencyRank = 8 (pymdp/ffi/common/modality_dispatch.h:25). */
#define B2_MAX_DEP_RANK 8
#define B2_MAX_FACTORS 16
#define B2_MAX_MODALITIES 32

/* EFE flag bits: identical values to the reference ABI
 * (pymdp/ffi/neg_efe/neg_efe_layout.h:23-42, pymdp/ffi/_efe.py FLAG_*). */
#define B2_FLAG_USE_UTILITY 1
#define B2_FLAG_USE_STATES_INFO_GAIN 2
#define B2_FLAG_USE_INDUCTIVE 4
#define B2_FLAG_USE_PARAM_INFO_GAIN 8
#define B2_FLAG_MODEL_PARAMS_STATIC 16
/* This build only (the reference ABI has no such bit): the policy matrix is the
 * full product of every factor's controls over T steps in the order of
 * control.construct_policies (pymdp/control.py:152-195), shared by all agents.
 * The tensor-core paths then evaluate every distinct policy prefix once
 * (depth t has prod(U)^(t+1) prefixes instead of P) and sum G along the tree.
 * Ignored when P != prod(U)^T, when the matrix is per agent, or by the SIMT path. */
#define B2_FLAG_POLICY_TREE 32
/* This build only: with B2_FLAG_POLICY_TREE and factor-local transitions
 * (B_dependencies[f] == [f] for every f), contract A one factor at a time over
 * the distinct predicted marginals of each factor (factor f has U_f^(t+1) of
 * them after step t, one per history of its own actions) instead of once per
 * policy prefix. Same G in another summation order, in FP32 with FP64
 * accumulation of G; the precision bits are not used. All four terms are
 * supported (the pA weights ride along the contraction as extra rows; the pB
 * and inductive terms are per factor history). Ignored (the other paths run)
 * when the tree conditions do not hold, a dependency tuple has rank above 3,
 * or a factor has more than 64 states. */
#define B2_FLAG_FACTORED 64
/* Precision selector, bits 8-9 of `flags` (unused by the reference ABI). */
#define B2_PRECISION_SHIFT 8
#define B2_PRECISION_FP32 0   /* SIMT FP32, FP32 accumulate (default)         */
#define B2_PRECISION_TF32X3 1 /* tcgen05 kind::tf32, 3-pass hi/lo split        */
#define B2_PRECISION_BF16 2   /* tcgen05 kind::f16, 3-pass BF16 hi/lo split,   */
                              /* FP32 accumulate                              */
/* The two tensor-core selectors fall back to the SIMT FP32 kernel when the
 * model exceeds their limits (more than 8 distinct dependency tuples, a
 * dependency tuple of rank above 4, more than 256 - T observation rows per
 * tuple, or a working set above 227 KB of shared memory). */

/* Message describing the last failing call on this thread ("" if none). */
const char* b2_last_error(void);
/* ABI version of this library (bumped on any signature change). */
int32_t b2_abi_version(void);
/* Capability bits; bit 2 = CUDA, mirroring pymdp_ffi_cpu_capabilities
 * (pymdp/ffi/registration/xla_register.cc:162-164, _core.py _CAP_CUDA). */
int32_t b2_capabilities(void);
/* Number of kernels this library has launched in this process (all entry
 * points, all devices). Lets callers count launches inside a timed region. */
uint64_t b2_launch_count(void);
/* Reads and clears the device error word that a kernel sets when one of its
 * bounded waits runs out (it then stops, frees its tensor memory and exits
 * instead of hanging). Synchronises the current device: diagnostics only.
 * Returns 0 (no error), 1 (a wait ran out) or -1 (the read failed). */
int32_t b2_device_error(void);

/* ================================================================== FPI ==
 * Drop-in for `pymdp_fpi_cuda_native` / FpiCudaDevice
 * (pymdp/ffi/registration/xla_register.cc:151-157, pymdp/ffi/fpi/fpi.h:30-33,
 * Python side pymdp/ffi/_fpi.py:143-270). Same buffers and attributes:
 *
 *   ll_flat  [batch, ll_offsets[M]]   per-modality log-likelihoods, each
 *                                      ll_m row-major over S[A_dep[m]]
 *   lp_flat  [batch, lp_offsets[F]]   per-factor log priors
 *   q_out    [batch, lp_offsets[F]]   posterior marginals (softmax of log q)
 *
 * Attributes S[F], ll_offsets[M+1], lp_offsets[F+1], A_dep_flat[...],
 * A_dep_offsets[M+1], num_iter. As in the reference, the batch is inferred
 * from the element counts (`lp_count / total_S`, fpi/fpi_entry.h:55-66) and
 * all three counts are checked. Runs exactly num_iter Jacobi iterations
 * (the reference JAX semantics, pymdp/algos.py:121-133; no early stop). */
int32_t b2_fpi(void* stream, const float* ll_flat, int64_t ll_count, const float* lp_flat,
               int64_t lp_count, float* q_out, int64_t q_count, const int64_t* S, int64_t S_len,
               const int64_t* ll_offsets, int64_t ll_offsets_len, const int64_t* lp_offsets,
               int64_t lp_offsets_len, const int64_t* A_dep_flat, int64_t A_dep_flat_len,
               const int64_t* A_dep_offsets, int64_t A_dep_offsets_len, int32_t num_iter);

/* Fused observation form of the same update: the log-likelihood slice gather
 * log(clip(A_m[o_m], eps)) (pymdp/maths.py:214-238 with a one-hot o_m) and
 * the log prior log(clip(prior, eps)) (pymdp/algos.py:110) are done inside
 * the kernel, so ll never exists in HBM.
 *
 *   A_flat    A_m of agent b at A_flat + b*A_agent_stride + A_offsets[m],
 *             shape (O[m], *S[A_dep[m]]) row-major. A_agent_stride = 0
 *             shares one A across the batch.
 *   obs       [batch, M] int32 observation indices, 0 <= obs < O[m].
 *             An index outside [0, O[m]) is the reference's all-zero one-hot
 *             (jax.nn.one_hot, pymdp/agent.py:673): modality m then adds
 *             nothing to that agent's update (pymdp/maths.py:233-235).
 *   prior     [batch, lp_offsets[F]] prior probabilities (not logs).
 *   q_out     [batch, lp_offsets[F]]
 *
 * The reference path this replaces is Agent.infer_states ->
 * inference.update_posterior_states -> algos.run_factorized_fpi
 * (pymdp/agent.py:773-821, pymdp/inference.py:171-191, pymdp/algos.py:88-155). */
int32_t b2_fpi_obs(void* stream, const float* A_flat, int64_t A_agent_stride,
                   const int64_t* A_offsets, int64_t A_offsets_len, const int64_t* O, int64_t O_len,
                   const int32_t* obs, const float* prior, float* q_out, int64_t batch,
                   const int64_t* S, int64_t S_len, const int64_t* A_dep_flat, int64_t A_dep_flat_len,
                   const int64_t* A_dep_offsets, int64_t A_dep_offsets_len, int32_t num_iter);

/* ================================================================== EFE ==
 * Drop-in for `pymdp_neg_efe_cuda_dev_execute` / NegEfeCudaDev
 * (pymdp/ffi/registration/xla_register.cc:89-96, pymdp/ffi/neg_efe/neg_efe.h:41-46,
 * Python side pymdp/ffi/_efe.py:491-711). Same 9 inputs, 1 output and
 * 13 int64 attribute arrays + flags:
 *
 *   policy_matrix int32 [P, T, F] (pm_batched = 0) or [Bn, P, T, F] (= 1)
 *   qs_init [Bn, qs_offsets[F]], A [Bn, A_offsets[M]], B [Bn, B_offsets[F]]
 *   (B_f flattened (S_f, *S[B_dep[f]], U_f)), C [Bn, C_offsets[M]] (C_m as
 *   (T, O_m)), I [Bn, I_offsets[F]], pA/pB (0 elements when unused),
 *   inductive_epsilon [1] or [Bn] (eps_batched).
 *   neg_efe_out [Bn, P]: G = -EFE per policy (pymdp/control.py:604-690).
 *
 * Element counts are checked like validate_buffer_counts
 * (neg_efe/neg_efe_layout.h:342-363). All four terms are implemented:
 * utility and state information gain (flag bits 0 and 1) on every precision
 * path; the inductive value (bit 2, pymdp/control.py:1021-1061) and parameter
 * information gain (bit 3, pymdp/control.py:511-602 with the exact Dirichlet
 * weight of pymdp/maths.py:783-808; pA and pB each 0 elements or
 * Bn * A_offsets[M] / Bn * B_offsets[F]) on the SIMT FP32 kernel whatever
 * precision bits 8-9 request. Bits 8-9 pick the contraction precision
 * (B2_PRECISION_*) of the other calls. An action in policy_matrix is read as
 * jnp indexing reads B_f[..., u] (pymdp/control.py:386): a negative one counts
 * from the end, then it is clamped to [0, U_f - 1]. */
int32_t b2_neg_efe(void* stream, const int32_t* policy_matrix, int64_t pm_count, int32_t pm_batched,
                   const float* qs_init, int64_t qs_count, const float* A, int64_t A_count,
                   const float* B, int64_t B_count, const float* C, int64_t C_count,
                   const float* I, int64_t I_count, const float* pA, int64_t pA_count,
                   const float* pB, int64_t pB_count, const float* inductive_epsilon,
                   int64_t eps_count, float* neg_efe_out, int64_t out_count, int64_t Bn, int64_t P,
                   int64_t T, int64_t F, int64_t M, const int64_t* S, const int64_t* O,
                   const int64_t* U, const int64_t* qs_offsets, const int64_t* A_offsets,
                   const int64_t* B_offsets, const int64_t* C_offsets, const int64_t* I_offsets,
                   const int64_t* I_depths, const int64_t* A_dep_flat, int64_t A_dep_flat_len,
                   const int64_t* A_dep_offsets, const int64_t* B_dep_flat, int64_t B_dep_flat_len,
                   const int64_t* B_dep_offsets, int32_t flags);

/* b2_neg_efe with a caller-owned cache of the tensor-core operand images (the
 * W images packed from A and C). The reference's CUDA path keeps such caches
 * inside the library, keyed by device pointer, when the caller sets
 * B2_FLAG_MODEL_PARAMS_STATIC (pymdp/ffi/neg_efe/neg_efe_cuda_entry.cc:40-90);
 * here the caller owns the buffer and its validity, so a reused address can
 * never hit a stale entry. When *pack_cache_valid is 0 the call packs A and C
 * into pack_cache (at least b2_neg_efe_pack_bytes bytes, 256-byte aligned) and
 * sets *pack_cache_valid to 1; when it is 1 the images are reused. The images
 * stay valid while A, C, Bn, the model layout and flag bits 0-1 and 8-9 are
 * unchanged; use the cache on one stream (or order the streams). Calls that
 * take the SIMT path ignore the cache. */
int32_t b2_neg_efe_cached(void* stream, const int32_t* policy_matrix, int64_t pm_count, int32_t pm_batched,
                          const float* qs_init, int64_t qs_count, const float* A, int64_t A_count,
                          const float* B, int64_t B_count, const float* C, int64_t C_count,
                          const float* I, int64_t I_count, const float* pA, int64_t pA_count,
                          const float* pB, int64_t pB_count, const float* inductive_epsilon,
                          int64_t eps_count, float* neg_efe_out, int64_t out_count, int64_t Bn, int64_t P,
                          int64_t T, int64_t F, int64_t M, const int64_t* S, const int64_t* O,
                          const int64_t* U, const int64_t* qs_offsets, const int64_t* A_offsets,
                          const int64_t* B_offsets, const int64_t* C_offsets, const int64_t* I_offsets,
                          const int64_t* I_depths, const int64_t* A_dep_flat, int64_t A_dep_flat_len,
                          const int64_t* A_dep_offsets, const int64_t* B_dep_flat, int64_t B_dep_flat_len,
                          const int64_t* B_dep_offsets, int32_t flags, uint8_t* pack_cache,
                          int64_t pack_cache_bytes, int32_t* pack_cache_valid);

/* Bytes of the pack cache b2_neg_efe_cached needs for these attributes, Bn and
 * flags (0 when the call would take the SIMT path). Host only: needs no GPU. */
int32_t b2_neg_efe_pack_bytes(int64_t Bn, int64_t P, int64_t T, int64_t F, int64_t M, const int64_t* S,
                              const int64_t* O, const int64_t* U, const int64_t* qs_offsets,
                              const int64_t* A_offsets, const int64_t* B_offsets, const int64_t* C_offsets,
                              const int64_t* I_offsets, const int64_t* I_depths, const int64_t* A_dep_flat,
                              int64_t A_dep_flat_len, const int64_t* A_dep_offsets, const int64_t* B_dep_flat,
                              int64_t B_dep_flat_len, const int64_t* B_dep_offsets, int32_t flags,
                              int64_t* bytes);

/* Size of the fixed device scratch behind b2_neg_efe_noalloc (16 MiB). */
#define B2_NOALLOC_SCRATCH_BYTES (16u << 20)

/* No counterpart in the reference: an addition of this library for callers
 * that must not allocate device memory during a call (a host that owns the
 * whole GPU through its own arena, a real-time loop that keeps allocator
 * latency out of its step, a runtime that forbids allocation inside its
 * handlers). Same arguments, validation and results as b2_neg_efe at
 * B2_PRECISION_FP32 (the SIMT kernel) for the utility and state
 * information-gain terms (flag bits 0 and 1), but its workspace of
 * Bn * T * sum_m K_m floats lives in one fixed device array of
 * B2_NOALLOC_SCRATCH_BYTES, held by every device that loads the library until
 * exit, and it calls no allocating routine. Calls whose workspace would
 * exceed that size, calls with B2_FLAG_USE_PARAM_INFO_GAIN or
 * B2_FLAG_USE_INDUCTIVE, and tensor-core precision selectors return
 * B2_ERR_UNSUPPORTED; an unknown precision selector returns
 * B2_ERR_INVALID_ARGUMENT, as in b2_neg_efe. All calls on a device share the array: calls that
 * overlap on the GPU race and give wrong results, so order them (one
 * stream). The first call on each device looks up the array's address with
 * that device current; make it before any stream capture begins. */
int32_t b2_neg_efe_noalloc(void* stream, const int32_t* policy_matrix, int64_t pm_count, int32_t pm_batched,
                           const float* qs_init, int64_t qs_count, const float* A, int64_t A_count,
                           const float* B, int64_t B_count, const float* C, int64_t C_count,
                           const float* I, int64_t I_count, const float* pA, int64_t pA_count,
                           const float* pB, int64_t pB_count, const float* inductive_epsilon,
                           int64_t eps_count, float* neg_efe_out, int64_t out_count, int64_t Bn, int64_t P,
                           int64_t T, int64_t F, int64_t M, const int64_t* S, const int64_t* O,
                           const int64_t* U, const int64_t* qs_offsets, const int64_t* A_offsets,
                           const int64_t* B_offsets, const int64_t* C_offsets, const int64_t* I_offsets,
                           const int64_t* I_depths, const int64_t* A_dep_flat, int64_t A_dep_flat_len,
                           const int64_t* A_dep_offsets, const int64_t* B_dep_flat, int64_t B_dep_flat_len,
                           const int64_t* B_dep_offsets, int32_t flags);

/* ================================================= sequence inference ==
 * Drop-in for the reference's run_mmp / run_vmp (pymdp/algos.py:392-430,
 * :512-571, reached from inference.update_posterior_states for
 * inference_algo "mmp" / "vmp", pymdp/inference.py), batched over agents:
 * marginal message passing (vmp = 0) or variational message passing
 * (vmp = 1) over a window of T steps, num_iter mirror-descent iterations of
 * step tau (update_marginals, :170-238), in FP64.
 *
 *   A        A_m of agent b at A + b * sum_m O[m] * K_m (A_batched = 1) or
 *            shared (0); each (O[m], *S[A_dep[m]]) row-major
 *   obs_idx  [Bn, T, M] int32 index observations (jnp indexing: clamped), or
 *   obs_distr [Bn, T, sum_m O[m]] distributions (exactly one of the two)
 *   B_seq    per agent, per factor the action-conditioned transitions
 *            (T - 1, S_f, *S[B_dep[f]]) row-major, factors concatenated
 *   prior    [Bn, sum_f S_f]; qs_out [Bn, T, sum_f S_f]
 * The FP64 window state (T x (sum_m K_m + 5 sum_f S_f) doubles) must fit
 * 200 KB of shared memory, else B2_ERR_UNSUPPORTED. */
int32_t b2_sequence_infer(void* stream, int32_t vmp, const float* A, int64_t A_count, int32_t A_batched,
                          const int64_t* O, int64_t M, const int32_t* obs_idx, const float* obs_distr,
                          int64_t obs_count, const float* B_seq, int64_t B_count, const float* prior,
                          int64_t prior_count, float* qs_out, int64_t qs_count, int64_t Bn, int64_t T, int64_t F,
                          const int64_t* S, const int64_t* A_dep_flat, int64_t A_dep_flat_len,
                          const int64_t* A_dep_offsets, const int64_t* B_dep_flat, int64_t B_dep_flat_len,
                          const int64_t* B_dep_offsets, int32_t num_iter, float tau);

/* ============================================================== adjoints ==
 * No counterpart in the reference's native kernels: the reference obtains
 * gradients with jax.grad of its JAX path (pymdp/ffi/_core.py:282-310,
 * `with_jax_grad`). These are hand-written reverse passes of the same
 * arithmetic, for model fitting.
 *
 * b2_neg_efe_bwd: given d_neg_efe = dL/dG [Bn, P], writes dL/dqs_init
 * [Bn, qs_offsets[F]], dL/dA, dL/dB, dL/dC (laid out like A, B, C). Utility
 * and state information gain only (flag bits 0 and 1). Arguments otherwise as
 * b2_neg_efe (no I / pA / pB / epsilon). FP32 with atomic accumulation over
 * policies; (T + 1) * total states <= 1024. */
int32_t b2_neg_efe_bwd(void* stream, const int32_t* policy_matrix, int64_t pm_count, int32_t pm_batched,
                       const float* qs_init, int64_t qs_count, const float* A, int64_t A_count,
                       const float* B, int64_t B_count, const float* C, int64_t C_count,
                       const float* d_neg_efe, int64_t dG_count, float* d_qs_init, float* d_A, float* d_B,
                       float* d_C, int64_t Bn, int64_t P, int64_t T, int64_t F, int64_t M, const int64_t* S,
                       const int64_t* O, const int64_t* U, const int64_t* qs_offsets, const int64_t* A_offsets,
                       const int64_t* B_offsets, const int64_t* C_offsets, const int64_t* A_dep_flat,
                       int64_t A_dep_flat_len, const int64_t* A_dep_offsets, const int64_t* B_dep_flat,
                       int64_t B_dep_flat_len, const int64_t* B_dep_offsets, int32_t flags);

/* b2_fpi_obs_bwd: reverse pass of b2_fpi_obs (unrolled through all num_iter
 * sweeps, FP64, every iterate recomputed on chip). Given d_q = dL/dq_out
 * [batch, S_tot], writes dL/dA (laid out like A_flat; only the observed rows
 * are non-zero; accumulated over agents when A_agent_stride = 0) and dL/dprior
 * [batch, S_tot]. Other arguments as b2_fpi_obs. */
int32_t b2_fpi_obs_bwd(void* stream, const float* A_flat, int64_t A_agent_stride, const int64_t* A_offsets,
                       int64_t A_offsets_len, const int64_t* O, int64_t O_len, const int32_t* obs,
                       const float* prior, const float* d_q, float* d_A, float* d_prior, int64_t batch,
                       const int64_t* S, int64_t S_len, const int64_t* A_dep_flat, int64_t A_dep_flat_len,
                       const int64_t* A_dep_offsets, int64_t A_dep_offsets_len, int32_t num_iter);

/* q_pi = softmax(gamma * neg_efe + log(clip(E, eps))) per agent — the step
 * the reference runs in XLA right after the FFI call
 * (pymdp/control.py:349 and :963). gamma is [Bn] (gamma_batched = 1) or a
 * single value; E is [Bn, P] (E_batched = 1) or [P]. */
int32_t b2_policy_posterior(void* stream, const float* neg_efe, const float* E, int32_t E_batched,
                            const float* gamma, int32_t gamma_batched, float* q_pi, int64_t Bn,
                            int64_t P);

/* Deterministic action selection (pymdp/control.py:115-150,
 * sampling_mode="full", action_selection="deterministic"): action[b, f] =
 * policy_matrix[argmax_p q_pi[b, p], 0, f], the first maximum on ties.
 * policy_matrix is [P, T, F] (shared) int32. */
int32_t b2_select_action(void* stream, const float* q_pi, const int32_t* policy_matrix,
                         int32_t* action, int64_t Bn, int64_t P, int64_t T, int64_t F);


/* Action selection with the reference's modes (pymdp/agent.py:939-967):
 * sampling_mode 0 = "full" (a policy, then its first step: control.py:115-150),
 * 1 = "marginal" (per control factor, from its first-step action marginal:
 * control.py:42-113; marginal mode needs U, host int64 [F], each <= 1024);
 * action_selection 0 = deterministic (first maximum), 1 = stochastic (a draw
 * from the categorical with logits alpha * log clip(x), by the Gumbel-max
 * trick, with uniforms from SplitMix64 over (seed, agent, factor, index): a
 * different generator from JAX's, and one stream per factor where the
 * reference reuses one key for every factor). policy_matrix [P, T, F] int32
 * (shared); alpha: device [Bn] (alpha_batched = 1) or a single value (read
 * only when stochastic); action [Bn, F] int32. */
#define B2_SAMPLE_MAX_U 1024
int32_t b2_sample_action(void* stream, const float* q_pi, const int32_t* policy_matrix, const int64_t* U,
                         int32_t* action, int64_t Bn, int64_t P, int64_t T, int64_t F, int32_t sampling_mode,
                         int32_t action_selection, const float* alpha, int32_t alpha_batched, uint64_t seed);

/* Agent.update_empirical_prior for inference_algo="fpi" (pymdp/agent.py:825-851):
 * out[b] = compute_expected_state(qs[b], B[b], action[b], B_dependencies)
 * (pymdp/control.py:351-389), the prior of the next step. qs [Bn,
 * qs_offsets[F]], B [Bn, B_offsets[F]] (B_f as (S_f, *S[B_dep[f]], U_f)),
 * action [Bn, F] int32 (read as jnp indexing reads B_f[..., u]: negative from
 * the end, then clamped to [0, U_f - 1]), out like qs. Attributes as
 * b2_neg_efe's. */
int32_t b2_expected_state(void* stream, const float* qs, int64_t qs_count, const float* B, int64_t B_count,
                          const int32_t* action, int64_t action_count, float* out, int64_t Bn, int64_t F,
                          const int64_t* S, const int64_t* U, const int64_t* qs_offsets, const int64_t* B_offsets,
                          const int64_t* B_dep_flat, int64_t B_dep_flat_len, const int64_t* B_dep_offsets);

/* Agent.multiaction_probabilities (pymdp/agent.py:908-937), batched:
 * out [Bn, n_unique]. marginal = 0 ("full"): out[b, i] = sum of q_pi[b, p]
 * over the policies p whose first-step actions equal unique_actions[i]
 * ([n_unique, F] int32; the reference's unique_multiactions,
 * pymdp/agent.py:396-399: the sorted distinct rows of policy_matrix[:, 0],
 * padded to prod(U) rows with -1). marginal = 1: the outer product of the
 * per-factor first-step action marginals (get_marginals,
 * pymdp/control.py:42-67), row-major over factors, n_unique = prod(U)
 * (unique_actions unused). policy_matrix [P, T, F] int32 (shared). */
int32_t b2_multiaction_probabilities(void* stream, const float* q_pi, const int32_t* policy_matrix,
                                     const int32_t* unique_actions, int64_t n_unique, int32_t marginal, int64_t Bn,
                                     int64_t P, int64_t T, int64_t F, const int64_t* U, float* out);

/* ------------------------------------------------ online Dirichlet learning
 * In-place Dirichlet updates of the flattened model buffers the FPI and EFE
 * entry points read (A_offsets / B_offsets / qs_offsets / dependency lists as
 * in b2_neg_efe; every agent's row holds its own copy). One launch updates
 * every agent and every modality (factor); one thread owns one column of one
 * agent's tensor. The reference runs these in JAX
 * (pymdp/learning.py:11-233, called from Agent.infer_parameters,
 * pymdp/agent.py:416-620, inference_algo "fpi"/"mmp"/"vmp" branch :564-567);
 * it has no FFI for them, so the entry points follow those functions'
 * arguments. lr is device [Bn] (lr_batched = 1) or a single device value.
 *
 * Observation model (learning.py:11-117):
 *   pA_m += lr * sum_t o_{m,t} (x) qs_{A_dep[m][0],t} (x) ...
 *   A_m   = clip(pA_m, MINVAL) / sum over the outcome axis
 * for every m with bit m of modality_mask set (unset = pA_m is None: neither
 * pA_m nor A_m is touched). qs: [Bn, T, S_tot]; obs: int32 [Bn, T, M] indices
 * (an index outside [0, O_m) adds nothing: jax.nn.one_hot gives zeros), or,
 * when obs_cat is non-null, float [Bn, T, sum O] distributions
 * (categorical_obs=True); obs_count counts the array passed. */
int32_t b2_update_obs_likelihood_dirichlet(
    void* stream, float* pA, float* A, int64_t A_count, const int32_t* obs, const float* obs_cat, int64_t obs_count,
    const float* qs, int64_t qs_count, const float* lr, int32_t lr_batched, int64_t Bn, int64_t T, int64_t F,
    int64_t M, const int64_t* S, const int64_t* O, const int64_t* qs_offsets, const int64_t* A_offsets,
    const int64_t* A_dep_flat, int64_t A_dep_flat_len, const int64_t* A_dep_offsets, int64_t modality_mask);

/* Transition model (learning.py:119-233 with the joints of
 * agent.py:539-543, :567): for transitions t < T-1 whose actions are all >= 0
 * (valid_transition_mask, agent.py:480-483),
 *   pB_f += lr * sum_t qs_{f,t+1} (x) qs_{B_dep[f][0],t} (x) ... (x) onehot(actions[t, f])
 *   B_f   = clip(pB_f, MINVAL) / sum over the next-state axis.
 * pB_f / B_f are [S_f, S_dep..., U_f] per agent; qs [Bn, T, S_tot] is the
 * belief sequence; actions int32 [Bn, T-1, F]. Factors without their bit in
 * factor_mask (factors_to_update) only get B_f renormalised from pB_f
 * (learning.py:201-215). When no agent has a valid transition, or T < 2,
 * nothing is written (the skip branch, agent.py:495-500, :603-604).
 * workspace: one device int32 of scratch (the any-valid flag); two launches. */
int32_t b2_update_state_transition_dirichlet(
    void* stream, float* pB, float* B, int64_t B_count, const float* qs, int64_t qs_count, const int32_t* actions,
    int64_t actions_count, const float* lr, int32_t lr_batched, int32_t* workspace, int64_t Bn, int64_t T, int64_t F,
    const int64_t* S, const int64_t* U, const int64_t* qs_offsets, const int64_t* B_offsets,
    const int64_t* B_dep_flat, int64_t B_dep_flat_len, const int64_t* B_dep_offsets, int64_t factor_mask);

/* The same update with the pairwise posteriors given instead of formed from
 * the belief sequence: the smoothing algorithms' branch of
 * Agent.infer_parameters (inference_algo "ovf" / "exact",
 * pymdp/agent.py:530-567, joints from inference.smoothing_ovf /
 * smoothing_exact) into update_state_transition_dirichlet
 * (pymdp/learning.py:119-157). joint: per agent, per factor the (T-1, S_f,
 * *S[B_dep[f]]) joints row-major, factors concatenated. A transition counts
 * when every action of that step is >= 0 (the reference's
 * _apply_transition_mask); the batch-wide skip and factor_mask as
 * b2_update_state_transition_dirichlet. */
int32_t b2_update_state_transition_from_joint(
    void* stream, float* pB, float* B, int64_t B_count, const float* joint, int64_t joint_count,
    const int32_t* actions, int64_t actions_count, const float* lr, int32_t lr_batched, int32_t* workspace, int64_t Bn,
    int64_t T, int64_t F, const int64_t* S, const int64_t* U, const int64_t* qs_offsets, const int64_t* B_offsets,
    const int64_t* B_dep_flat, int64_t B_dep_flat_len, const int64_t* B_dep_offsets, int64_t factor_mask);

/* ------------------------------------------- exact single-factor HMM smoothing
 * A batch of single-factor HMMs (pymdp's column-stochastic orientation,
 * B[next, current(, action)]), one agent per CTA, recurrences in FP64.
 *
 * b2_hmm_smoother = run_exact_single_factor_hmm_scan (pymdp/algos.py:1132-1208):
 * log-likelihoods from A and the observations (compute_log_likelihood,
 * pymdp/maths.py:214-263; obs int32 [Bn, T, M] indices, or, when obs_dist is
 * non-null, float [Bn, T, sum O] distributions as distr_obs=True), the filter
 * (hmm_filter_scan_colstoch, :959-988) and the smoother from the filtered
 * marginals (hmm_smoother_from_filtered_colstoch, :1049-1130).
 *   A      [Bn (A_batched) or 1, sum_m O_m * K]: A_m[o, k] row-major per modality
 *   prior  [Bn, K]
 *   B      U >= 1: [Bn (B_batched) or 1, K, K, U] with actions int32 [Bn, T-1]
 *          (null allowed when U == 1); U == 0: time-varying [Bn or 1, T-1, K, K]
 *   action_mode 0: jnp indexing (negative from the end, then clamped), as
 *          B0[:, :, u] in run_exact_single_factor_hmm_scan; 1: a negative
 *          action is the identity transition (invalid_action_mode="identity",
 *          pymdp/inference.py:112-163, used by smoothing_exact)
 *   outputs (float, null = not written; filtered is required):
 *          mll [Bn], filtered / predicted / smoothed [Bn, T, K],
 *          joint [Bn, T-1, K, K] (joint[t, j, i] = p(s_{t+1}=j, s_t=i | o)),
 *          cond  [Bn, T-1, K, K] (cond[t, j, i] = p(s_t=i | s_{t+1}=j, o), the
 *          reference's qss). K <= 128. */
int32_t b2_hmm_smoother(void* stream, const float* A, int64_t A_count, int32_t A_batched, const int64_t* O,
                        int64_t M, const int32_t* obs, const float* obs_dist, int64_t obs_count,
                        const float* prior, int64_t prior_count, const float* B, int64_t B_count,
                        int32_t B_batched, int64_t U, const int32_t* actions, int64_t actions_count,
                        int32_t action_mode, int64_t Bn, int64_t T, int64_t K, float* mll, float* filtered,
                        float* predicted, float* smoothed, float* joint, float* cond);

/* hmm_smoother_from_filtered_colstoch (pymdp/algos.py:1049-1130) and
 * smoothing_exact (pymdp/inference.py:595-634, action_mode 1) from given
 * filtered marginals [Bn, T, K]; B, actions and outputs as above. */
int32_t b2_hmm_smoother_from_filtered(void* stream, const float* filtered, int64_t filtered_count,
                                      const float* B, int64_t B_count, int32_t B_batched, int64_t U,
                                      const int32_t* actions, int64_t actions_count, int32_t action_mode,
                                      int64_t Bn, int64_t T, int64_t K, float* smoothed, float* joint,
                                      float* cond);

/* ------------------------------------------------------ uneven-size rollout
 * Closed-loop rollout of many agents of DIFFERENT sizes in one persistent
 * launch. Replaces, for inference_algo="fpi", no learning and deterministic
 * action selection, the reference's `rollout` (pymdp/envs/rollout.py:468-700)
 * over a `PymdpEnv` built from each agent's own A / B / D: per step and agent
 *   prior  = D at the first step, else B[..., a_prev] . qs_prev
 *            (_resolve_empirical_prior, rollout.py:65-84; agent.py:825-851);
 *   qs     = infer_states (FPI, algos.py:88-155), in FP64;
 *   G      = neg-EFE of every policy (control.py:604-690; utility and state
 *            information gain per `flags`), FP32 accumulation with the A
 *            operand in FP32 or BF16;
 *   q_pi   = softmax(gamma G + log E), E uniform (control.py:349);
 *   action = first step of the first maximum of q_pi (control.py:115-150);
 *   env    = state' ~ B[:, state, action], obs' ~ A[:, state'] (envs/env.py:
 *            333-400); the environment's draws use a counter-based generator
 *            (SplitMix64 over seed, agent, step, stream), not JAX's PRNG.
 * Transitions are factor-local: B_f[next, prev, u], stored action-major (see
 * b2_ro_agent.B_off). Policies are all
 * prod(U)^T action sequences in the order of control.construct_policies
 * (control.py:152-195). */
#define B2_RO_MAX_F 4
#define B2_RO_MAX_M 8
#define B2_RO_MAX_S 64
#define B2_RO_MAX_O 32
#define B2_RO_MAX_K 4096
#define B2_RO_MAX_STOT 256
#define B2_RO_MAX_P 1024
#define B2_RO_MAX_COLS 64
#define B2_RO_TAB_FLOATS 6144

/* One agent. Offsets are element offsets into the b2_ro_buffers arrays. */
typedef struct b2_ro_agent {
  int32_t F, M, T, P;       /* factors, modalities, policy_len, prod(U)^T     */
  int32_t n_multi, w0;      /* prod(U); prod(U)^(T-1)                         */
  int32_t S_tot, sum_K;     /* sum S_f; sum K_m                               */
  int32_t S[B2_RO_MAX_F], U[B2_RO_MAX_F];
  int32_t qs_off[B2_RO_MAX_F];  /* start of factor f within the S_tot entries */
  int32_t ustride[B2_RO_MAX_F]; /* prod(U[f+1:]) (row-major multi-action)     */
  /* Reduced policy space. A factor that no modality observes leaves neg-EFE
   * unchanged, so policies that differ only in its actions have equal G; they
   * are evaluated once, over the observed factors' actions, and expanded when
   * q_pi is formed (ties then resolve to the first policy, as in the
   * reference). */
  int32_t obs_mask;             /* bit f: some modality depends on factor f    */
  int32_t n_multi_r, P_r, w0_r; /* prod(U_observed); n_multi_r^T; ^(T-1)      */
  int32_t ustride_r[B2_RO_MAX_F]; /* stride of f in the reduced multi-action,
                                     0 for unobserved factors                 */
  int32_t O[B2_RO_MAX_M], K[B2_RO_MAX_M], rank[B2_RO_MAX_M];
  int32_t dep[B2_RO_MAX_M][B2_RO_MAX_F];     /* ascending factor indices      */
  int32_t dstride[B2_RO_MAX_M][B2_RO_MAX_F]; /* stride of each dep axis in K  */
  int64_t A_off[B2_RO_MAX_M]; /* [A_m; lin_m]: (O_m + 1) x K_m, row-major     */
  int64_t C_off[B2_RO_MAX_M]; /* C_m: O_m log-preferences                     */
  int64_t B_off[B2_RO_MAX_F]; /* B_f stored U_f x S_f x S_f (action, previous
                                 state, next state): B[next, prev, u] at
                                 (u * S_f + prev) * S_f + next                 */
  int64_t D_off;              /* S_tot                                         */
  int64_t ll_off;             /* sum_K doubles of scratch                      */
  int64_t qs_base;            /* S_tot entries of qs / qs64                    */
  int64_t G_off;              /* P entries of G                                */
  float gamma;
  int32_t reserved;
} b2_ro_agent;

/* A unit of policy evaluation: reduced policies [p_lo, p_hi) of one agent. */
typedef struct b2_ro_tile {
  int32_t agent, p_lo, p_hi, reserved;
} b2_ro_tile;

/* Device buffers of one rollout (counts in elements). */
typedef struct b2_ro_buffers {
  const b2_ro_agent* agents; /* device copy of the descriptors                */
  const b2_ro_tile* tiles;   /* device copy of the tiles                       */
  float* Aprime;             /* A rows filled by the caller; lin rows by setup */
  uint16_t* Aprime_bf16;     /* BF16 image of Aprime (precision BF16 only)     */
  int64_t Aprime_count;
  const float* B;
  int64_t B_count;
  const float* C;
  int64_t C_count;
  const float* D;
  int64_t D_count;
  double* ll;
  int64_t ll_count;
  float* qs;                 /* FP32 posterior per agent                       */
  double* qs64;              /* FP64 posterior per agent                       */
  int64_t qs_count;
  float* G;                  /* P per agent (the first P_r hold reduced G)     */
  int64_t G_count;
  int32_t* env_state;        /* n_agents x B2_RO_MAX_F                         */
  int32_t* obs;              /* n_agents x B2_RO_MAX_M                         */
  int16_t* rec_obs;          /* optional: steps x n_agents x B2_RO_MAX_M       */
  int16_t* rec_state;        /* optional: steps x n_agents x B2_RO_MAX_F       */
  int16_t* rec_action;       /* optional: steps x n_agents x B2_RO_MAX_F       */
  float* rec_qs;             /* optional: steps x qs_count                      */
  float* rec_G;              /* optional: steps x G_count                       */
  uint32_t* sync;            /* scratch, >= 2 * steps + 32 words               */
  int64_t sync_count;
} b2_ro_buffers;

/* Launch shape: threads per CTA (128, 256, 512), K-chunk of the policy
 * contraction (32, 64), largest tile (policies per tile, <= 64) and
 * precision (B2_PRECISION_FP32 or B2_PRECISION_BF16). */
typedef struct b2_ro_config {
  int32_t threads, kc, cols, precision;
} b2_ro_config;

/* No counterpart in the reference (its rollout precomputes nothing): fills
 * lin_m[k] = sum_o A_m[o, k] (C_m[o] [flag bit 0] + log A_m[o, k] [bit 1]),
 * the row of [A_m; lin_m] that carries utility and -H_A . x, in FP64, and the
 * BF16 image when `Aprime_bf16` is set. Run once after the A rows change. */
int32_t b2_rollout_setup(void* stream, const b2_ro_agent* agents_host, int64_t n_agents,
                         const b2_ro_buffers* buffers, int32_t flags);

/* Runs `steps` rollout steps of every agent, from an environment reset (state ~
 * D, first observation ~ A), in ONE cooperative persistent launch (plus a
 * memset of `sync`), so a CUDA graph can hold the whole rollout. `agents_host`
 * / `tiles_host` are host copies of buffers->agents / ->tiles and are
 * validated on every call; the tiles must cover every reduced policy
 * [0, P_r) of every agent exactly once. Device-side failures (a grid barrier that waited too long)
 * are reported in sync[2] (non-zero) with a code in sync[3]. Overlapping
 * calls on the same buffers race. */
int32_t b2_rollout(void* stream, const b2_ro_agent* agents_host, int64_t n_agents, const b2_ro_tile* tiles_host,
                   int64_t n_tiles, const b2_ro_buffers* buffers, int64_t steps, uint64_t seed, int32_t num_iter,
                   int32_t flags, const b2_ro_config* config);

#ifdef __cplusplus
}
#endif
#endif /* PYMDP_B200_H_ */
