/* cbc_b200.h -- C ABI of the B200 CKM1D ensemble integrator (libcbc_b200.so).
 *
 * Plain C, raw device pointers and sizes only.  Every entry point returns 0 on
 * success or a negative CBC_E* code; the message of the last failure is
 * available from cbc_last_error(ctx).  No C++ exception crosses this boundary.
 * All work is enqueued on the caller's CUDA stream (cudaStream_t passed as
 * void*; NULL = legacy default stream).  One context per host thread.
 *
 * Reference interface replaced (kalmi901/coupled-bubble-control):
 *   the backend solver called by Model.solve
 *     coupledbubble_control/models/model.py:108-162 (Model.solve)
 *     coupledbubble_control/models/ckm1d.py:214-253 (_make_solver)
 *     coupledbubble_control/backends/numba/rkck45_coupled_numba_solver.py:8-126
 *     coupledbubble_control/backends/cupy_cuda/rkck45_coupled_cupy_solver.py:8-106
 *   and the fused kernel it launches
 *     coupledbubble_control/backends/numba/rkck45_coupled_numba_stepper.py:116-706
 *     coupledbubble_control/backends/cupy_cuda/cuda_src/rkck45_coupled_cuda_sover.cu:206-846
 */
#ifndef CBC_B200_H
#define CBC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes ---- */
#define CBC_OK 0
#define CBC_E_INVALID (-1)      /* bad argument (null pointer, size out of range) */
#define CBC_E_UNSUPPORTED (-2)  /* valid but not supported (e.g. K > 32, nk > 4) */
#define CBC_E_CUDA (-3)         /* a CUDA runtime call failed */
#define CBC_E_NOMEM (-4)        /* device or host allocation failed */

/* ---- per-system status codes written to status_flags
 *      (reference rkck45_coupled_numba_stepper.py:27-33) ---- */
#define CBC_ACTIVE 0
#define CBC_SUCCESS 1
#define CBC_EVENT_TERMINAL 2
#define CBC_MAX_STEPS_REACHED (-1)
#define CBC_STEP_SIZE_LIMIT (-2)
#define CBC_CONVERGENCE_FAILURE (-3)
#define CBC_SINGULARITY_OR_NAN (-4)

/* ---- launch modes of cbc_solve ---- */
#define CBC_LAUNCH_RELAUNCH 0 /* reference host loop: kernel_steps per launch, then a
                                 device->host check whether every system finished */
#define CBC_LAUNCH_SINGLE 1   /* one launch with the whole step budget, no host sync */

/* ---- implicit-coupling solvers (cbc_spec.lin_solver) ----
 * CBC_LIN_RICHARDSON: relaxed Richardson iteration v <- v + w (b - A v) from
 *   v = b, stopped on the residual norm (reference ckm1d_def.py:303-404); the
 *   reference's own (and the default) behaviour.
 * CBC_LIN_LU: direct solve of the 2K x 2K system by Gauss-Jordan elimination
 *   with partial pivoting (pivot search and pivot-row broadcast by warp
 *   shuffles inside a system's lanes); exact to rounding, never fails to
 *   converge (a zero or non-finite pivot counts as a convergence failure).
 *   No counterpart in the reference's GPU kernels; its CPU path offers
 *   direct-type solvers (reference/CKM1D_reference.py:364-518). */
#define CBC_LIN_RICHARDSON 0
#define CBC_LIN_LU 1

typedef struct cbc_context cbc_context;

/* Model/execution/solver specification.  Mirrors ModelSpec, ExecutionSpec and
 * SolverSpec (reference models/specs.py:6-72).  ac: 0 CONST, 1 SW_N, 2 SW_A.
 * dense_mode: 0 the reference's sample schedule (first step at or after the
 * scheduled time, next = stored time + (t_end - t_begin)/(ndo-1)), 1 exact grid
 * (steps are shortened to land on t_begin + k (t_end - t_begin)/(ndo-1)). */
typedef struct cbc_spec {
  int32_t ns;           /* systems                                   */
  int32_t ups;          /* bubbles per system, 1..32                 */
  int32_t tile;         /* row width of the buffers (>= ups)         */
  int32_t ndo;          /* dense samples per system, 0 = none        */
  int32_t nk;           /* harmonic components, 1..4                 */
  int32_t ac;           /* acoustic field type                       */
  int32_t dense_mode;   /* 0 reference schedule, 1 exact grid        */
  int32_t lin_max_iter; /* Richardson iteration limit (100)          */
  double atol, rtol;    /* 1e-9, 1e-9                                */
  double min_step, max_step;          /* 1e-16, 0.1                  */
  double lin_atol, lin_rtol;          /* 1e-9, 1e-9                  */
  double lin_relaxation;              /* 2/3                         */
  double etol;                        /* event tolerance, 1e-5       */
  double col_threshold;               /* collision gap factor - 1, 0.1 */
  int32_t lin_solver;   /* implicit coupling: CBC_LIN_RICHARDSON (0, the
                           reference's relaxed Richardson iteration) or
                           CBC_LIN_LU (1, direct solve)                     */
  int32_t reserved;
} cbc_spec;

/* Device buffers in the reference layout (models/model.py:56-106,
 * models/buffers.py:29-71), mutated in place.  Shapes, row-major:
 *   actual_time, time_end, time_begin, time_step, actual_event   (ns)        f64
 *   actual_state                                                 (4, ns, tile) f64  R, X, U, V
 *   unit_params                                                  (13, ns, tile) f64
 *   system_params                                                (5, ns)     f64
 *   control_params                                               (4 nk, ns)  f64
 *   coupling_matrices                                            (3, ups, ns, tile) f64
 *   dense_index, status_flags                                    (ns)        i32
 *   dense_time                                                   (ndo, ns)   f64
 *   dense_state                                                  (ndo, 4, ns, tile) f64
 *   total_steps, rejected_steps, convergence_success,
 *   convergence_failures                                         (ns)        i32 (may be NULL)
 *   lin_iters (Richardson iterations, not in the reference)      (ns)        i64 (may be NULL)
 * dense_* may be NULL when ndo == 0.  Counters are incremented, not reset. */
typedef struct cbc_buffers {
  double* actual_time;
  const double* time_end;
  const double* time_begin;
  double* time_step;
  double* actual_state;
  const double* unit_params;
  const double* system_params;
  const double* control_params;
  const double* coupling_matrices;
  int32_t* dense_index;
  double* dense_time;
  double* dense_state;
  double* actual_event;
  int32_t* status_flags;
  int32_t* total_steps;
  int32_t* rejected_steps;
  int32_t* convergence_success;
  int32_t* convergence_failures;
  int64_t* lin_iters;
} cbc_buffers;

/* Optional per-call report of cbc_solve. */
typedef struct cbc_solve_stats {
  int32_t launches;       /* kernel launches made                          */
  int32_t active_left;    /* systems still active after the last launch (RELAUNCH mode) */
  double device_ms;       /* sum of per-launch device times (CUDA events)  */
} cbc_solve_stats;

/* Library version (major * 10000 + minor * 100 + patch). */
int32_t cbc_version(void);

/* Creates a context on `device` (CUDA ordinal).  Allocates a few bytes of
 * device memory for the completion counter and pinned host memory for its
 * read-back. */
int32_t cbc_create(cbc_context** out, int32_t device);
int32_t cbc_destroy(cbc_context* ctx);
/* Message of the last failure on this context ("" if none).  Valid until the
 * next call on the context.  ctx may be NULL (returns the global message). */
const char* cbc_last_error(const cbc_context* ctx);

/* Kernels this context has enqueued so far (a plan's kernels count once per
 * cbc_plan_launch).  Diagnostic; no reference counterpart. */
int64_t cbc_kernel_launches(const cbc_context* ctx);

/* Advances every system of a reference-layout ensemble by at most
 * ceil(max_steps / kernel_steps) * kernel_steps Cash-Karp steps, stopping
 * each system at time_end, at a terminal collision event or on failure.
 * Replaces the backend solver(...) of the reference
 * (backends/numba/rkck45_coupled_numba_solver.py:8-126) together with the
 * kernel it launches.  Results do not depend on kernel_steps: every launch
 * resumes exactly where the previous one stopped.  Systems still active when
 * the budget is spent get CBC_MAX_STEPS_REACHED.  `stats` may be NULL. */
int32_t cbc_solve(cbc_context* ctx, const cbc_spec* spec, const cbc_buffers* buf,
                  int64_t max_steps, int32_t kernel_steps, int32_t launch_mode, void* stream,
                  cbc_solve_stats* stats);

/* ---- batched mixed-K form --------------------------------------------------
 * A ragged ensemble: systems of different bubble counts K (1..32) in one set of
 * arrays.  Bubbles of system s are bubble_offset[s] .. bubble_offset[s]+K_s-1.
 * Layout (device memory, row-major, f64 unless noted):
 *   bubble_offset, coupling_offset   (ns) i64
 *   state                            (nb, 4)         R, X, U, V; 16-byte aligned
 *   unit_params                      (nb, up_stride) the 13 constants of
 *                                                    models/ckm1d.py:154-168
 *   system_params                    (ns, sp_stride) the 5 constants of ckm1d.py:171-175
 *   control_params                   (ns, cp_stride) PA[nk], omega[nk], phase[nk], wave[nk]
 *   coupling                         per system at coupling_offset[s]: (3, K, K),
 *                                    [c][j][i] = matrix c, source j, receiver i
 *   t, t_end, t_begin, h, event      (ns)
 *   status, dense_index              (ns) i32
 *   dense_time                       (ndo, ns)       sample-major
 *   dense_state                      (ndo, nb, 4)    sample-major; 16-byte aligned
 *   steps, rejected, conv_ok, conv_fail (ns) i32, lin_iters (ns) i64: optional
 * The spec's ns, ups and tile fields are ignored; its solver fields, nk, ac,
 * ndo and dense_mode apply to every system.  The solvers only read the
 * offsets, parameters, coupling, t_begin and t_end; cbc_admit writes all of them for
 * the slots it fills and a plan made by cbc_env_plan_create writes
 * control_params and t_end (the actions and the step's end time, see
 * cbc_env_io), which is why they are not const. */
typedef struct cbc_ensemble {
  int32_t ns;
  int32_t up_stride, sp_stride, cp_stride;
  int64_t nb;
  int64_t* bubble_offset;
  int64_t* coupling_offset;
  double* state;
  double* unit_params;
  double* system_params;
  double* control_params;
  double* coupling;
  double* t;
  double* t_end;
  double* t_begin;
  double* h;
  double* event;
  int32_t* status;
  int32_t* dense_index;
  double* dense_time;
  double* dense_state;
  int32_t* steps;
  int32_t* rejected;
  int32_t* conv_ok;
  int32_t* conv_fail;
  int64_t* lin_iters;
  int64_t* trace_load_ns;  /* optional (ns) i64: GPU global timer when a slot picked the system up */
  int64_t* trace_done_ns;  /* optional (ns) i64: GPU global timer when its result was written back */
} cbc_ensemble;

/* Work list: system ids grouped in buckets of equal K (device array `order`),
 * each bucket ordered longest expected work first.  bucket_K, bucket_begin
 * (nbuckets + 1 entries), and the optional tuning arrays threads (per-block
 * threads, 32..128), blocks_per_sm and share are host arrays.
 * share[b] (0..1], optional: the bucket's fraction of the GPU at the start.
 * With shares, every bucket starts at once with share[b] of a full-GPU grid;
 * the rest of each bucket's grid is launched behind all of them and fills SMs
 * as other buckets drain.  Without shares each bucket gets a full-GPU grid
 * and the buckets overlap only at their tails. */
typedef struct cbc_work {
  const int32_t* order;
  int32_t nbuckets;
  const int32_t* bucket_K;
  const int32_t* bucket_begin;
  const int32_t* threads;
  const int32_t* blocks_per_sm;
  const float* share;
  /* Latency lanes (may be NULL).  exclusive[b] > 0 launches bucket b first as
   * exclusive[b] blocks of 128 threads that each request all shared memory of
   * an SM, so each runs alone on its SM (minimum per-step latency for the
   * longest systems); every other bucket then sizes its grids for the
   * remaining SMs.  share[b] is ignored for such buckets. */
  const int32_t* exclusive;
  /* Time slice (0 = none): every system still running budget_ns nanoseconds
   * (device clock) after the solve started stops after its current step with
   * status -1, exactly as if max_steps had been reached, and resumes
   * bit-identically on the next call.  Lets a caller re-plan the order of the
   * remaining work from the progress observed so far. */
  int64_t budget_ns;
  /* 0: max_steps limits the steps of each system within this call (the
   * reference's kernel_steps).  1: it limits the steps accumulated in
   * ensemble.steps over all calls, so that a solve split into time slices
   * stops every system at exactly the step a single call would. */
  int32_t steps_total;
  int32_t reserved;
  /* Tuning (host arrays, may be NULL; results never depend on them):
   * slots[b] systems held per warp, 1..32/K (default 32/K: every lane
   * busy; fewer lowers intra-warp divergence); min_blocks[b] the
   * register-budget variant of the bucket's kernel, 0 (default) or 1 (one
   * more resident block per SM asked of the compiler, fewer registers per
   * thread; K <= 8 only, ignored above).  Chosen per K by the project's
   * autotuner (cbc_b200/autotune.py) together with threads. */
  const int32_t* slots;
  const int32_t* min_blocks;
} cbc_work;

typedef struct cbc_plan cbc_plan;

/* Advances every system of the ensemble by at most max_steps steps (per
 * system, per call) or until it finishes.  One persistent work-stealing kernel
 * per bucket, buckets on forked streams that join back into `stream`.
 * Results are bit-identical to cbc_solve on the same systems.  No reference
 * counterpart: the reference integrates one (NS, K) shape per kernel build
 * (backends/cupy_cuda/kernel_loader.py:35-63); this is its batched form. */
int32_t cbc_ensemble_solve(cbc_context* ctx, const cbc_spec* spec, const cbc_ensemble* ens,
                           const cbc_work* work, int64_t max_steps, void* stream);

/* The same batched solve, allocating nothing: no cudaMalloc / cudaFree and no
 * host heap on success.  It is for callers that must not allocate while they
 * step the ensemble: a training or control loop whose device memory is held
 * by another allocator (a PyTorch caching allocator that has reserved the
 * GPU, a fixed per-process memory budget), where a cudaMalloc would fail or
 * stall the whole device, or code that calls the solver from a place where
 * allocation is not allowed.  Their buffers (the cbc_ensemble arrays) are
 * theirs; the solver only needs 144 bytes of its own, which are built into
 * the library and held by every GPU that loads it until the process exits.
 * Its scheduling scratch (the work-list cursors and the time-slice epoch,
 * 144 bytes) is a static device array of the library.  Its device address is
 * looked up (cudaGetSymbolAddress) once per device by cbc_create, with that
 * device current, and kept for the life of the process: a process that
 * resets a device (cudaDeviceReset) must not call this entry point on that
 * device afterwards.  With CUDA's lazy module loading (the default), the
 * first launch of each bucket kernel on a device loads that kernel, which
 * may allocate driver memory: make one warm-up call per K bucket shape before
 * the region that must not allocate (or run with CUDA_MODULE_LOADING=EAGER).
 * The cursors are zeroed by each call on `stream` before its kernels.  Work
 * lists of more than CBC_MAX_BUCKETS (32) buckets are rejected with
 * CBC_E_INVALID.  The scratch is shared by all calls on a device: calls whose
 * executions overlap in time (different streams, no ordering between them)
 * race on it and must not be issued.  No counterpart in the reference. */
int32_t cbc_ensemble_solve_noalloc(cbc_context* ctx, const cbc_spec* spec, const cbc_ensemble* ens,
                                   const cbc_work* work, int64_t max_steps, void* stream);

/* Captures the same launch sequence into a CUDA graph bound to these buffers;
 * cbc_plan_launch replays it on `stream` (one graph launch per solve).  If
 * `stream` is itself being captured into a graph of the caller's (e.g. by
 * torch.cuda.graph), cbc_plan_launch adds the plan's graph as a child node of
 * that graph instead of launching it. */
int32_t cbc_plan_create(cbc_context* ctx, const cbc_spec* spec, const cbc_ensemble* ens,
                        const cbc_work* work, int64_t max_steps, cbc_plan** out);
int32_t cbc_plan_launch(cbc_plan* plan, void* stream);
int32_t cbc_plan_destroy(cbc_plan* plan);

/* ---- device-side admission (parameter precompute on the GPU) ---------------
 * Scalar constants of the precompute, evaluated on the host from the
 * material properties and the reference frequency f (Hz), exactly as
 * cbc_b200.models.ckm1d.precompute_constants does: two_pi = 2 pi,
 * w_ref = two_pi f, l_ref = c / f, st2 = 2 sigma, k1 = 1 - 3 gamma,
 * p0pv = P0 - Pv, k4 = 4 mu / rho, tw = two_pi / w_ref,
 * k6 = tw^2 / c / rho, hl = l_ref / 2, k9 = two_pi / rho, k10 = 2 two_pi / 3,
 * k11 = 6 two_pi mu, km2 = (18 mu / rho) tw, system_params the 5 per-system
 * constants (3 gamma, 1 / w_ref, l_ref / two_pi, c, 1 / rho / c), pi = pi. */
typedef struct cbc_precompute_consts {
  double two_pi, pi, w_ref, l_ref, rho, cl, p0, pv;
  double st2, k1, p0pv, k4, tw, k6, hl, k9, k10, k11, km2;
  double system_params[5];
} cbc_precompute_consts;

/* Doubles per request record of cbc_admit for nk harmonics:
 * [K, slot, bubble_offset, coupling_offset, span, PA[nk] (bar), FR[nk] (kHz),
 *  PS[nk] (phase / pi), R0[32] (um, first K used), X0[32] (positions in
 *  units of the reference wavelength, first K used)]. */
#define CBC_ADMIT_RECORD(nk) (5 + 3 * (nk) + 64)

/* Writes n raw requests (device array `records`, n * CBC_ADMIT_RECORD(nk)
 * doubles) into their slots of the ensemble: bubble_offset / coupling_offset
 * of the slot, the 13 bubble constants, the per-system and control
 * parameters, the 3 K x K coupling block, the initial state (R = 1, X = X0,
 * U = V = 0), t = 0, t_end = span, t_begin = 0, h = 1e-6, event = -1,
 * status 0 and zero counters.  One warp per request.  Bit-identical to the
 * host precompute (reference models/ckm1d.py:133-202, model.py:180-225),
 * which it replaces for served requests.  coupling_len: doubles in
 * ens->coupling; a record whose slot or ranges fall outside the ensemble is
 * skipped.  No reference counterpart on the GPU. */
int32_t cbc_admit(cbc_context* ctx, const cbc_ensemble* ens, const cbc_precompute_consts* consts,
                  const double* records, int32_t n, int32_t nk, int64_t coupling_len, void* stream);

/* ---- vec-env step ------------------------------------------------------------
 * Device buffers of one environment step around the batched solve (uniform K,
 * one system per environment, ns * K == nb).  Before the solve, for every env
 * s: control_params[s][a] = actions[s * act_stride + a] * act_scale for
 * a < n_act (the PA columns: bar -> Pa with act_scale 1e5), t = 0,
 * t_end = t_span, h = h0, event = -1, status = 0.  After the solve:
 * obs[s][0..K-1] = x, obs[s][K..2K-1] = R (float32), failed[s] = status != 1
 * (failed may be NULL).  Reference: PosNBC1D.step
 * (envs/bubble_1D_pos_control.py:503-538: set_action :732-749,
 * advance_time :816-826, check_termination :772-789, observe :756-769). */
typedef struct cbc_env_io {
  const float* actions;
  int32_t n_act;
  int32_t act_stride;
  double act_scale;
  float* obs;
  uint8_t* failed;
  int32_t K;
  int32_t pad;
  double t_span;
  double h0;
  /* ---- optional fused epilogue: reward, termination and resets ----------
   * Used when rewards != NULL (then every pointer below must be set).  After
   * the observation, for every env s (reference get_rewards :792-813,
   * check_termination :772-789, final_termination :830-853), in float32:
   *   td_i = |targets[s][i] - x_i|, success = all td_i <= tol,
   *   td_i = 0 where td_i < tol, dist = mean_i (td_i * r_dnorm)^reward_exp,
   *   intensity = sqrt(sum_a actions[s][a]^2),
   *   rewards[s] = -w_dist dist - w_intensity intensity + neg_reward failed
   *                + pos_reward success,
   *   total_rewards[s] += rewards[s], algo_steps[s] += 1,
   *   terminated[s] = failed | success, time_outs[s] = algo_steps >= episode_length.
   * A finished env (terminated or timed out) keeps final_obs[s] = its
   * observation, episode_return[s] / episode_len[s] its totals, and is reset
   * in place (reset_envs :583-614): new positions and targets from the scene
   * generator (reference SceneGenerator :183-242; uniform draws from a
   * counter-based hash of (seed, env, reset_count[s])), state R = 1, X = the
   * positions, U = V = 0, observation [positions, 1], totals 0,
   * reset_count[s] += 1.  done[s] = 1 marks the envs reset in this step. */
  float* targets;          /* (ns, K) */
  float* rewards;          /* (ns) */
  uint8_t* terminated;     /* (ns) */
  uint8_t* time_outs;      /* (ns) */
  uint8_t* done;           /* (ns) */
  int32_t* algo_steps;     /* (ns) */
  float* total_rewards;    /* (ns) */
  float* final_obs;        /* (ns, 2K) */
  float* episode_return;   /* (ns) */
  int32_t* episode_len;    /* (ns) */
  int64_t* reset_count;    /* (ns) */
  double position_tolerance, r_dnorm, reward_exp, w_dist, w_intensity, pos_reward, neg_reward;
  double min_distance, max_distance, domain_lo, domain_hi;   /* scene generator (margins applied) */
  int32_t episode_length;
  int32_t pad2;
  uint64_t seed;
} cbc_env_io;

/* Resets the envs s with mask[s] != 0 (every env when mask is NULL) exactly
 * as the fused epilogue resets a finished env (scene generator draws, state,
 * observation, totals, reset_count).  Needs the epilogue fields of io. */
int32_t cbc_env_reset(cbc_context* ctx, const cbc_ensemble* ens, const cbc_env_io* io, const uint8_t* mask,
                      void* stream);

/* A plan whose graph is env prologue -> batched solve -> env epilogue; one
 * cbc_plan_launch is one environment step for every env (io == NULL gives
 * the plain cbc_plan_create graph). */
int32_t cbc_env_plan_create(cbc_context* ctx, const cbc_spec* spec, const cbc_ensemble* ens,
                            const cbc_work* work, int64_t max_steps, const cbc_env_io* io,
                            cbc_plan** out);

#ifdef __cplusplus
}
#endif

#endif /* CBC_B200_H */
