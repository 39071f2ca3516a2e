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
} cbc_spec;

/* Device buffers in the reference layout (models/model.py:56-106,
 * models/buffers.py:314-356), mutated in place.  Shapes, row-major:
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

#ifdef __cplusplus
}
#endif

#endif /* CBC_B200_H */
