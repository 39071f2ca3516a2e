// vecenv.cu -- device-side prologue/epilogue of one vec-env step, fused into
// the batched solve's CUDA graph.
//
// Replaces, for the physics part of an environment step of the reference
// PosNBC1D (envs/bubble_1D_pos_control.py:503-538):
//   set_action   (:732-749)  actions -> control parameters (index_copy_ via torch)
//   advance_time (:816-826)  actual_time = 0, time_step = 1e-6, actual_event = -1
//   check_termination (:772-789) status_flags != 1 -> failure, then zero_()
//   observe      (:756-769)  positions (and radii) -> float32 observation
// Each of those is a separate torch op (plus the solver's host loop) in the
// reference; here they are two small kernels captured around the solve, so an
// env step is one graph launch and the observation lands in a caller-owned
// float32 tensor without a copy.
#include <new>
#include <vector>

#include "cbc_internal.h"
#include "ensemble.h"

namespace cbc {

// One thread per environment (system).
__global__ void env_begin_kernel(int ns, const float* __restrict__ actions, int n_act, int act_stride,
                                 double act_scale, double* control, int cp_stride, double* t, double* t_end,
                                 double* h, double* event, int* status, double t_span, double h0) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  for (int a = 0; a < n_act; ++a)
    control[(long long)s * cp_stride + a] = (double)actions[(long long)s * act_stride + a] * act_scale;
  t[s] = 0.0;
  t_end[s] = t_span;
  h[s] = h0;
  event[s] = -1.0;
  status[s] = 0;
}

// One thread per bubble: obs[s][i] = x_i, obs[s][K + i] = R_i (float32),
// failed[s] = status != SUCCESS (written by the first bubble of each system).
__global__ void env_end_kernel(int ns, long long nb, const long long* __restrict__ bubble_offset,
                               const double* __restrict__ state, const int* __restrict__ status, int K,
                               float* obs, unsigned char* failed) {
  const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= (long long)ns * K) return;
  const int s = (int)(b / K);
  const int i = (int)(b - (long long)s * K);
  const long long row = bubble_offset[s] + i;
  if (row >= nb) return;
  const double2 rx = reinterpret_cast<const double2*>(state + row * 4)[0];
  obs[(long long)s * 2 * K + i] = (float)rx.y;
  obs[(long long)s * 2 * K + K + i] = (float)rx.x;
  if (i == 0 && failed) failed[s] = (status[s] != ST_SUCCESS) ? 1 : 0;
}

}  // namespace cbc

namespace cbc {

int32_t enqueue_env_begin(cbc_context* ctx, const cbc_ensemble* e, const cbc_env_io* io, cudaStream_t st) {
  const int threads = 128;
  const int blocks = (e->ns + threads - 1) / threads;
  ++ctx->launches;
  env_begin_kernel<<<blocks, threads, 0, st>>>(e->ns, io->actions, io->n_act, io->act_stride, io->act_scale,
                                                e->control_params, e->cp_stride, e->t,
                                                e->t_end, e->h, e->event, e->status,
                                                io->t_span, io->h0);
  CBC_CUDA_TRY(ctx, cudaGetLastError());
  return CBC_OK;
}

int32_t enqueue_env_end(cbc_context* ctx, const cbc_ensemble* e, const cbc_env_io* io, cudaStream_t st) {
  const int threads = 128;
  const long long n = (long long)e->ns * io->K;
  const int blocks = (int)((n + threads - 1) / threads);
  ++ctx->launches;
  env_end_kernel<<<blocks, threads, 0, st>>>(e->ns, e->nb, (const long long*)e->bubble_offset, e->state,
                                              e->status, io->K, io->obs, io->failed);
  CBC_CUDA_TRY(ctx, cudaGetLastError());
  return CBC_OK;
}

}  // namespace cbc
