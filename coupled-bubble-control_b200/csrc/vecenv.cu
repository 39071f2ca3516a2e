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

// ---- fused epilogue: reward, termination, resets ---------------------------

// SplitMix64 finaliser (Steele, Lea and Flood, "Fast splittable pseudorandom
// number generators", OOPSLA 2014): the counter-based uniform draws of the
// scene generator.
__host__ __device__ inline unsigned long long splitmix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Uniform [0, 1) draw j of stream `which` (0 positions, 1 targets) for the
// count-th reset of env s.
__device__ inline double env_uniform(unsigned long long seed, long long s, long long count, int which, int j) {
  const unsigned long long key = seed ^ ((unsigned long long)s * 0xD1B54A32D192ED03ull) ^
                                 ((unsigned long long)count * 0xABC98388FB8FAC03ull) ^
                                 ((unsigned long long)(which * 64 + j) * 0x8CB92BA72F3D8DD7ull);
  return (double)(splitmix64(key) >> 11) * (1.0 / 9007199254740992.0);
}

// A random chain of K bubbles (reference SceneGenerator, 'random' positions,
// 'center' alignment, envs/bubble_1D_pos_control.py:183-242): K - 1 gaps of
// min_distance plus uniform extras up to (max - min), scaled down to fit the
// domain, the chain centred in it.
__device__ inline void env_positions(const cbc_env_io& io, long long s, long long count, int which, int K,
                                     double* out) {
  const double lo = io.domain_lo, hi = io.domain_hi;
  if (K == 1) {
    out[0] = 0.5 * (lo + hi);
    return;
  }
  const int gn = K - 1;
  const double avail = hi - lo;
  const double room = io.max_distance - io.min_distance;
  const double limit = avail - gn * io.min_distance;
  double ext[32];
  double ssum = 0.0;
  for (int j = 0; j < gn; ++j) {
    ext[j] = env_uniform(io.seed, s, count, which, j) * room;
    ssum = ssum + ext[j];
  }
  double sc = limit / (ssum > 1e-12 ? ssum : 1e-12);
  sc = sc < 1.0 ? sc : 1.0;
  double gsum = 0.0;
  for (int j = 0; j < gn; ++j) {
    ext[j] = ext[j] * sc + io.min_distance;
    gsum = gsum + ext[j];
  }
  out[0] = lo + 0.5 * (avail - gsum);
  for (int j = 0; j < gn; ++j) out[j + 1] = out[j] + ext[j];
}

__device__ inline void env_reset_one(const cbc_ensemble& e, const cbc_env_io& io, long long s) {
  const int K = io.K;
  const long long count = io.reset_count[s];
  double pos[32], tgt[32];
  env_positions(io, s, count, 0, K, pos);
  env_positions(io, s, count, 1, K, tgt);
  const long long row = e.bubble_offset[s];
  for (int i = 0; i < K; ++i) {
    double* st = e.state + (row + i) * 4;
    st[0] = 1.0;
    st[1] = pos[i];
    st[2] = 0.0;
    st[3] = 0.0;
    io.targets[s * K + i] = (float)tgt[i];
    io.obs[s * 2 * K + i] = (float)pos[i];
    io.obs[s * 2 * K + K + i] = 1.0f;
  }
  io.algo_steps[s] = 0;
  io.total_rewards[s] = 0.0f;
  io.reset_count[s] = count + 1;
}

// One thread per env: observation, reward, termination, and the reset of
// the envs that finished.
__global__ void env_epilogue_kernel(cbc_ensemble e, cbc_env_io io) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= e.ns) return;
  const int K = io.K;
  const long long row = e.bubble_offset[s];
  float* ob = io.obs + s * 2 * K;
  for (int i = 0; i < K; ++i) {
    const double2 rx = reinterpret_cast<const double2*>(e.state + (row + i) * 4)[0];
    ob[i] = (float)rx.y;
    ob[K + i] = (float)rx.x;
  }
  const bool fail = e.status[s] != ST_SUCCESS;
  if (io.failed) io.failed[s] = fail ? 1 : 0;
  const float tol = (float)io.position_tolerance;
  const float rdn = (float)io.r_dnorm;
  const float ex = (float)io.reward_exp;
  bool success = true;
  float dsum = 0.0f;
  for (int i = 0; i < K; ++i) {
    float td = fabsf(io.targets[s * K + i] - ob[i]);
    success = success && (td <= tol);
    td = (td < tol) ? 0.0f : td;
    float v = td * rdn;
    v = v > 0.0f ? v : 0.0f;
    dsum = dsum + (ex == 0.5f ? sqrtf(v) : powf(v, ex));
  }
  const float dist = dsum / (float)K;
  float a2 = 0.0f;
  for (int a = 0; a < io.n_act; ++a) {
    const float av = io.actions[s * io.act_stride + a];
    a2 = a2 + av * av;
  }
  const float intensity = sqrtf(a2);
  const float r = -(float)io.w_dist * dist - (float)io.w_intensity * intensity +
                  (float)io.neg_reward * (fail ? 1.0f : 0.0f) + (float)io.pos_reward * (success ? 1.0f : 0.0f);
  io.rewards[s] = r;
  const float tot = io.total_rewards[s] + r;
  const int steps = io.algo_steps[s] + 1;
  io.total_rewards[s] = tot;
  io.algo_steps[s] = steps;
  const bool term = fail || success;
  const bool tout = steps >= io.episode_length;
  io.terminated[s] = term ? 1 : 0;
  io.time_outs[s] = tout ? 1 : 0;
  const bool done = term || tout;
  io.done[s] = done ? 1 : 0;
  if (!done) return;
  for (int i = 0; i < 2 * K; ++i) io.final_obs[s * 2 * K + i] = ob[i];
  io.episode_return[s] = tot;
  io.episode_len[s] = steps;
  env_reset_one(e, io, s);
}

__global__ void env_reset_kernel(cbc_ensemble e, cbc_env_io io, const unsigned char* mask) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= e.ns) return;
  if (mask && !mask[s]) return;
  env_reset_one(e, io, s);
}

bool env_epilogue_fields_ok(const cbc_env_io* io) {
  return io->targets && io->rewards && io->terminated && io->time_outs && io->done && io->algo_steps &&
         io->total_rewards && io->final_obs && io->episode_return && io->episode_len && io->reset_count &&
         io->episode_length >= 1 && io->K >= 1 && io->K <= 32 && io->domain_hi > io->domain_lo;
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
  if (io->rewards) {
    const int threads = 128;
    const int blocks = (e->ns + threads - 1) / threads;
    ++ctx->launches;
    env_epilogue_kernel<<<blocks, threads, 0, st>>>(*e, *io);
    CBC_CUDA_TRY(ctx, cudaGetLastError());
    return CBC_OK;
  }
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

using namespace cbc;

extern "C" int32_t cbc_env_reset(cbc_context* ctx, const cbc_ensemble* e, const cbc_env_io* io,
                                 const uint8_t* mask, void* stream) {
  if (!ctx) return fail(nullptr, CBC_E_INVALID, "context is NULL");
  ctx->err.clear();
  if (!e || !io || !e->bubble_offset || !e->state || !io->obs || !env_epilogue_fields_ok(io))
    return fail(ctx, CBC_E_INVALID, "env reset needs the ensemble and every epilogue field of io");
  if ((long long)io->K * e->ns != e->nb) return fail(ctx, CBC_E_INVALID, "env io: ns * K must equal nb");
  DeviceGuard dg(ctx->device);
  const int threads = 128;
  const int blocks = (e->ns + threads - 1) / threads;
  ++ctx->launches;
  env_reset_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(*e, *io, mask);
  CBC_CUDA_TRY(ctx, cudaGetLastError());
  return CBC_OK;
}
