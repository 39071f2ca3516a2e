// plain.cu -- reference-layout CKM1D integrator (the drop-in solver) and the
// context entry points of libcbc_b200.so.
//
// plain_kernel<KB> is the one-launch-per-K form: a static mapping of systems to
// warps (floor(32/K) systems per warp, one lane per bubble) over the caller's
// reference-layout buffers, advancing each system by at most `budget` steps.
// It replaces the fused kernel of the reference
// (backends/numba/rkck45_coupled_numba_stepper.py:116-706) and cbc_solve
// replaces the host launch loop (backends/numba/rkck45_coupled_numba_solver.py:29-91).
#include "cbc_internal.h"

namespace cbc {

struct RefLayout {
  int ns, ups, tile;
  double* actual_time;
  const double* time_end;
  const double* time_begin;
  double* time_step;
  double* actual_state;
  const double* unit_params;
  const double* system_params;
  const double* control_params;
  const double* coupling;
  int* dense_index;
  double* dense_time;
  double* dense_state;
  double* actual_event;
  int* status;
  int* total_steps;
  int* rejected_steps;
  int* conv_success;
  int* conv_failures;
  long long* lin_iters;
};

template <int KB>
__device__ __forceinline__ void ref_store_dense(const RefLayout& L, const LaneState& S, const Geo& g,
                                                long long s, int slot) {
  const long long NST = (long long)L.ns * L.tile;
  if (g.li == 0) L.dense_time[(long long)slot * L.ns + s] = S.t;
#pragma unroll
  for (int c = 0; c < 4; ++c) L.dense_state[((long long)slot * 4 + c) * NST + s * L.tile + g.li] = S.y[c];
}

template <int KB, int KC, int LIN>
__global__ void __launch_bounds__(128, min_blocks_for(KB)) plain_kernel(RefLayout L, Params P, long long budget, int final_launch,
                                                    int* active_counter) {
  extern __shared__ __align__(16) double smem[];
  const Geo g = make_geo(KC > 0 ? KC : L.ups);
  const WarpSmem W = warp_smem(smem, L.ups, P.nk, LIN);
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long s = warp * g.G + g.grp;
  const bool have = g.valid && s < L.ns;
  const long long NST = (long long)L.ns * L.tile;
  const long long lane_off = s * L.tile + g.li;

  LaneState S;
  MView M;
  M.m = L.coupling + (have ? lane_off : 0);
  M.sc = (long long)L.ups * NST;
  M.sj = NST;
  S.active = false;
  S.status = ST_ACTIVE;
  double g_store = 0.0;
  if (have) {
#pragma unroll
    for (int c = 0; c < 4; ++c) S.y[c] = L.actual_state[c * NST + lane_off];
    store_bubble_consts(W, g, L.unit_params + lane_off, NST);
    store_coupling(W, g, M);
    S.sp0 = L.system_params[0 * (long long)L.ns + s];
    S.sp3 = L.system_params[3 * (long long)L.ns + s];
    S.t = L.actual_time[s];
    S.t_end = L.time_end[s];
    S.t_begin = L.time_begin[s];
    S.h = L.time_step[s];
    S.idx = (P.ndo > 0) ? L.dense_index[s] : 0;
    g_store = L.actual_event[s];
    const double prev = (P.ndo > 0 && S.idx > 0) ? L.dense_time[(long long)(S.idx - 1) * L.ns + s] : 0.0;
    prologue(S, P, g_store, prev, L.status[s]);
    if (g.li == 0)
      store_harmonics(W, g, L.system_params[1 * (long long)L.ns + s], L.system_params[2 * (long long)L.ns + s],
                      L.system_params[4 * (long long)L.ns + s], L.control_params + s, P.nk, L.ns);
  }
  __syncwarp();

  // first dense sample and initial event value (stepper.py:333-358)
  if (S.active && P.ndo > 0) {
    bool st = false;
    if (P.dense_mode == 0) st = (S.idx < P.ndo) && (S.dnext <= S.t);
    else st = (S.idx < P.ndo) && (S.t >= grid_time(S, S.idx, P.ndo));
    if (st) {
      ref_store_dense<KB>(L, S, g, s, S.idx);
      S.idx += 1;
      if (P.dense_mode == 0) {
        const double nx = S.t + S.ddt;
        S.dnext = nx < S.t_end ? nx : S.t_end;
      }
    }
  }
  {
    const double g0 = group_event<KB>(S.y, upv(W, g, 12), g, P.col);
    if (S.active) S.g_old = g0;
  }

  for (long long it = 0; it < budget; ++it) {
    if (!__any_sync(FULL, S.active)) break;
    const bool st = step<KB, KC, LIN>(g, P, W, M, S);
    if (st) ref_store_dense<KB>(L, S, g, s, S.idx);
    after_store(S, P, st);
  }

  if (have) {
    if (S.status == ST_ACTIVE && final_launch) S.status = ST_MAX_STEPS;
#pragma unroll
    for (int c = 0; c < 4; ++c) L.actual_state[c * NST + lane_off] = S.y[c];
    if (g.li == 0) {
      L.actual_time[s] = S.t;
      L.time_step[s] = S.h;
      L.actual_event[s] = S.g_old;
      L.status[s] = S.status;
      if (P.ndo > 0) L.dense_index[s] = S.idx;
      if (L.total_steps) L.total_steps[s] += S.steps;
      if (L.rejected_steps) L.rejected_steps[s] += S.rejected;
      if (L.conv_success) L.conv_success[s] += S.conv_ok;
      if (L.conv_failures) L.conv_failures[s] += S.conv_fail;
      if (L.lin_iters) L.lin_iters[s] += S.lin_iters;
      if (S.status == ST_ACTIVE && active_counter) atomicAdd(active_counter, 1);
    }
  }
}

template <int KB, int KC, int LIN>
cudaError_t launch_plain(const RefLayout& L, const Params& P, long long budget, int final_launch, int* counter,
                         cudaStream_t stream) {
  const int G = 32 / L.ups;
  const long long warps = (L.ns + G - 1) / G;
  int dev = 0;
  cudaError_t de = cudaGetDevice(&dev);
  if (de != cudaSuccess) return de;
  int cap = 0;
  de = cudaDeviceGetAttribute(&cap, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (de != cudaSuccess) return de;
  const int threads = block_threads_for(L.ups, P.nk, LIN, (size_t)cap, 128);
  const long long blocks = (warps * 32 + threads - 1) / threads;
  const size_t shmem = sizeof(double) * (size_t)smem_doubles_per_warp(L.ups, P.nk, LIN) * (threads / 32);
  if (shmem > 48 * 1024) {
    cudaError_t e =
        cudaFuncSetAttribute(plain_kernel<KB, KC, LIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem);
    if (e != cudaSuccess) return e;
  }
  plain_kernel<KB, KC, LIN><<<(unsigned)blocks, threads, shmem, stream>>>(L, P, budget, final_launch, counter);
  return cudaGetLastError();
}

cudaError_t launch_plain_any(const RefLayout& L, const Params& P, long long budget, int final_launch,
                             int* counter, cudaStream_t stream) {
  return dispatch_k(L.ups, [&](auto kb, auto kc) {
    return dispatch_lin(P.lin, [&](auto lin) {
      return launch_plain<decltype(kb)::value, decltype(kc)::value, decltype(lin)::value>(L, P, budget,
                                                                                         final_launch, counter,
                                                                                         stream);
    });
  });
}

}  // namespace cbc

using namespace cbc;

extern "C" {

int32_t cbc_version(void) { return 100; }

int32_t cbc_create(cbc_context** out, int32_t device) {
  if (!out) return fail(nullptr, CBC_E_INVALID, "out is NULL");
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return fail(nullptr, CBC_E_CUDA, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
  if (device < 0 || device >= ndev) return fail(nullptr, CBC_E_INVALID, "device %d out of range (%d devices)", device, ndev);
  cbc_context* ctx = new (std::nothrow) cbc_context();
  if (!ctx) return fail(nullptr, CBC_E_NOMEM, "context allocation failed");
  ctx->device = device;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  e = cudaMalloc(&ctx->d_counter, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_head, kScheduleBytes);
  if (e == cudaSuccess) e = cudaMallocHost(&ctx->h_counter, sizeof(int));
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev1);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming);
  int prio_low = 0, prio_high = 0;
  if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  for (int i = 0; i < CBC_SIDE_STREAMS && e == cudaSuccess; ++i) {
    e = cudaEventCreateWithFlags(&ctx->join[i], cudaEventDisableTiming);
    // first half: higher priority (bucket start grids); second half: lowest
    // priority (backfill grids only take SMs no start grid is waiting for)
    const int prio = i < CBC_SIDE_STREAMS / 2 ? prio_high : prio_low;
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&ctx->side[i], cudaStreamNonBlocking, prio);
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->capture, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = noalloc_scratch_address(device, &ctx->noalloc_scratch);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    cbc_destroy(ctx);
    return fail(nullptr, CBC_E_CUDA, "context set-up failed: %s", cudaGetErrorString(e));
  }
  *out = ctx;
  return CBC_OK;
}

int32_t cbc_destroy(cbc_context* ctx) {
  if (!ctx) return CBC_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->device);
  if (ctx->d_counter) cudaFree(ctx->d_counter);
  if (ctx->d_head) cudaFree(ctx->d_head);
  if (ctx->h_counter) cudaFreeHost(ctx->h_counter);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->fork) cudaEventDestroy(ctx->fork);
  for (int i = 0; i < CBC_SIDE_STREAMS; ++i) {
    if (ctx->join[i]) cudaEventDestroy(ctx->join[i]);
    if (ctx->side[i]) cudaStreamDestroy(ctx->side[i]);
  }
  if (ctx->capture) cudaStreamDestroy(ctx->capture);
  cudaSetDevice(prev);
  delete ctx;
  return CBC_OK;
}

const char* cbc_last_error(const cbc_context* ctx) {
  if (ctx) return ctx->err.c_str();
  return global_error().c_str();
}

int32_t cbc_solve(cbc_context* ctx, const cbc_spec* spec, const cbc_buffers* b, int64_t max_steps,
                  int32_t kernel_steps, int32_t launch_mode, void* stream_, cbc_solve_stats* stats) {
  if (!ctx) return fail(nullptr, CBC_E_INVALID, "context is NULL");
  ctx->err.clear();
  int32_t rc = check_spec(ctx, spec);
  if (rc) return rc;
  if (!b) return fail(ctx, CBC_E_INVALID, "buffers is NULL");
  if (max_steps < 1 || kernel_steps < 1) return fail(ctx, CBC_E_INVALID, "max_steps and kernel_steps must be >= 1");
  if (launch_mode != CBC_LAUNCH_RELAUNCH && launch_mode != CBC_LAUNCH_SINGLE)
    return fail(ctx, CBC_E_INVALID, "unknown launch mode %d", launch_mode);
  if (!b->actual_time || !b->time_end || !b->time_begin || !b->time_step || !b->actual_state || !b->unit_params ||
      !b->system_params || !b->control_params || !b->coupling_matrices || !b->actual_event || !b->status_flags)
    return fail(ctx, CBC_E_INVALID, "a required buffer pointer is NULL");
  if (spec->ndo > 0 && (!b->dense_index || !b->dense_time || !b->dense_state))
    return fail(ctx, CBC_E_INVALID, "ndo > 0 needs dense_index, dense_time and dense_state");

  RefLayout L;
  L.ns = spec->ns;
  L.ups = spec->ups;
  L.tile = spec->tile;
  L.actual_time = b->actual_time;
  L.time_end = b->time_end;
  L.time_begin = b->time_begin;
  L.time_step = b->time_step;
  L.actual_state = b->actual_state;
  L.unit_params = b->unit_params;
  L.system_params = b->system_params;
  L.control_params = b->control_params;
  L.coupling = b->coupling_matrices;
  L.dense_index = b->dense_index;
  L.dense_time = b->dense_time;
  L.dense_state = b->dense_state;
  L.actual_event = b->actual_event;
  L.status = b->status_flags;
  L.total_steps = b->total_steps;
  L.rejected_steps = b->rejected_steps;
  L.conv_success = b->convergence_success;
  L.conv_failures = b->convergence_failures;
  L.lin_iters = (long long*)b->lin_iters;
  const Params P = make_params(*spec);
  cudaStream_t stream = (cudaStream_t)stream_;

  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != ctx->device) CBC_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  struct Restore {
    int d;
    ~Restore() { cudaSetDevice(d); }
  } restore{prev};

  const long long launches = (max_steps + kernel_steps - 1) / kernel_steps;
  int32_t n = 0;
  double dev_ms = 0.0;
  int32_t left = -1;
  if (launch_mode == CBC_LAUNCH_SINGLE) {
    CBC_CUDA_TRY(ctx, cudaEventRecord(ctx->ev0, stream));
    CBC_CUDA_TRY(ctx, launch_plain_any(L, P, launches * (long long)kernel_steps, 1, nullptr, stream));
    ++ctx->launches;
    CBC_CUDA_TRY(ctx, cudaEventRecord(ctx->ev1, stream));
    n = 1;
    if (stats) {
      CBC_CUDA_TRY(ctx, cudaEventSynchronize(ctx->ev1));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
      dev_ms = ms;
    }
  } else {
    // the reference host loop: launch, synchronise, stop when every system is done
    for (long long l = 0; l < launches; ++l) {
      const int final_launch = (l + 1 == launches);
      CBC_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_counter, 0, sizeof(int), stream));
      CBC_CUDA_TRY(ctx, cudaEventRecord(ctx->ev0, stream));
      CBC_CUDA_TRY(ctx, launch_plain_any(L, P, kernel_steps, final_launch, ctx->d_counter, stream));
      ++ctx->launches;
      CBC_CUDA_TRY(ctx, cudaEventRecord(ctx->ev1, stream));
      CBC_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_counter, ctx->d_counter, sizeof(int), cudaMemcpyDeviceToHost, stream));
      CBC_CUDA_TRY(ctx, cudaStreamSynchronize(stream));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
      dev_ms += ms;
      ++n;
      left = *ctx->h_counter;
      if (left == 0) break;
    }
  }
  if (stats) {
    stats->launches = n;
    stats->active_left = left;
    stats->device_ms = dev_ms;
  }
  return CBC_OK;
}

}  // extern "C"
