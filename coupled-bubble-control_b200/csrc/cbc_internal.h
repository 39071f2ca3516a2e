// cbc_internal.h -- host-side helpers shared by the translation units of
// libcbc_b200.so (context, error reporting, parameter conversion).
#pragma once

#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <mutex>
#include <string>

#include "../../include/cbc_b200.h"

#include <type_traits>
#include "ckm1d_core.cuh"

#define CBC_MAX_BUCKETS 32   // two launches per bucket fit CBC_SIDE_STREAMS
#define CBC_SIDE_STREAMS 64

struct cbc_context {
  int device = 0;
  int sm_count = 0;
  int* d_counter = nullptr;       // device: systems still active after a launch
  int* h_counter = nullptr;       // pinned host mirror
  int* d_head = nullptr;          // device: work-list cursors of cbc_ensemble_solve
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[CBC_SIDE_STREAMS] = {};
  cudaStream_t side[CBC_SIDE_STREAMS] = {};
  cudaStream_t capture = nullptr;  // stream used to capture plans into graphs
  long long launches = 0;          // kernels enqueued (plans: per replay)
  void* noalloc_scratch = nullptr; // device address of the static scratch of cbc_ensemble_solve_noalloc
  std::string err;
};

namespace cbc {

// Makes `device` current for the lifetime of the guard, restoring the
// caller's device afterwards.
struct DeviceGuard {
  int prev = 0;
  explicit DeviceGuard(int device) {
    cudaGetDevice(&prev);
    if (prev != device) cudaSetDevice(device);
  }
  ~DeviceGuard() { cudaSetDevice(prev); }
};

// Message store for failures that happen without a context.
inline std::string& global_error() {
  static std::string s;
  return s;
}
inline std::mutex& global_error_mutex() {
  static std::mutex m;
  return m;
}

inline int32_t fail(cbc_context* ctx, int32_t code, const char* fmt, ...) __attribute__((format(printf, 3, 4)));
inline int32_t fail(cbc_context* ctx, int32_t code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  else {
    std::lock_guard<std::mutex> lk(global_error_mutex());
    global_error() = buf;
  }
  return code;
}

#define CBC_CUDA_TRY(ctx, call)                                                              \
  do {                                                                                       \
    cudaError_t e__ = (call);                                                                \
    if (e__ != cudaSuccess)                                                                  \
      return ::cbc::fail((ctx), CBC_E_CUDA, "%s failed: %s", #call, cudaGetErrorString(e__)); \
  } while (0)

inline Params make_params(const cbc_spec& s) {
  Params p;
  p.atol = s.atol;
  p.rtol = s.rtol;
  p.min_step = s.min_step;
  p.max_step = s.max_step;
  p.lin_atol2 = s.lin_atol * s.lin_atol;
  p.lin_rtol2 = s.lin_rtol * s.lin_rtol;
  p.omega = s.lin_relaxation;
  p.etol = s.etol;
  p.col = 1.0 + s.col_threshold;
  p.lin_max_iter = s.lin_max_iter;
  p.ndo = s.ndo;
  p.dense_mode = s.dense_mode;
  p.nk = s.nk;
  p.ac = s.ac;
  p.lin = s.lin_solver;
  return p;
}

inline int32_t check_spec(cbc_context* ctx, const cbc_spec* s) {
  if (!s) return fail(ctx, CBC_E_INVALID, "spec is NULL");
  if (s->ns < 1) return fail(ctx, CBC_E_INVALID, "ns must be >= 1 (got %d)", s->ns);
  if (s->ups < 1) return fail(ctx, CBC_E_INVALID, "ups must be >= 1 (got %d)", s->ups);
  if (s->ups > 32) return fail(ctx, CBC_E_UNSUPPORTED, "ups = %d: at most 32 bubbles per system", s->ups);
  if (s->tile < s->ups) return fail(ctx, CBC_E_INVALID, "tile (%d) < ups (%d)", s->tile, s->ups);
  if (s->nk < 1 || s->nk > NKMAX)
    return fail(ctx, CBC_E_UNSUPPORTED, "nk = %d: 1..%d harmonic components supported", s->nk, NKMAX);
  if (s->ac < 0 || s->ac > 2) return fail(ctx, CBC_E_INVALID, "ac = %d: expected 0 CONST, 1 SW_N, 2 SW_A", s->ac);
  if (s->ndo < 0) return fail(ctx, CBC_E_INVALID, "ndo must be >= 0");
  if (s->dense_mode < 0 || s->dense_mode > 1) return fail(ctx, CBC_E_INVALID, "dense_mode must be 0 or 1");
  if (s->lin_max_iter < 0) return fail(ctx, CBC_E_INVALID, "lin_max_iter must be >= 0");
  if (s->lin_solver != CBC_LIN_RICHARDSON && s->lin_solver != CBC_LIN_LU)
    return fail(ctx, CBC_E_INVALID, "lin_solver = %d: expected 0 (Richardson) or 1 (direct)", s->lin_solver);
  if (!(s->min_step > 0.0) || !(s->max_step >= s->min_step))
    return fail(ctx, CBC_E_INVALID, "need 0 < min_step <= max_step");
  if (!(s->atol > 0.0) || !(s->rtol >= 0.0)) return fail(ctx, CBC_E_INVALID, "need atol > 0, rtol >= 0");
  return CBC_OK;
}

// Scheduling scratch of one batched solve: the work-list cursors (one int per
// bucket) followed by the epoch word (device clock at the solve's start).
constexpr size_t kHeadBytes = sizeof(int) * CBC_MAX_BUCKETS;
constexpr size_t kScheduleBytes = kHeadBytes + 2 * sizeof(long long);

// Device address of the static scheduling scratch of
// cbc_ensemble_solve_noalloc on `device` (which must be current); looked up
// once per device.  *out stays NULL for device ordinals beyond its table.
cudaError_t noalloc_scratch_address(int device, void** out);

// Threads per block for a kernel of K bubbles per system: `requested`, cut
// to whole warps whose shared memory fits the device's per-block limit
// (K = 32 with its partner coefficients or augmented rows in shared memory
// needs ~67 KB per warp, so at most three warps per block).
inline int block_threads_for(int K, int nk, int lin, size_t max_block_smem, int requested) {
  const size_t per_warp = sizeof(double) * (size_t)smem_doubles_per_warp(K, nk, lin);
  int warps = requested / 32;
  if (per_warp > 0 && (size_t)warps * per_warp > max_block_smem) warps = (int)(max_block_smem / per_warp);
  if (warps < 1) warps = 1;
  return warps * 32;
}

// Smallest power-of-two instantiation that holds K bubbles per system.
inline int kb_for(int K) {
  if (K <= 2) return 2;
  if (K <= 4) return 4;
  if (K <= 8) return 8;
  if (K <= 16) return 16;
  return 32;
}

// Calls f(KB, KC) with std::integral_constant arguments: KB the power-of-two
// lanes per system slot, KC the exact K when it is compiled in (K <= 8: the
// group geometry, partner loops and reductions fold to constants), else 0
// (K read at run time).
template <int V>
using IC = std::integral_constant<int, V>;

// Calls f(IC<LIN>) for the implicit-coupling solver of a launch.
template <class F>
decltype(auto) dispatch_lin(int lin, F&& f) {
  if (lin == LIN_LU) return f(IC<LIN_LU>{});
  return f(IC<LIN_RICHARDSON>{});
}

// Calls f(IC<MB>) for the register-budget variant of a batched launch.
template <class F>
decltype(auto) dispatch_mb(int mb, F&& f) {
  if (mb == 1) return f(IC<1>{});
  return f(IC<0>{});
}

template <class F>
decltype(auto) dispatch_k(int K, F&& f) {
  switch (K) {
    case 1: return f(IC<2>{}, IC<1>{});
    case 2: return f(IC<2>{}, IC<2>{});
    case 3: return f(IC<4>{}, IC<3>{});
    case 4: return f(IC<4>{}, IC<4>{});
    case 5: return f(IC<8>{}, IC<5>{});
    case 6: return f(IC<8>{}, IC<6>{});
    case 7: return f(IC<8>{}, IC<7>{});
    case 8: return f(IC<8>{}, IC<8>{});
    case 16: return f(IC<16>{}, IC<16>{});
    case 32: return f(IC<32>{}, IC<32>{});
    default:
      if (K <= 16) return f(IC<16>{}, IC<0>{});
      return f(IC<32>{}, IC<0>{});
  }
}

}  // namespace cbc
