// capi_ensemble.cu -- C ABI of the batched mixed-K form: direct solve and
// CUDA-graph plans.  See ensemble.cu for the device side.
#include <mutex>
#include <new>
#include <vector>

#include "cbc_internal.h"
#include "ensemble.h"

struct cbc_plan {
  cbc_context* ctx = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int* d_head = nullptr;  // one work-list cursor per bucket, then the epoch word (kScheduleBytes)
  int nbuckets = 0;
  long long kernels = 0;  // kernels in the captured graph
};

namespace cbc {

int32_t enqueue_env_begin(cbc_context* ctx, const cbc_ensemble* e, const cbc_env_io* io, cudaStream_t st);
int32_t enqueue_env_end(cbc_context* ctx, const cbc_ensemble* e, const cbc_env_io* io, cudaStream_t st);
bool env_epilogue_fields_ok(const cbc_env_io* io);

static int32_t check_ensemble(cbc_context* ctx, const cbc_spec* spec, const cbc_ensemble* e, const cbc_work* w) {
  if (!spec) return fail(ctx, CBC_E_INVALID, "spec is NULL");
  if (spec->nk < 1 || spec->nk > NKMAX)
    return fail(ctx, CBC_E_UNSUPPORTED, "nk = %d: 1..%d harmonic components supported", spec->nk, NKMAX);
  if (spec->ac < 0 || spec->ac > 2) return fail(ctx, CBC_E_INVALID, "ac = %d out of range", spec->ac);
  if (spec->ndo < 0 || spec->dense_mode < 0 || spec->dense_mode > 1 || spec->lin_max_iter < 0)
    return fail(ctx, CBC_E_INVALID, "ndo, dense_mode or lin_max_iter out of range");
  if (spec->lin_solver != CBC_LIN_RICHARDSON && spec->lin_solver != CBC_LIN_LU)
    return fail(ctx, CBC_E_INVALID, "lin_solver = %d: expected 0 (Richardson) or 1 (direct)", spec->lin_solver);
  if (!(spec->min_step > 0.0) || !(spec->max_step >= spec->min_step) || !(spec->atol > 0.0))
    return fail(ctx, CBC_E_INVALID, "need 0 < min_step <= max_step and atol > 0");
  if (!e || !w) return fail(ctx, CBC_E_INVALID, "ensemble or work list is NULL");
  if (e->ns < 1 || e->nb < 1) return fail(ctx, CBC_E_INVALID, "empty ensemble");
  if (!e->bubble_offset || !e->coupling_offset || !e->state || !e->unit_params || !e->system_params ||
      !e->control_params || !e->coupling || !e->t || !e->t_end || !e->t_begin || !e->h || !e->event || !e->status)
    return fail(ctx, CBC_E_INVALID, "a required ensemble pointer is NULL");
  if (spec->ndo > 0 && (!e->dense_index || !e->dense_time || !e->dense_state))
    return fail(ctx, CBC_E_INVALID, "ndo > 0 needs dense_index, dense_time and dense_state");
  if (e->up_stride < 13 || e->sp_stride < 5 || e->cp_stride < 4 * spec->nk)
    return fail(ctx, CBC_E_INVALID, "parameter row strides too small (need >= 13, 5, 4 nk)");
  if (((uintptr_t)e->state & 15) || (spec->ndo > 0 && ((uintptr_t)e->dense_state & 15)))
    return fail(ctx, CBC_E_INVALID, "state and dense_state must be 16-byte aligned");
  if (!w->order || w->nbuckets < 1 || w->nbuckets > CBC_MAX_BUCKETS || !w->bucket_K || !w->bucket_begin)
    return fail(ctx, CBC_E_INVALID, "work list needs 1..%d buckets", CBC_MAX_BUCKETS);
  for (int b = 0; b < w->nbuckets; ++b) {
    const int K = w->bucket_K[b];
    if (K < 1 || K > 32) return fail(ctx, CBC_E_UNSUPPORTED, "bucket %d: K = %d (1..32 supported)", b, K);
    if (w->bucket_begin[b] < 0 || w->bucket_begin[b + 1] < w->bucket_begin[b])
      return fail(ctx, CBC_E_INVALID, "bucket %d: bad range", b);
    if (w->threads && (w->threads[b] < 32 || w->threads[b] > 128 || (w->threads[b] & 31)))
      return fail(ctx, CBC_E_INVALID, "bucket %d: threads per block must be 32..128, a multiple of 32", b);
    if (w->exclusive && w->exclusive[b] < 0)
      return fail(ctx, CBC_E_INVALID, "bucket %d: exclusive must be >= 0", b);
    if (w->slots && (w->slots[b] < 1 || w->slots[b] > 32 / K))
      return fail(ctx, CBC_E_INVALID, "bucket %d: slots = %d, need 1..%d for K = %d", b, w->slots[b], 32 / K, K);
    if (w->min_blocks && (w->min_blocks[b] < 0 || w->min_blocks[b] > 1))
      return fail(ctx, CBC_E_INVALID, "bucket %d: min_blocks variant must be 0 or 1", b);
  }
  if (w->budget_ns < 0) return fail(ctx, CBC_E_INVALID, "budget_ns must be >= 0");
  if (w->steps_total != 0 && w->steps_total != 1) return fail(ctx, CBC_E_INVALID, "steps_total must be 0 or 1");
  if (w->steps_total && !e->steps) return fail(ctx, CBC_E_INVALID, "steps_total needs ensemble.steps");
  return CBC_OK;
}

static EnsLayout make_layout(const cbc_ensemble* e) {
  EnsLayout E;
  E.ns = e->ns;
  E.nb = e->nb;
  E.bubble_offset = (const long long*)e->bubble_offset;
  E.coupling_offset = (const long long*)e->coupling_offset;
  E.state = e->state;
  E.unit_params = e->unit_params;
  E.system_params = e->system_params;
  E.control_params = e->control_params;
  E.coupling = e->coupling;
  E.t = e->t;
  E.t_end = e->t_end;
  E.t_begin = e->t_begin;
  E.h = e->h;
  E.event = e->event;
  E.status = e->status;
  E.dense_index = e->dense_index;
  E.dense_time = e->dense_time;
  E.dense_state = e->dense_state;
  E.steps = e->steps;
  E.rejected = e->rejected;
  E.conv_ok = e->conv_ok;
  E.conv_fail = e->conv_fail;
  E.lin_iters = (long long*)e->lin_iters;
  E.trace_load_ns = (long long*)e->trace_load_ns;
  E.trace_done_ns = (long long*)e->trace_done_ns;
  E.up_stride = e->up_stride;
  E.sp_stride = e->sp_stride;
  E.cp_stride = e->cp_stride;
  return E;
}

// Persistent grid sizes per bucket, computed before any capture.  first[b]
// blocks start with the launch; second[b] more are launched behind every
// bucket's first grid (backfill).  A full-GPU grid is the resident blocks per
// SM (occupancy, or the work list's smaller override) times the SM count; no
// bucket gets more warps than it has systems to fill.
// Default block size of the batched kernels.  Four warps: with all K
// buckets resident at once, 128-thread blocks gave 1.8x the useful work per
// second of 64-thread blocks on the mixed-K workload (B200, measured).
constexpr int kDefaultThreads = 128;
constexpr float kStartFill = 0.85f;

constexpr int kExclusiveThreads = 128;

// Per-bucket launch parameters.  The storage is a template parameter so that
// the allocation-free entry point can use fixed arrays (FixedVec) while the
// others keep std::vector.
template <class T>
using HeapVec = std::vector<T>;

template <class T>
struct FixedVec {
  T v[CBC_MAX_BUCKETS];
  void assign(size_t n, T x) {
    for (size_t i = 0; i < n && i < CBC_MAX_BUCKETS; ++i) v[i] = x;
  }
  T& operator[](size_t i) { return v[i]; }
  const T& operator[](size_t i) const { return v[i]; }
};

template <template <class> class V>
struct GridsT {
  V<int> first, second, threads;
  V<size_t> smem;      // dynamic shared memory request (0: what the kernel needs)
  V<char> exclusive;
  V<int> slots, mb;    // systems per warp, register-budget variant
};
using Grids = GridsT<HeapVec>;

static bool is_exclusive(const cbc_work* w, int b) {
  return w->exclusive && w->exclusive[b] > 0 && w->bucket_begin[b + 1] > w->bucket_begin[b];
}

template <class G = Grids>
static G grid_sizes(cbc_context* ctx, const cbc_spec* spec, const cbc_work* w) {
  G g;
  g.first.assign(w->nbuckets, 0);
  g.second.assign(w->nbuckets, 0);
  g.threads.assign(w->nbuckets, kDefaultThreads);
  g.smem.assign(w->nbuckets, 0);
  g.exclusive.assign(w->nbuckets, 0);
  g.slots.assign(w->nbuckets, 32);
  g.mb.assign(w->nbuckets, 0);
  for (int b = 0; b < w->nbuckets; ++b) {
    if (w->slots) g.slots[b] = w->slots[b];
    if (w->min_blocks && w->bucket_K[b] <= 8) g.mb[b] = w->min_blocks[b];
  }
  // latency lanes first: one block per SM each
  int excl_sms = 0;
  for (int b = 0; b < w->nbuckets; ++b) {
    if (!is_exclusive(w, b)) continue;
    int n = w->exclusive[b];
    if (excl_sms + n > ctx->sm_count / 2) n = ctx->sm_count / 2 - excl_sms;
    if (n < 1) continue;
    g.exclusive[b] = 1;
    g.first[b] = n;
    g.threads[b] = block_threads_for(w->bucket_K[b], spec->nk, spec->lin_solver, max_block_smem(ctx->device),
                                     kExclusiveThreads);
    g.smem[b] = max_block_smem(ctx->device);
    excl_sms += n;
  }
  const float rest = 1.f - (float)excl_sms / (float)ctx->sm_count;
  for (int b = 0; b < w->nbuckets; ++b) {
    const int begin = w->bucket_begin[b], end = w->bucket_begin[b + 1];
    if (end <= begin || g.exclusive[b]) continue;
    const int K = w->bucket_K[b];
    const int threads = block_threads_for(K, spec->nk, spec->lin_solver, max_block_smem(ctx->device),
                                          w->threads ? w->threads[b] : kDefaultThreads);
    g.threads[b] = threads;
    const int per_sm = resident_blocks(K, spec->nk, threads, spec->lin_solver, g.mb[b]);
    int full = (int)((float)(per_sm * ctx->sm_count) * rest);
    if (full < 1) full = 1;
    if (w->blocks_per_sm && w->blocks_per_sm[b] > 0 && w->blocks_per_sm[b] < per_sm)
      full = (int)((float)(w->blocks_per_sm[b] * ctx->sm_count) * rest);
    if (full < 1) full = 1;
    const int per_warp = (32 / K < g.slots[b]) ? 32 / K : g.slots[b];
    const long long warps_needed = ((long long)(end - begin) + per_warp - 1) / per_warp;
    const long long blocks_needed = (warps_needed * 32 + threads - 1) / threads;
    if (full > blocks_needed) full = (int)blocks_needed;
    if (w->share) {
      float sh = w->share[b];
      if (!(sh > 0.f)) sh = 0.f;
      if (sh > 1.f) sh = 1.f;
      // blocks of different buckets pack imperfectly on an SM: start grids
      // use at most kStartFill of the GPU so that every bucket's fits at once
      int f = (int)(sh * kStartFill * (float)full + 0.5f);
      if (f < 1) f = 1;
      if (f > full) f = full;
      g.first[b] = f;
      g.second[b] = full - f;
    } else {
      g.first[b] = full;
    }
  }
  return g;
}

// Enqueues the whole batched solve on `stream`: every bucket on its own
// forked stream (ctx->side[b]), joined back into `stream`.
template <class G>
static int32_t enqueue(cbc_context* ctx, const cbc_spec* spec, const cbc_ensemble* e, const cbc_work* w,
                       const G& grids, int64_t max_steps, int* d_head, cudaStream_t stream) {
  const EnsLayout E = make_layout(e);
  const Params P = make_params(*spec);
  CBC_CUDA_TRY(ctx, cudaMemsetAsync(d_head, 0, sizeof(int) * w->nbuckets, stream));
  long long* epoch = reinterpret_cast<long long*>(reinterpret_cast<char*>(d_head) + kHeadBytes);
  if (w->budget_ns > 0) {
    CBC_CUDA_TRY(ctx, launch_stamp(epoch, stream));
    ++ctx->launches;
  }
  CBC_CUDA_TRY(ctx, cudaEventRecord(ctx->fork, stream));
  int used_first = 0, used_second = 0;
  // pass 0: the latency lanes (exclusive SMs), then every other bucket's
  // first grid; pass 1: the backfill grids, launched after all first grids so
  // that they only take SMs other buckets release
  for (int pass = 0; pass < 3; ++pass) {
    for (int b = 0; b < w->nbuckets; ++b) {
      const int begin = w->bucket_begin[b], end = w->bucket_begin[b + 1];
      if (end <= begin) continue;
      if ((pass == 0) != (grids.exclusive[b] != 0)) continue;
      const int blocks = pass < 2 ? grids.first[b] : grids.second[b];
      if (blocks <= 0) continue;
      const int slot = pass < 2 ? used_first : CBC_SIDE_STREAMS / 2 + used_second;
      if (slot >= (pass < 2 ? CBC_SIDE_STREAMS / 2 : CBC_SIDE_STREAMS))
        return fail(ctx, CBC_E_UNSUPPORTED, "too many bucket launches");
      const int K = w->bucket_K[b];
      cudaStream_t s = ctx->side[slot];
      CBC_CUDA_TRY(ctx, cudaStreamWaitEvent(s, ctx->fork, 0));
      CBC_CUDA_TRY(ctx, launch_ensemble_bucket(E, P, w->order, begin, end, K, d_head + b, max_steps,
                                               w->steps_total, epoch, w->budget_ns, blocks, grids.threads[b], s,
                                               grids.smem[b], grids.slots[b], grids.mb[b]));
      ++ctx->launches;
      CBC_CUDA_TRY(ctx, cudaEventRecord(ctx->join[slot], s));
      CBC_CUDA_TRY(ctx, cudaStreamWaitEvent(stream, ctx->join[slot], 0));
      if (pass < 2) ++used_first;
      else ++used_second;
    }
  }
  return CBC_OK;
}

}  // namespace cbc

using namespace cbc;

extern "C" {

int32_t cbc_ensemble_solve(cbc_context* ctx, const cbc_spec* spec, const cbc_ensemble* e, const cbc_work* w,
                           int64_t max_steps, void* stream) {
  if (!ctx) return fail(nullptr, CBC_E_INVALID, "context is NULL");
  ctx->err.clear();
  int32_t rc = check_ensemble(ctx, spec, e, w);
  if (rc) return rc;
  if (max_steps < 1) return fail(ctx, CBC_E_INVALID, "max_steps must be >= 1");
  DeviceGuard dg(ctx->device);
  const Grids grids = grid_sizes(ctx, spec, w);
  return enqueue(ctx, spec, e, w, grids, max_steps, ctx->d_head, (cudaStream_t)stream);
}

// ---- allocation-free batched solve -------------------------------------
// For callers that cannot cudaMalloc while they step (their device memory is
// held by another allocator or a fixed budget).  Host code must not pass
// g_noalloc_scratch itself to a kernel: in host code the name stands for a
// host-side shadow; the device address comes from cudaGetSymbolAddress.
// Scheduling scratch of cbc_ensemble_solve_noalloc: CBC_MAX_BUCKETS work-list
// cursors, then the epoch word (kScheduleBytes = 144 bytes per device).  The
// cursors are zeroed by every call on its stream before its kernels run; the
// epoch word is written by the call's stamp kernel when budget_ns > 0.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScheduleBytes];
static_assert(kScheduleBytes == sizeof(int) * CBC_MAX_BUCKETS + 2 * sizeof(long long), "scratch layout");

constexpr int kNoallocMaxDevices = 64;
static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[kNoallocMaxDevices] = {};

}  // extern "C"

namespace cbc {

// Device address of g_noalloc_scratch on `device`, looked up once per device
// (cudaGetSymbolAddress, which also loads this file's module on that device)
// and cached for the life of the process.  Called by cbc_create with the
// device current, so that cbc_ensemble_solve_noalloc itself never loads the
// module for the scratch.
cudaError_t noalloc_scratch_address(int device, void** out) {
  *out = nullptr;
  if (device < 0 || device >= kNoallocMaxDevices) return cudaSuccess;  // entry point reports it
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    const cudaError_t ce = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (ce != cudaSuccess) return ce;
    g_noalloc_ptr[device] = p;
  }
  *out = g_noalloc_ptr[device];
  return cudaSuccess;
}

}  // namespace cbc

extern "C" {

int32_t cbc_ensemble_solve_noalloc(cbc_context* ctx, const cbc_spec* spec, const cbc_ensemble* e,
                                   const cbc_work* w, int64_t max_steps, void* stream) {
  if (!ctx) return fail(nullptr, CBC_E_INVALID, "context is NULL");
  ctx->err.clear();
  int32_t rc = check_ensemble(ctx, spec, e, w);
  if (rc) return rc;
  if (max_steps < 1) return fail(ctx, CBC_E_INVALID, "max_steps must be >= 1");
  if (ctx->device < 0 || ctx->device >= kNoallocMaxDevices)
    return fail(ctx, CBC_E_UNSUPPORTED, "cbc_ensemble_solve_noalloc: device %d beyond %d", ctx->device,
                kNoallocMaxDevices);
  void* scratch = ctx->noalloc_scratch;
  if (!scratch) return fail(ctx, CBC_E_CUDA, "cbc_ensemble_solve_noalloc: static scratch address unavailable");
  DeviceGuard dg(ctx->device);
  const auto grids = grid_sizes<GridsT<FixedVec>>(ctx, spec, w);
  return enqueue(ctx, spec, e, w, grids, max_steps, static_cast<int*>(scratch), (cudaStream_t)stream);
}

int32_t cbc_plan_create(cbc_context* ctx, const cbc_spec* spec, const cbc_ensemble* e, const cbc_work* w,
                        int64_t max_steps, cbc_plan** out) {
  return cbc_env_plan_create(ctx, spec, e, w, max_steps, nullptr, out);
}

int32_t cbc_env_plan_create(cbc_context* ctx, const cbc_spec* spec, const cbc_ensemble* e, const cbc_work* w,
                            int64_t max_steps, const cbc_env_io* io, cbc_plan** out) {
  if (!ctx) return fail(nullptr, CBC_E_INVALID, "context is NULL");
  ctx->err.clear();
  if (!out) return fail(ctx, CBC_E_INVALID, "out is NULL");
  *out = nullptr;
  int32_t rc = check_ensemble(ctx, spec, e, w);
  if (rc) return rc;
  if (max_steps < 1) return fail(ctx, CBC_E_INVALID, "max_steps must be >= 1");
  if (io) {
    if (!io->actions || !io->obs || io->n_act < 0 || io->n_act > e->cp_stride || io->act_stride < io->n_act ||
        io->K < 1 || io->K > 32 || (long long)io->K * e->ns != e->nb || !(io->t_span > 0.0) || !(io->h0 > 0.0))
      return fail(ctx, CBC_E_INVALID, "env io: need actions, obs, 0 <= n_act <= cp_stride, a uniform K with "
                                      "ns * K == nb, t_span > 0 and h0 > 0");
    if (io->rewards && !env_epilogue_fields_ok(io))
      return fail(ctx, CBC_E_INVALID, "env io: the reward epilogue needs every one of its buffers, "
                                      "episode_length >= 1 and domain_hi > domain_lo");
  }
  DeviceGuard dg(ctx->device);
  cbc_plan* p = new (std::nothrow) cbc_plan();
  if (!p) return fail(ctx, CBC_E_NOMEM, "plan allocation failed");
  p->ctx = ctx;
  p->nbuckets = w->nbuckets;
  cudaError_t ce = cudaMalloc(&p->d_head, kScheduleBytes);
  if (ce != cudaSuccess) {
    delete p;
    return fail(ctx, CBC_E_CUDA, "cudaMalloc: %s", cudaGetErrorString(ce));
  }
  const Grids grids = grid_sizes(ctx, spec, w);
  cudaStream_t cs = ctx->capture;
  const long long launches_before = ctx->launches;
  ce = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (ce != cudaSuccess) {
    cbc_plan_destroy(p);
    return fail(ctx, CBC_E_CUDA, "cudaStreamBeginCapture: %s", cudaGetErrorString(ce));
  }
  if (io) rc = enqueue_env_begin(ctx, e, io, cs);
  if (rc == CBC_OK) rc = enqueue(ctx, spec, e, w, grids, max_steps, p->d_head, cs);
  if (rc == CBC_OK && io) rc = enqueue_env_end(ctx, e, io, cs);
  p->kernels = ctx->launches - launches_before;
  ctx->launches = launches_before;  // counted when the plan is launched
  cudaGraph_t g = nullptr;
  ce = cudaStreamEndCapture(cs, &g);
  if (rc != CBC_OK || ce != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cbc_plan_destroy(p);
    if (rc != CBC_OK) return rc;
    return fail(ctx, CBC_E_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(ce));
  }
  p->graph = g;
  ce = cudaGraphInstantiate(&p->exec, g, 0);
  if (ce != cudaSuccess) {
    cbc_plan_destroy(p);
    return fail(ctx, CBC_E_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(ce));
  }
  *out = p;
  return CBC_OK;
}

int64_t cbc_kernel_launches(const cbc_context* ctx) { return ctx ? ctx->launches : 0; }

int32_t cbc_plan_launch(cbc_plan* p, void* stream) {
  if (!p) return fail(nullptr, CBC_E_INVALID, "plan is NULL");
  p->ctx->err.clear();
  DeviceGuard dg(p->ctx->device);
  cudaStream_t st = (cudaStream_t)stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CBC_CUDA_TRY(p->ctx, cudaStreamIsCapturing(st, &cap));
  if (cap == cudaStreamCaptureStatusActive) {
    // the caller is capturing its own graph (e.g. torch.cuda.graph): a graph
    // launch is not allowed there, so the plan's graph becomes a child node
    // of the graph being captured, after the stream's current dependencies
    cudaGraph_t outer = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    unsigned long long id = 0;
    CBC_CUDA_TRY(p->ctx, cudaStreamGetCaptureInfo(st, &cap, &id, &outer, &deps, &ndeps));
    cudaGraphNode_t node = nullptr;
    CBC_CUDA_TRY(p->ctx, cudaGraphAddChildGraphNode(&node, outer, deps, ndeps, p->graph));
    CBC_CUDA_TRY(p->ctx, cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
  } else {
    CBC_CUDA_TRY(p->ctx, cudaGraphLaunch(p->exec, st));
  }
  p->ctx->launches += p->kernels;
  return CBC_OK;
}

int32_t cbc_plan_destroy(cbc_plan* p) {
  if (!p) return CBC_OK;
  DeviceGuard dg(p->ctx->device);
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->d_head) cudaFree(p->d_head);
  delete p;
  return CBC_OK;
}

}  // extern "C"
