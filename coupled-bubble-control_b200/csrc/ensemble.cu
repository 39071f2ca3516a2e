// ensemble.cu -- batched mixed-K integrator: persistent, work-stealing kernels
// over a ragged ensemble, launched together (optionally as one CUDA graph).
//
// The reference can only integrate one (NS, K) ensemble per kernel build
// (all shapes are compile-time macros, backends/cupy_cuda/kernel_loader.py:35-63;
// one thread per bubble padded to TILE = next_pow2(K), specs.py:40-52) and
// relaunches every kernel_steps steps with a host synchronisation.  Here:
//   * systems of any K <= 32 live in one ragged ensemble (CSR offsets);
//   * a work list orders the systems by K bucket, longest expected work first;
//   * each warp holds floor(32/K) system slots; whenever a system finishes,
//     its slot writes the result back and claims the next system of its bucket
//     with one atomicAdd per warp, so lanes never idle while work remains;
//   * one persistent kernel per K bucket (instantiated for KB = 2,4,8,16,32
//     lanes per system slot), launched on forked streams so the buckets overlap
//     and a bucket's tail is filled by the next bucket's warps.
// Integration arithmetic is the same device code as the reference-layout
// kernel (ckm1d_core.cuh), so results are bit-identical to the CPU oracle.
#include "cbc_internal.h"
#include "ensemble.h"


namespace cbc {

template <int KB>
__device__ __forceinline__ void ens_store_dense(const EnsLayout& E, const LaneState& S, const Geo& g, int s,
                                                long long boff, int slot) {
  if (g.li == 0) E.dense_time[(long long)slot * E.ns + s] = S.t;
  double* d = E.dense_state + ((long long)slot * E.nb + boff + g.li) * 4;
  reinterpret_cast<double2*>(d)[0] = make_double2(S.y[0], S.y[1]);
  reinterpret_cast<double2*>(d)[1] = make_double2(S.y[2], S.y[3]);
}

// Loads system s into this lane's slot (lane li of the group) and runs the
// prologue.  Called only by lanes whose group claimed s.
template <int KB>
__device__ __forceinline__ void ens_load(const EnsLayout& E, const Params& P, const Geo& g, int s, LaneState& S,
                                         MView& M, const WarpSmem& W, long long& boff) {
  boff = E.bubble_offset[s];
  if (g.li == 0 && E.trace_load_ns) E.trace_load_ns[s] = global_ns();
  const long long b = boff + g.li;
  const double2* st = reinterpret_cast<const double2*>(E.state + b * 4);
  const double2 s01 = st[0], s23 = st[1];
  S.y[0] = s01.x;
  S.y[1] = s01.y;
  S.y[2] = s23.x;
  S.y[3] = s23.y;
  store_bubble_consts(W, g, E.unit_params + b * E.up_stride, 1);
  const double* sp = E.system_params + (long long)s * E.sp_stride;
  S.sp0 = sp[0];
  S.sp3 = sp[3];
  S.t = E.t[s];
  S.t_end = E.t_end[s];
  S.t_begin = E.t_begin[s];
  S.h = E.h[s];
  S.idx = (P.ndo > 0) ? E.dense_index[s] : 0;
  const double prev = (P.ndo > 0 && S.idx > 0) ? E.dense_time[(long long)(S.idx - 1) * E.ns + s] : 0.0;
  prologue(S, P, E.event[s], prev, E.status[s]);
  M.m = E.coupling + E.coupling_offset[s] + g.li;
  M.sc = (long long)g.K * g.K;
  M.sj = g.K;
  store_coupling(W, g, M);
  if (g.li == 0) store_harmonics(W, g, sp[1], sp[2], sp[4], E.control_params + (long long)s * E.cp_stride, P.nk, 1);
}

template <int KB>
__device__ __forceinline__ void ens_writeback(const EnsLayout& E, const Params& P, const Geo& g, int s,
                                              long long boff, LaneState& S) {
  double2* st = reinterpret_cast<double2*>(E.state + (boff + g.li) * 4);
  st[0] = make_double2(S.y[0], S.y[1]);
  st[1] = make_double2(S.y[2], S.y[3]);
  if (g.li == 0) {
    if (E.trace_done_ns) E.trace_done_ns[s] = global_ns();
    E.t[s] = S.t;
    E.h[s] = S.h;
    E.event[s] = S.g_old;
    E.status[s] = S.status;
    if (P.ndo > 0) E.dense_index[s] = S.idx;
    if (E.steps) E.steps[s] += S.steps;
    if (E.rejected) E.rejected[s] += S.rejected;
    if (E.conv_ok) E.conv_ok[s] += S.conv_ok;
    if (E.conv_fail) E.conv_fail[s] += S.conv_fail;
    if (E.lin_iters) E.lin_iters[s] += S.lin_iters;
  }
}

// Persistent worker: warps claim systems of bucket [begin, end) of the work
// list until it is empty.  All systems of a bucket have the same K (<= KB).
template <int KB, int KC, int LIN, int MB>
__global__ void __launch_bounds__(128, min_blocks_variant(KB, MB))
    ensemble_kernel(EnsLayout E, Params P, const int* __restrict__ order, int begin, int end, int K, int* head,
                    long long max_steps, int steps_total, const long long* epoch, long long budget_ns,
                    int slots) {
  extern __shared__ __align__(16) double smem[];
  const Geo g = make_geo(KC > 0 ? KC : K, slots);
  const WarpSmem W = warp_smem(smem, g.K, P.nk, LIN);
  const int lane = threadIdx.x & 31;
  const bool leader = g.valid && g.li == 0;

  LaneState S;
  MView M;
  M.m = E.coupling;
  M.sc = M.sj = 0;
  S.active = false;
  S.status = ST_ACTIVE;
  S.steps = 0;
  int sys = -1;           // system in this lane's slot (-1: none)
  long long boff = 0;
  long long step_base = 0;  // steps the system had accumulated before it was loaded (steps_total)
  bool drained = false;   // work list exhausted for this warp (warp-uniform)
  const long long deadline = budget_ns > 0 ? epoch[0] + budget_ns : 0;
  bool sliced_out = false;  // time slice over (warp-uniform); independent of drained

  while (true) {
    // ---- time slice over: stop every slot after its current step ----
    if (deadline != 0 && !sliced_out) {
      long long now = 0;
      if (lane == 0) now = global_ns();
      now = __shfl_sync(FULL, now, 0);
      if (now >= deadline) {
        sliced_out = true;
        drained = true;
      }
    }
    if (sliced_out && S.active) {
      S.status = ST_MAX_STEPS;
      S.active = false;
    }
    // ---- retire finished systems and refill empty slots (warp-uniform) ----
    const bool retire = g.valid && sys >= 0 && !S.active;
    if (__any_sync(FULL, retire)) {
      if (retire) ens_writeback<KB>(E, P, g, sys, boff, S);
      if (retire) sys = -1;
    }
    const bool want = leader && sys < 0 && !drained;
    const unsigned wmask = __ballot_sync(FULL, want);
    if (wmask) {
      int base_idx = 0;
      if (lane == 0) base_idx = atomicAdd(head, __popc(wmask));
      base_idx = __shfl_sync(FULL, base_idx, 0);
      int claim = -1;
      if (want) {
        const int idx = begin + base_idx + __popc(wmask & ((1u << lane) - 1u));
        claim = (idx < end) ? order[idx] : -1;
      }
      if (__any_sync(FULL, want && claim < 0)) drained = true;
      // hand the claimed system id to every lane of the group
      // (both shuffles are executed by every lane: never inside a
      // short-circuit or a divergent branch)
      const int got = __shfl_sync(FULL, claim, g.base);
      const int leader_wanted = __shfl_sync(FULL, (int)want, g.base);
      const bool fresh = g.valid && sys < 0 && got >= 0 && leader_wanted != 0;
      if (fresh) {
        sys = got;
        ens_load<KB>(E, P, g, sys, S, M, W, boff);
        step_base = (steps_total && E.steps) ? (long long)E.steps[sys] : 0;
        if (S.active && step_base >= max_steps) {
          S.status = ST_MAX_STEPS;
          S.active = false;
        }
      }
      __syncwarp();
      // first dense sample and initial event value for the fresh systems
      if (fresh && S.active && P.ndo > 0) {
        bool stq;
        if (P.dense_mode == 0) stq = (S.idx < P.ndo) && (S.dnext <= S.t);
        else stq = (S.idx < P.ndo) && (S.t >= grid_time(S, S.idx, P.ndo));
        if (stq) {
          ens_store_dense<KB>(E, S, g, sys, boff, S.idx);
          S.idx += 1;
          if (P.dense_mode == 0) {
            const double nx = S.t + S.ddt;
            S.dnext = nx < S.t_end ? nx : S.t_end;
          }
        }
      }
      const double g0 = group_event<KB>(S.y, upv(W, g, 12), g, P.col);
      if (fresh && S.active) S.g_old = g0;
      // systems that arrive already finished go straight back out
      continue;
    }
    if (!__any_sync(FULL, S.active)) {
      if (!__any_sync(FULL, sys >= 0)) break;  // nothing left in any slot
      continue;
    }
    // ---- one Cash-Karp step for every active slot ----
    const bool stq = step<KB, KC, LIN>(g, P, W, M, S);
    if (stq) ens_store_dense<KB>(E, S, g, sys, boff, S.idx);
    after_store(S, P, stq);
    if (S.active && S.steps + step_base >= max_steps) {
      S.status = ST_MAX_STEPS;
      S.active = false;
    }
  }
}

size_t max_block_smem(int device) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  return (size_t)v;
}

// Every batched kernel asks for the same (maximum) shared-memory carveout, so
// that blocks of different bucket kernels can share an SM: with per-kernel
// carveouts an SM configured for one kernel takes no block of another until it
// drains, which serialises the buckets.
template <int KB, int KC, int LIN, int MB>
cudaError_t configure_ensemble_kernel(size_t shmem) {
  cudaError_t e = cudaFuncSetAttribute(ensemble_kernel<KB, KC, LIN, MB>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared);
  // the opt-in limit is raised to the device maximum (never lowered again), so
  // a launch captured earlier with a larger request stays valid
  if (e == cudaSuccess && shmem > 48 * 1024) {
    int dev = 0;
    e = cudaGetDevice(&dev);
    const size_t cap = max_block_smem(dev);
    if (e == cudaSuccess) {
      if (shmem > cap) return cudaErrorInvalidValue;
      e = cudaFuncSetAttribute(ensemble_kernel<KB, KC, LIN, MB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap);
    }
  }
  return e;
}

__global__ void stamp_kernel(long long* epoch) { *epoch = global_ns(); }

cudaError_t launch_stamp(long long* epoch, cudaStream_t stream) {
  stamp_kernel<<<1, 1, 0, stream>>>(epoch);
  return cudaGetLastError();
}

cudaError_t launch_ensemble_bucket(const EnsLayout& E, const Params& P, const int* order, int begin, int end,
                                   int K, int* head, long long max_steps, int steps_total,
                                   const long long* epoch, long long budget_ns, int blocks, int threads,
                                   cudaStream_t stream, size_t smem_bytes, int slots, int mb) {
  return dispatch_k(K, [&](auto kb, auto kc) {
    return dispatch_lin(P.lin, [&](auto lin) {
      return dispatch_mb(decltype(kb)::value <= 8 ? mb : 0, [&](auto mbv) {
        constexpr int KB = decltype(kb)::value, KC = decltype(kc)::value, LIN = decltype(lin)::value,
                      MB = decltype(mbv)::value;
        size_t shmem = sizeof(double) * (size_t)smem_doubles_per_warp(K, P.nk, LIN) * (threads / 32);
        if (smem_bytes > shmem) shmem = smem_bytes;
        cudaError_t e = configure_ensemble_kernel<KB, KC, LIN, MB>(shmem);
        if (e != cudaSuccess) return e;
        ensemble_kernel<KB, KC, LIN, MB><<<blocks, threads, shmem, stream>>>(
            E, P, order, begin, end, K, head, max_steps, steps_total, epoch, budget_ns, slots);
        return cudaGetLastError();
      });
    });
  });
}

int resident_blocks(int K, int nk, int threads, int lin, int mb) {
  const size_t shmem = sizeof(double) * (size_t)smem_doubles_per_warp(K, nk, lin) * (threads / 32);
  int n = 0;
  const cudaError_t e = dispatch_k(K, [&](auto kb, auto kc) {
    return dispatch_lin(lin, [&](auto li) {
      return dispatch_mb(decltype(kb)::value <= 8 ? mb : 0, [&](auto mbv) {
        constexpr int KB = decltype(kb)::value, KC = decltype(kc)::value, LIN = decltype(li)::value,
                      MB = decltype(mbv)::value;
        configure_ensemble_kernel<KB, KC, LIN, MB>(shmem);
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ensemble_kernel<KB, KC, LIN, MB>, threads, shmem);
      });
    });
  });
  return (e == cudaSuccess && n > 0) ? n : 1;
}

}  // namespace cbc
