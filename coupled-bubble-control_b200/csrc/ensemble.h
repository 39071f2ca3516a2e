// ensemble.h -- device view of a ragged mixed-K ensemble (the batched layout).
//
// Layout in HBM (all row-major, float64 unless noted):
//   K[ns] (int32), bubble_offset[ns] (int64: first bubble of system s),
//   coupling_offset[ns] (int64: first element of the 3*K*K block of s)
//   state[nb][4]              R, X, U, V per bubble (32 B rows, double2 loads)
//   unit_params[nb][up_stride]  the 13 per-bubble constants (ckm1d.py:154-168)
//   system_params[ns][sp_stride]  the 5 per-system constants (ckm1d.py:171-175)
//   control_params[ns][cp_stride] PA[nk], omega[nk], phase[nk], wave number[nk]
//   coupling[...]             per system: M[c][j][i], c = 0..2, i receiving bubble
//   t, t_end, t_begin, h, event (ns) f64; status, dense_index (ns) i32
//   dense_time[ndo][ns], dense_state[ndo][nb][4]  (sample-major)
//   steps, rejected, conv_ok, conv_fail (ns) i32, lin_iters (ns) i64 (optional)
#pragma once

namespace cbc {

struct EnsLayout {
  int ns;
  long long nb;
  const long long* bubble_offset;
  const long long* coupling_offset;
  double* state;
  const double* unit_params;
  const double* system_params;
  const double* control_params;
  const double* coupling;
  double* t;
  const double* t_end;
  const double* t_begin;
  double* h;
  double* event;
  int* status;
  int* dense_index;
  double* dense_time;
  double* dense_state;
  int* steps;
  int* rejected;
  int* conv_ok;
  int* conv_fail;
  long long* lin_iters;
  long long* trace_load_ns;   // optional: %globaltimer when a slot picked the system up
  long long* trace_done_ns;   // optional: %globaltimer when its result was written back
  int up_stride, sp_stride, cp_stride;
};

__device__ __forceinline__ long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return (long long)t;
}

// smem_bytes: dynamic shared memory per block; 0 = what the kernel needs.
// A larger request keeps other blocks off the SM (latency lanes).
// epoch: device word holding the solve's start time (written by
// launch_stamp); budget_ns > 0 stops every system budget_ns after it.
cudaError_t launch_ensemble_bucket(const EnsLayout& E, const Params& P, const int* order, int begin, int end,
                                   int K, int* head, long long max_steps, int steps_total,
                                   const long long* epoch, long long budget_ns, int blocks, int threads,
                                   cudaStream_t stream, size_t smem_bytes = 0, int slots = 32, int mb = 0);
// Writes the device clock (%globaltimer, ns) to *epoch.
cudaError_t launch_stamp(long long* epoch, cudaStream_t stream);
size_t max_block_smem(int device);
int resident_blocks(int K, int nk, int threads, int lin = LIN_RICHARDSON, int mb = 0);

}  // namespace cbc
