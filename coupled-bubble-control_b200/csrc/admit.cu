// admit.cu -- device-side admission of raw solve requests into slots of a
// ragged ensemble: the parameter precompute (reference models/ckm1d.py:133-202,
// build_parameters and build_control_parameters) and the default initial
// state (model.py:180-225), one warp per request, one lane per bubble.
//
// The arithmetic is that of cbc_b200/models/ckm1d.py (bubble_constants,
// coupling_constants, system_constants): the same products and quotients in
// the same order, IEEE double, no contraction (-fmad=false), with the scalar
// constants evaluated once on the host and passed in (cbc_precompute_consts).
// The result is therefore bit-identical to the host precompute, so a served
// request integrates exactly as it would through Ensemble.from_scene.
#include "cbc_internal.h"
#include "ensemble.h"

namespace cbc {

__global__ void admit_kernel(cbc_ensemble e, cbc_precompute_consts c, const double* __restrict__ rec, int n,
                             int nk, long long coupling_len) {
  const int warp = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  const int li = threadIdx.x & 31;
  if (warp >= n) return;
  const int RL = CBC_ADMIT_RECORD(nk);
  const double* r = rec + (long long)warp * RL;
  const int K = (int)r[0];
  const int s = (int)r[1];
  const long long boff = (long long)r[2];
  const long long coff = (long long)r[3];
  const double span = r[4];
  const double* PA = r + 5;
  const double* FR = PA + nk;
  const double* PS = FR + nk;
  const double* R0um = PS + nk;
  const double* X0 = R0um + 32;
  // a record that does not fit the ensemble is skipped (never written)
  if (K < 1 || K > 32 || s < 0 || s >= e.ns || boff < 0 || boff + K > e.nb || coff < 0 ||
      coff + 3LL * K * K > coupling_len)
    return;

  if (li == 0) {
    e.bubble_offset[s] = boff;
    e.coupling_offset[s] = coff;
    double* sp = e.system_params + (long long)s * e.sp_stride;
    for (int m = 0; m < 5; ++m) sp[m] = c.system_params[m];
    double* cp = e.control_params + (long long)s * e.cp_stride;
    for (int k = 0; k < nk; ++k) {
      const double f = FR[k] * 1000.0;        // kHz -> Hz
      cp[k] = PA[k] * 1.0e5;                  // bar -> Pa
      cp[nk + k] = f * c.two_pi;              // angular frequency
      cp[2 * nk + k] = PS[k] * c.pi;          // phase
      cp[3 * nk + k] = c.two_pi * f / c.cl;   // wave number
    }
    e.t[s] = 0.0;
    e.t_end[s] = span;
    e.t_begin[s] = 0.0;
    e.h[s] = 1e-6;
    e.event[s] = -1.0;
    e.status[s] = 0;
    if (e.dense_index) e.dense_index[s] = 0;
    if (e.steps) e.steps[s] = 0;
    if (e.rejected) e.rejected[s] = 0;
    if (e.conv_ok) e.conv_ok[s] = 0;
    if (e.conv_fail) e.conv_fail[s] = 0;
    if (e.lin_iters) e.lin_iters[s] = 0;
  }
  if (li >= K) return;
  const double R0 = R0um[li] * 1e-6;          // um -> m
  // state R = 1, X = X0, U = V = 0 (dimensionless)
  double* st = e.state + (boff + li) * 4;
  st[0] = 1.0;
  st[1] = X0[li];
  st[2] = 0.0;
  st[3] = 0.0;
  // the 13 bubble constants (ckm1d.py bubble_constants)
  const double sv = c.two_pi / R0 / c.w_ref;
  const double s2 = sv * sv;
  const double pe = c.st2 / R0 + c.p0 - c.pv;
  const double q = c.hl / R0;
  const double wr = c.w_ref * R0;
  double* up = e.unit_params + (boff + li) * e.up_stride;
  up[0] = pe * s2 / c.rho;
  up[1] = c.k1 * pe * sv / c.cl / c.rho;
  up[2] = c.p0pv * s2 / c.rho;
  up[3] = (c.st2 / R0 / c.rho) * s2;
  up[4] = c.k4 / (R0 * R0) * c.tw;
  up[5] = s2 / c.rho;
  up[6] = c.k6 / R0;
  up[7] = R0 * c.w_ref / c.two_pi / c.cl;
  up[8] = q * q;
  up[9] = c.k9 / R0 / c.l_ref / (wr * wr);
  up[10] = c.k10 * ((R0 * R0) * R0);
  up[11] = c.k11 * R0;
  up[12] = R0 / c.l_ref;
  // coupling coefficients M[m][j][i] for receiving bubble i = this lane
  // (ckm1d.py coupling_constants), zero for j == i
  const double Ri2 = R0 * R0;
  double* M = e.coupling + coff;
  const long long KK = (long long)K * K;
  for (int j = 0; j < K; ++j) {
    const double Rj = R0um[j] * 1e-6;
    const double rl = Rj / c.l_ref;
    const double cube_j = (Rj * Rj) * Rj;
    const double cube_rl = (rl * rl) * rl;
    const bool self = (j == li);
    M[0 * KK + (long long)j * K + li] = self ? 0.0 : cube_j / Ri2 / c.l_ref;
    M[1 * KK + (long long)j * K + li] = self ? 0.0 : 3.0 * cube_rl;
    M[2 * KK + (long long)j * K + li] = self ? 0.0 : c.km2 * cube_rl / Ri2;
  }
}

}  // namespace cbc

using namespace cbc;

extern "C" {

int32_t cbc_admit(cbc_context* ctx, const cbc_ensemble* e, const cbc_precompute_consts* c, const double* records,
                  int32_t n, int32_t nk, int64_t coupling_len, void* stream) {
  if (!ctx) return fail(nullptr, CBC_E_INVALID, "context is NULL");
  ctx->err.clear();
  if (!e || !c || (n > 0 && !records)) return fail(ctx, CBC_E_INVALID, "ensemble, constants or records is NULL");
  if (n < 0) return fail(ctx, CBC_E_INVALID, "n must be >= 0");
  if (nk < 1 || nk > NKMAX) return fail(ctx, CBC_E_UNSUPPORTED, "nk = %d: 1..%d harmonic components supported", nk, NKMAX);
  if (!e->bubble_offset || !e->coupling_offset || !e->state || !e->unit_params || !e->system_params ||
      !e->control_params || !e->coupling || !e->t || !e->t_end || !e->t_begin || !e->h || !e->event || !e->status)
    return fail(ctx, CBC_E_INVALID, "a required ensemble pointer is NULL");
  if (e->up_stride < 13 || e->sp_stride < 5 || e->cp_stride < 4 * nk)
    return fail(ctx, CBC_E_INVALID, "parameter row strides too small (need >= 13, 5, 4 nk)");
  if (n == 0) return CBC_OK;
  DeviceGuard dg(ctx->device);
  const int threads = 128;
  const long long blocks = ((long long)n * 32 + threads - 1) / threads;
  admit_kernel<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(*e, *c, records, n, nk, coupling_len);
  ++ctx->launches;
  CBC_CUDA_TRY(ctx, cudaGetLastError());
  return CBC_OK;
}

}  // extern "C"
