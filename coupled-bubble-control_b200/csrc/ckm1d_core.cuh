// ckm1d_core.cuh -- per-lane CKM1D right-hand side and Cash-Karp step for sm_100a.
//
// Execution model: one lane per bubble.  A system of K bubbles occupies K
// consecutive lanes of a warp ("group"); a warp holds floor(32/K) systems.
// Everything that couples bubbles (coupling terms, the implicit-coupling
// iteration, reductions for norms, error ratio and the collision event) is
// exchanged with full-warp __shfl_sync inside the group, so no block barrier
// and no shared-memory atomics are needed (the reference synchronises the
// whole block 4x per Richardson iteration, ckm1d_def.py:303-404).  Control flow
// that contains shuffles is warp-uniform; per-system decisions only select
// values.  Per-system scalars (t, h, event value, ...) are held redundantly by
// every lane of the group and stay identical because every lane computes them
// from the same shuffled inputs.
//
// Numerics: FP64 throughout, compiled with -fmad=false; every fused
// multiply-add is an explicit fma().  Operation order matches
// oracle/ckm1d_oracle.cpp line for line, and the elementary functions come
// from cbc_math.h, so results equal the CPU oracle bit for bit.  The algorithm
// restates coupledbubble_control/backends/numba/sysmtem_definitions/ckm1d_def.py
// (acoustic_field_1d :79-114, ode_fun :408-497, explicit_coupling :164-246,
// mat_vec_product :250-299, implicit_coupling :303-404, event_fun :499-556) and
// rkck45_coupled_numba_stepper.py (:362-677).
#pragma once

#include <stdint.h>
#include "cbc_math.h"

namespace cbc {

constexpr unsigned FULL = 0xffffffffu;
constexpr int NKMAX = 4;                        // harmonic components supported
constexpr int HC_PER_K = 7;                     // per-harmonic constants
constexpr double TWO_PI = 6.283185307179586;    // 2.0 * np.pi

// Cash-Karp tableau (stepper.py:15-24)
constexpr double A2 = 1.0 / 5.0, A3 = 3.0 / 10.0, A4 = 3.0 / 5.0, A5 = 1.0, A6 = 7.0 / 8.0;
constexpr double B21 = 1.0 / 5.0;
constexpr double B31 = 3.0 / 40.0, B32 = 9.0 / 40.0;
constexpr double B41 = 3.0 / 10.0, B42 = -9.0 / 10.0, B43 = 6.0 / 5.0;
constexpr double B51 = -11.0 / 54.0, B52 = 5.0 / 2.0, B53 = -70.0 / 27.0, B54 = 35.0 / 27.0;
constexpr double B61 = 1631.0 / 55296.0, B62 = 175.0 / 512.0, B63 = 575.0 / 13824.0,
                 B64 = 44275.0 / 110592.0, B65 = 253.0 / 4096.0;
constexpr double C1 = 37.0 / 378.0, C3 = 250.0 / 621.0, C4 = 125.0 / 594.0, C6 = 512.0 / 1771.0;
constexpr double CP1 = 2825.0 / 27648.0, CP3 = 18575.0 / 48384.0, CP4 = 13525.0 / 55296.0,
                 CP5 = 277.0 / 14336.0, CP6 = 1.0 / 4.0;
constexpr double CE1 = C1 - CP1, CE3 = C3 - CP3, CE4 = C4 - CP4, CE5 = 0.0 - CP5, CE6 = C6 - CP6;

// Per-system status codes (stepper.py:27-33).
enum : int {
  ST_ACTIVE = 0, ST_SUCCESS = 1, ST_EVENT = 2,
  ST_MAX_STEPS = -1, ST_STEP_LIMIT = -2, ST_CONV_FAIL = -3, ST_NONFINITE = -4
};

// Solver constants shared by every system of a launch.
struct Params {
  double atol, rtol, min_step, max_step;
  double lin_atol2, lin_rtol2, omega, etol, col;
  int lin_max_iter;
  int ndo;         // dense samples per system
  int dense_mode;  // 0 reference schedule, 1 exact grid
  int nk;          // harmonics
  int ac;          // 0 CONST, 1 SW_N, 2 SW_A
};

// Position of this lane inside its system group.
struct Geo {
  int K;       // bubbles per system (warp-uniform)
  int G;       // groups per warp = 32 / K
  int grp;     // group index (clamped to a valid slot for idle lanes)
  int base;    // first lane of the group
  int li;      // bubble index of this lane
  bool valid;  // lane belongs to a group
};

__device__ __forceinline__ Geo make_geo(int K) {
  Geo g;
  const int lane = threadIdx.x & 31;
  g.K = K;
  g.G = 32 / K;
  const int grp = lane / K;
  g.valid = grp < g.G;
  g.grp = g.valid ? grp : 0;
  g.base = g.valid ? grp * K : lane;
  g.li = g.valid ? lane - grp * K : 0;
  return g;
}

__device__ __forceinline__ double shfl(double v, int src) { return __shfl_sync(FULL, v, src); }

// Coupling matrices of this lane's system: M(c, j, i=this lane) = m[c*sc + j*sj]
struct MView {
  const double* __restrict__ m;  // points at M(0, 0, i)
  long long sc, sj;
};

// Per-lane integrator state (bubble + copies of the system scalars).
struct LaneState {
  double y[4];                 // R, X, U, V
  double up[13];
  double c73, c47;             // up7/3, up4*up7
  double sp0, sp3;             // 3 gamma, c
  double t, t_end, t_begin, h, g_old;
  double dnext, ddt;           // dense schedule (next sample time, spacing)
  int idx;                     // dense samples stored
  int status;
  bool active;
  int steps, rejected, conv_ok, conv_fail;
  long long lin_iters;
};

// Per-system harmonic constants in shared memory, component-major so that
// the groups of a warp hit distinct banks: hc[(7k + c) * G + grp].
//   c = 0 w0*omega, 1 phase, 2 l0*wave, 3 PA, 4 PA*omega, 5 PA*wave, 6 PA*u0
// Written by lane 0 of the group from system parameters sp1 = 1/omega_ref,
// sp2 = lambda_ref/2pi, sp4 = 1/(rho c) and the control parameters
// cp[m * cp_stride], m = 0..4nk-1 (PA, omega, phase, wave number).
__device__ __forceinline__ void store_harmonics(double* hc, const Geo& g, double sp1, double sp2,
                                                double sp4, const double* cp, int nk,
                                                long long cp_stride) {
  // acoustic_field_1d (ckm1d_def.py:95-97): w0 = 2pi sp[1], l0 = 2pi sp[2], u0 = sp[4]
  const double w0 = TWO_PI * sp1;
  const double l0 = TWO_PI * sp2;
  const double u0 = sp4;
  for (int k = 0; k < nk; ++k) {
    const double amps = cp[k * cp_stride], omega = cp[(nk + k) * cp_stride],
                 phase = cp[(2 * nk + k) * cp_stride], wave = cp[(3 * nk + k) * cp_stride];
    double* h = hc + (HC_PER_K * k) * g.G + g.grp;
    h[0 * g.G] = w0 * omega;
    h[1 * g.G] = phase;
    h[2 * g.G] = l0 * wave;
    h[3 * g.G] = amps;
    h[4 * g.G] = amps * omega;
    h[5 * g.G] = amps * wave;
    h[6 * g.G] = amps * u0;
  }
}

__device__ __forceinline__ double hcv(const double* hc, const Geo& g, int k, int c) {
  return hc[(HC_PER_K * k + c) * g.G + g.grp];
}

// Sum of v over the group, ascending bubble index (fixed order).
template <int KB>
__device__ __forceinline__ double group_sum(double v, const Geo& g) {
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < KB; ++j)
    if (j < g.K) s = s + shfl(v, g.base + j);
  return s;
}

// Minimum of v over the group, starting from 1e30; NaN entries never win
// (same as the oracle's sequential "if (v < m) m = v" scan).
template <int KB>
__device__ __forceinline__ double group_min(double v, const Geo& g) {
  double m = 1.0e30;
#pragma unroll
  for (int j = 0; j < KB; ++j)
    if (j < g.K) {
      const double x = shfl(v, g.base + j);
      if (x < m) m = x;
    }
  return m;
}

// AND of a per-lane predicate over the group.
__device__ __forceinline__ bool group_all(bool p, const Geo& g) {
  const unsigned bad = __ballot_sync(FULL, !p);
  const unsigned gm = (g.K >= 32) ? FULL : (((1u << g.K) - 1u) << g.base);
  return (bad & gm) == 0u;
}

// event_fun (ckm1d_def.py:499-556): min over neighbours of
// |x_i - x_{i+1}| - (R_i R0_i + R_{i+1} R0_{i+1}) / lambda * (1 + threshold).
template <int KB>
__device__ __forceinline__ double group_event(const double y[4], double up12, const Geo& g, double col) {
  const double ri = y[0] * up12;
  const double rj = __shfl_down_sync(FULL, ri, 1);
  const double xj = __shfl_down_sync(FULL, y[1], 1);
  double gap = 1e30;
  if (g.li + 1 < g.K) gap = fabs(y[1] - xj) - (ri + rj) * col;
  // sequential min with initial 1e30 (NaN never wins)
  double m = 1e30;
#pragma unroll
  for (int j = 0; j < KB; ++j)
    if (j < g.K) {
      const double x = shfl(gap, g.base + j);
      if (x < m) m = x;
    }
  return m;
}

// RHS of the whole system, evaluated by its K lanes: dy of this lane's bubble.
// Returns via conv/iters the outcome of the implicit-coupling iteration.
template <int KB>
__device__ __forceinline__ void rhs(const Geo& g, const Params& P, const double* hc, const MView& M,
                                    const LaneState& S, bool on, double t, const double y[4],
                                    double dy[4], bool& conv, int& iters) {
  const int K = g.K;
  const int li = g.li;
  const double x0 = y[0], x1 = y[1], x2 = y[2], x3 = y[3];

  // ---- time harmonics (system-uniform): lane k computes harmonic k ----
  double st[NKMAX], ct[NKMAX];
  if (P.nk <= K) {
    const int k = li < P.nk ? li : 0;
    double s_, c_;
    cbcm::sincos(fma(hcv(hc, g, k, 0), t, hcv(hc, g, k, 1)), &s_, &c_);
#pragma unroll
    for (int kk = 0; kk < NKMAX; ++kk)
      if (kk < P.nk) {
        st[kk] = shfl(s_, g.base + kk);
        ct[kk] = shfl(c_, g.base + kk);
      }
  } else {
#pragma unroll
    for (int kk = 0; kk < NKMAX; ++kk)
      if (kk < P.nk) cbcm::sincos(fma(hcv(hc, g, kk, 0), t, hcv(hc, g, kk, 1)), &st[kk], &ct[kk]);
  }

  // ---- uncoupled Keller--Miksis + translation (ckm1d_def.py:418-447) ----
  const double* up = S.up;
  const double rx0 = 1.0 / x0;
  const double p = cbcm::pow_pos(rx0, S.sp0);
  double pa = 0.0, pt = 0.0, px = 0.0, ux = 0.0;
#pragma unroll
  for (int k = 0; k < NKMAX; ++k) {
    if (k < P.nk) {
      const double a = hcv(hc, g, k, 3), aw = hcv(hc, g, k, 4);
      if (P.ac == 0) {  // CONST
        pa = fma(a, st[k], pa);
        pt = fma(aw, ct[k], pt);
      } else {
        double sx, cx;
        cbcm::sincos(fma(hcv(hc, g, k, 2), x1, hcv(hc, g, k, 1)), &sx, &cx);
        const double awv = hcv(hc, g, k, 5), au = hcv(hc, g, k, 6);
        if (P.ac == 1) {  // SW_N
          pa = fma(a * sx, st[k], pa);
          pt = fma(aw * sx, ct[k], pt);
          px = fma(awv * cx, st[k], px);
          ux = fma(au * cx, ct[k], ux);
        } else {  // SW_A
          pa = fma(a * cx, st[k], pa);
          pt = fma(aw * cx, ct[k], pt);
          px = fma(-(awv * sx), st[k], px);
          ux = fma(-(au * sx), ct[k], ux);
        }
      }
    }
  }
  const double q = fma(up[7], x2, 1.0);
  double N = fma(up[1], x2, up[0]) * p;
  N = fma(-up[2], q, N);
  N = fma(-up[3], rx0, N);
  N = fma(-(up[4] * x2), rx0, N);
  const double w = fma(-S.c73, x2, 1.0);
  N = fma((-1.5 * w) * x2, x2, N);
  N = fma(-(q * up[5]), pa, N);
  N = fma(-(up[6] * pt), x0, N);
  N = fma(up[8] * x3, x3, N);
  const double D = fma(-(up[7] * x0), x2, x0) + S.c47;
  const double rD = 1.0 / D;
  const double x02 = x0 * x0;
  const double x03 = x02 * x0;
  const double Fb1 = -(up[10] * x03) * px;
  const double Fd = -(up[11] * x0) * fma(x3, S.sp3, -ux);
  const double rx03 = (rx0 * rx0) * rx0;
  double b0 = N * rD;
  double b1 = fma((3.0 * (Fb1 + Fd)) * up[9], rx03, -(((3.0 * x2) * rx0) * x3));
  const double cpf0 = rD, cpf1 = x3 * rD, cpf2 = x2 * rx0, cpf3 = rx0 * rx0;

  // ---- explicit coupling + matrix of the implicit system, ascending j ----
  double g0 = 0.0, g1 = 0.0, tn = 0.0, tg2 = 0.0, tg3 = 0.0;
  double Am[KB], Bm[KB], Cm[KB], Dm[KB];
#pragma unroll
  for (int j = 0; j < KB; ++j) {
    Am[j] = 0.0; Bm[j] = 0.0; Cm[j] = 0.0; Dm[j] = 0.0;
    if (j < K) {
      const int src = g.base + j;
      // neighbour state; its coupling terms are recomputed exactly as the
      // owning lane computes them (cheaper than shuffling seven terms)
      const double xj0 = shfl(x0, src), xj1 = shfl(x1, src), xj2 = shfl(x2, src), xj3 = shfl(x3, src);
      if (j != li && on) {
        const double j02 = xj0 * xj0;
        const double j03 = j02 * xj0;
        const double h0j = xj0 * (xj2 * xj2);
        const double h1j = j02 * xj2;
        const double h2j = h1j * xj3;
        const double h3j = j03 * xj3;
        const double h4j = h3j * xj3;
        const double delta = x1 - xj1;
        const double sg = (double)((delta > 0.0) - (delta < 0.0));
        const double ad = fabs(delta);
        const double rd = 1.0 / (ad > 1e-30 ? ad : 1e-30);
        const double rd2 = rd * rd;
        const double srd2 = rd2 * sg;
        const double rd3 = rd2 * rd;
        const double m0 = __ldg(M.m + j * M.sj);
        const double m1 = __ldg(M.m + M.sc + j * M.sj);
        const double m2 = __ldg(M.m + 2 * M.sc + j * M.sj);
        double t0 = fma(2.5 * srd2, h2j, rd3 * h4j);
        t0 = fma(2.0 * rd, h0j, t0);
        g0 = fma(-m0, t0, g0);
        const double t1 = fma(srd2, h1j, rd3 * h3j);
        g1 = fma(-0.5 * m0, t1, g1);
        const double t2 = fma(2.0 * srd2, h0j, (5.0 * rd3) * h2j);
        tn = fma(m1, t2, tn);
        tg2 = fma(m1, t1, tg2);
        tg3 = fma(m2, t1, tg3);
        Am[j] = (m0 * rd) * j02;
        Bm[j] = ((0.5 * m0) * srd2) * j03;
        Cm[j] = -((m1 * srd2) * j02);
        Dm[j] = -((m1 * rd3) * j03);
      }
    }
  }
  b0 = fma(g0, cpf0, fma(g1, cpf1, b0));
  b1 = b1 + fma(tg2, cpf2, fma(tg3, cpf3, tn));

  // ---- implicit coupling: relaxed Richardson from v = b (ckm1d_def.py:303-404) ----
  const double bn = group_sum<KB>(fma(b0, b0, b1 * b1), g);
  const double rt = P.lin_rtol2 * bn;
  const double tol2 = rt > P.lin_atol2 ? rt : P.lin_atol2;
  double vr = b0, vt = b1;
  conv = !on;
  iters = 0;
  for (int it = 0; it < P.lin_max_iter; ++it) {
    if (__all_sync(FULL, conv)) break;
    double ar = 0.0, at = 0.0;
#pragma unroll
    for (int j = 0; j < KB; ++j)
      if (j < K) {
        const double vrj = shfl(vr, g.base + j), vtj = shfl(vt, g.base + j);
        if (j != li) {
          ar = fma(Am[j], vrj, fma(Bm[j], vtj, ar));
          at = fma(Cm[j], vrj, fma(Dm[j], vtj, at));
        }
      }
    const double ax0 = fma(ar, cpf0, vr);
    const double ax1 = at + vt;
    const double r0 = b0 - ax0;
    const double r1 = b1 - ax1;
    const double rn = group_sum<KB>(fma(r0, r0, r1 * r1), g);
    if (!conv) {
      ++iters;
      if (rn < tol2) {
        conv = true;
      } else {
        vr = fma(P.omega, r0, vr);
        vt = fma(P.omega, r1, vt);
      }
    }
  }
  if (!on) conv = true;
  dy[0] = x2;
  dy[1] = x3;
  dy[2] = vr;
  dy[3] = vt;
}

// Exact sample time k of the grid dense mode.
__device__ __forceinline__ double grid_time(const LaneState& S, int k, int ndo) {
  if (k >= ndo - 1 && ndo > 1) return S.t_end;
  return fma((double)k, S.ddt, S.t_begin);
}

// Sets up the dense schedule and the status at (re)load time.  Mirrors the
// kernel prologue (stepper.py:179-214) with the launch-transparent dense
// schedule.  `prev_time` is the time of the last stored sample (idx > 0).
// A stored failure status (-2, -3, -4) keeps the system stopped, so a failed
// system does not retry at every relaunch; -1 (budget spent) resumes.
__device__ __forceinline__ void prologue(LaneState& S, const Params& P, double g_store, double prev_time,
                                         int status_in) {
  S.status = (S.t >= S.t_end) ? ST_SUCCESS : ST_ACTIVE;
  if (fabs(g_store) < P.etol) S.status = ST_EVENT;
  if (status_in <= ST_STEP_LIMIT) S.status = status_in;
  S.active = (S.status == ST_ACTIVE);
  S.g_old = g_store;
  S.ddt = (P.ndo == 1) ? (S.t_end - S.t_begin)
                       : (P.ndo > 1 ? (S.t_end - S.t_begin) / (double)(P.ndo - 1) : 0.0);
  if (P.dense_mode == 0) {
    if (S.idx == 0) S.dnext = S.t;
    else {
      const double nx = prev_time + S.ddt;
      S.dnext = nx < S.t_end ? nx : S.t_end;
    }
  }
  S.steps = S.rejected = S.conv_ok = S.conv_fail = 0;
  S.lin_iters = 0;
}

__device__ __forceinline__ void tally(LaneState& S, bool on, bool cv, int it, int& conv_fail_here) {
  if (!on) return;
  S.lin_iters += it;
  if (cv) ++S.conv_ok;
  else { ++S.conv_fail; ++conv_fail_here; }
}

// One adaptive Cash-Karp step for every active group of the warp
// (stepper.py:362-677).  Returns true (per lane) if a dense sample must be
// stored after this step; the caller writes it.
template <int KB>
__device__ __forceinline__ bool step(const Geo& g, const Params& P, const double* hc, const MView& M,
                                     LaneState& S) {
  const bool on = S.active;
  double h = S.h;
  if (h < P.min_step) h = P.min_step;
  if (h > P.max_step) h = P.max_step;
  const double rem = S.t_end - S.t;
  if (h > rem) h = rem;
  bool landing = false;
  double t_land = 0.0;
  if (P.dense_mode == 1 && S.idx < P.ndo) {
    t_land = grid_time(S, S.idx, P.ndo);
    const double remk = t_land - S.t;
    if (h >= remk) {
      h = remk;
      landing = true;
    }
  }
  const double t = S.t;
  const double* y = S.y;
  double k1[4], k2[4], k3[4], k4[4], k5[4], k6[4], ys[4];
  bool cv;
  int it;
  int conv_fail_here = 0;

  rhs<KB>(g, P, hc, M, S, on, t, y, k1, cv, it);
  tally(S, on, cv, it, conv_fail_here);
#pragma unroll
  for (int c = 0; c < 4; ++c) ys[c] = fma(h, B21 * k1[c], y[c]);
  rhs<KB>(g, P, hc, M, S, on, fma(A2, h, t), ys, k2, cv, it);
  tally(S, on, cv, it, conv_fail_here);
#pragma unroll
  for (int c = 0; c < 4; ++c) ys[c] = fma(h, fma(B32, k2[c], B31 * k1[c]), y[c]);
  rhs<KB>(g, P, hc, M, S, on, fma(A3, h, t), ys, k3, cv, it);
  tally(S, on, cv, it, conv_fail_here);
#pragma unroll
  for (int c = 0; c < 4; ++c) ys[c] = fma(h, fma(B43, k3[c], fma(B42, k2[c], B41 * k1[c])), y[c]);
  rhs<KB>(g, P, hc, M, S, on, fma(A4, h, t), ys, k4, cv, it);
  tally(S, on, cv, it, conv_fail_here);
#pragma unroll
  for (int c = 0; c < 4; ++c)
    ys[c] = fma(h, fma(B54, k4[c], fma(B53, k3[c], fma(B52, k2[c], B51 * k1[c]))), y[c]);
  rhs<KB>(g, P, hc, M, S, on, fma(A5, h, t), ys, k5, cv, it);
  tally(S, on, cv, it, conv_fail_here);
#pragma unroll
  for (int c = 0; c < 4; ++c)
    ys[c] = fma(h, fma(B65, k5[c], fma(B64, k4[c], fma(B63, k3[c], fma(B62, k2[c], B61 * k1[c])))), y[c]);
  rhs<KB>(g, P, hc, M, S, on, fma(A6, h, t), ys, k6, cv, it);
  tally(S, on, cv, it, conv_fail_here);

  // candidate (c2 = c5 = 0)
  double yn[4];
  bool fin = true;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const double acc = fma(C6, k6[c], fma(C4, k4[c], fma(C3, k3[c], C1 * k1[c])));
    yn[c] = fma(h, acc, y[c]);
    fin = fin && cbcm::isfinite_(yn[c]);
  }
  const bool finite = group_all(fin, g);
  if (on) ++S.steps;

  const double g_new = group_event<KB>(yn, S.up[12], g, P.col);
  const bool crossing = (S.g_old * g_new < 0.0);
  // embedded error estimate, per lane (ce2 = 0)
  double ratio_l = 1.0e30;
  bool ok_l = true;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const double es = fma(CE6, k6[c], fma(CE5, k5[c], fma(CE4, k4[c], fma(CE3, k3[c], CE1 * k1[c]))));
    const double e = fabs(h * es) + 1.0e-18;
    const double ay = fabs(yn[c]), ao = fabs(y[c]);
    const double tl = P.rtol * (ay > ao ? ay : ao);
    const double tol = tl > P.atol ? tl : P.atol;
    const double r = tol / e;
    if (r < ratio_l) ratio_l = r;
    if (r < 1.0) ok_l = false;
  }
  const double ratio = group_min<KB>(ratio_l, g);
  const bool okerr = group_all(ok_l, g);

  bool store = false;
  if (on) {
    bool ok;
    double h_next;
    if (crossing) {
      const double abs_old = fabs(S.g_old);
      const double denom = abs_old + fabs(g_new);
      h_next = h * ((abs_old / (denom + 1e-15)) * 0.99);
      ok = false;
    } else if (!finite) {
      S.status = ST_NONFINITE;
      S.active = false;
      ++S.rejected;
      S.h = h;
      return false;
    } else {
      ok = okerr;
      double fac;
      if (ok) {
        double f = 0.9 * cbcm::pow_pos(ratio, 0.2);
        f = f > 0.2 ? f : 0.2;
        fac = f < 5.0 ? f : 5.0;
      } else {
        double f = 0.9 * cbcm::pow_pos(ratio, 0.25);
        f = f > 0.1 ? f : 0.1;
        fac = f < 0.5 ? f : 0.5;
      }
      h_next = h * fac;
    }
    if (ok) {
      S.t = landing ? t_land : t + h;
#pragma unroll
      for (int c = 0; c < 4; ++c) S.y[c] = yn[c];
      S.g_old = g_new;
    } else {
      ++S.rejected;
      if (h <= P.min_step) {
        S.status = conv_fail_here ? ST_CONV_FAIL : ST_STEP_LIMIT;
        S.active = false;
        S.h = h_next;
        return false;
      }
    }
    S.h = h_next;
    // dense output decision (stepper.py:634-645, stored slot never overwritten)
    if (P.dense_mode == 0) {
      store = (S.idx < P.ndo) && (S.dnext <= S.t);
    } else {
      store = ok && landing;
    }
    // termination (stepper.py:651-662): evaluated after the caller stores
  }
  return store;
}

// After a dense store (if any): advance the schedule and test termination.
__device__ __forceinline__ void after_store(LaneState& S, const Params& P, bool stored) {
  if (!S.active) return;
  if (stored) {
    S.idx += 1;
    if (P.dense_mode == 0) {
      const double nx = S.t + S.ddt;
      S.dnext = nx < S.t_end ? nx : S.t_end;
    }
  }
  if (S.t >= S.t_end) {
    S.status = ST_SUCCESS;
    S.active = false;
  } else if (fabs(S.g_old) < P.etol) {
    S.status = ST_EVENT;
    S.active = false;
  }
}

}  // namespace cbc
