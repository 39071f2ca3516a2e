// ckm1d_core.cuh -- per-lane CKM1D right-hand side and Cash-Karp step for sm_100a.
//
// Execution model: one lane per bubble.  A system of K bubbles occupies K
// consecutive lanes of a warp ("group"); a warp holds floor(32/K) systems.
// Everything that couples bubbles (coupling terms, the implicit-coupling
// iteration, reductions for norms, error ratio and the collision event) is
// exchanged inside the warp -- full-warp __shfl_sync, or per-warp
// shared-memory records ordered by __syncwarp (partner states; the iterates
// for K > 8) -- so no block barrier and no shared-memory atomics are needed
// (the reference synchronises the
// whole block 4x per Richardson iteration, ckm1d_def.py:303-404).  Control flow
// that contains shuffles is warp-uniform; per-system decisions only select
// values.  Per-system scalars (t, h, event value, ...) are held redundantly by
// every lane of the group and stay identical because every lane computes them
// from the same shuffled inputs.
//
// Canonical evaluation order (shared with oracle/ckm1d_oracle.cpp):
//   * pair sums of bubble i run over the partners j = (i + d) mod K,
//     d = 1 .. K-1 (every lane does useful work in every iteration; no
//     masked diagonal term);
//   * sums over the bubbles of a system (norms of the implicit-coupling
//     iteration) are pairwise trees over the next power of two, zero padded;
//   * min / all reductions are order independent.
// Numerics: FP64 throughout, compiled with -fmad=false; every fused
// multiply-add is an explicit fma() and the elementary functions come from
// cbc_math.h, so results equal the CPU oracle bit for bit.  The algorithm
// restates coupledbubble_control/backends/numba/sysmtem_definitions/ckm1d_def.py
// (acoustic_field_1d :79-114, ode_fun :408-497, explicit_coupling :164-246,
// mat_vec_product :250-299, implicit_coupling :303-404, event_fun :499-556) and
// rkck45_coupled_numba_stepper.py (:362-677).
//
// Per-warp shared memory (WarpSmem): the group's harmonic constants, the
// lane's 13 bubble constants (+2 derived) and the six stage derivatives.
// Keeping these out of registers lets more warps stay resident.
#pragma once

#include <stdint.h>
#include <string.h>
#include <utility>
#include "cbc_math.h"

namespace cbc {

constexpr unsigned FULL = 0xffffffffu;
constexpr int NKMAX = 4;                        // harmonic components supported
constexpr int HC_PER_K = 7;                     // per-harmonic constants
constexpr int NUPS = 15;                        // 13 bubble constants + up7/3 + up4*up7
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

// Stage tableau for the stage loop: row s (1..5) combines k_1..k_s.
static __constant__ double kStageA[6] = {0.0, A2, A3, A4, A5, A6};
static __constant__ double kStageB[6][5] = {{0, 0, 0, 0, 0},
                                     {B21, 0, 0, 0, 0},
                                     {B31, B32, 0, 0, 0},
                                     {B41, B42, B43, 0, 0},
                                     {B51, B52, B53, B54, 0},
                                     {B61, B62, B63, B64, B65}};

// Resident 128-thread blocks per SM the register allocation is tuned for, per
// lanes-per-system instantiation (ptxas: KB=2 fits 128 registers and KB=4 168
// without spills; KB=8 needs ~250; KB >= 16 keeps its pair arrays in local
// memory either way).
__host__ __device__ constexpr int min_blocks_for(int KB) { return KB <= 2 ? 4 : (KB <= 4 ? 3 : (KB <= 8 ? 2 : 1)); }

// Register-budget variant MB of the batched kernels: MB = 1 asks ptxas for one
// more resident 128-thread block per SM (fewer registers per thread, possibly
// spills; more warps to hide latency).  The autotuner measures which is
// faster.  K > 8 kernels are limited by shared memory and have only MB = 0.
__host__ __device__ constexpr int min_blocks_variant(int KB, int MB) { return min_blocks_for(KB) + (KB <= 8 ? MB : 0); }

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
  int lin;         // implicit-coupling solver: LIN_RICHARDSON or LIN_LU
};

// Position of this lane inside its system group.
struct Geo {
  int K;       // bubbles per system (warp-uniform)
  int G;       // groups per warp = 32 / K
  int grp;     // group index (clamped to a valid slot for idle lanes)
  int base;    // first lane of the group
  int li;      // bubble index of this lane
  int lane;
  bool valid;  // lane belongs to a group
};

// slots: systems a warp holds at most (fewer than 32 / K leaves lanes idle:
// less intra-warp divergence for fewer systems in flight; a tuning knob).
__device__ __forceinline__ Geo make_geo(int K, int slots = 32) {
  Geo g;
  const int lane = threadIdx.x & 31;
  g.lane = lane;
  g.K = K;
  g.G = 32 / K;                          // layout of the group regions (unchanged by slots)
  const int grp = lane / K;
  g.valid = grp < g.G && grp < slots;    // groups past `slots` stay idle
  g.grp = g.valid ? grp : 0;
  g.base = g.valid ? grp * K : lane;
  g.li = g.valid ? lane - grp * K : 0;
  return g;
}

__device__ __forceinline__ double shfl(double v, int src) { return __shfl_sync(FULL, v, src); }

// Source lane of partner d (1 <= d < K) of this lane: bubble (li + d) mod K.
__device__ __forceinline__ int partner_lane(const Geo& g, int d) {
  int j = g.li + d;
  if (j >= g.K) j -= g.K;
  return g.base + j;
}

// The same for shared-memory exchange records: lanes outside every group read
// their own record (always inside the warp's 32 records).
__device__ __forceinline__ int partner_rec(const Geo& g, int d) { return g.valid ? partner_lane(g, d) : g.lane; }

// Open pairwise tree over a[0..n-1] (n <= N): at width w, a[i] += a[i + w]
// for i a multiple of 2w with i + w < n; a lone last element is carried up.
// ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + a6).  0.0 for n = 0.  For
// non-negative terms it equals the zero-padded tree of group_sum.
template <int N>
__device__ __forceinline__ double tree_open(double (&a)[N], int n) {
#pragma unroll
  for (int w = 1; w < N; w <<= 1) {
#pragma unroll
    for (int i = 0; i + w < N; i += 2 * w)
      if (i + w < n) a[i] = a[i] + a[i + w];
  }
  return n > 0 ? a[0] : 0.0;
}

// Per-warp shared-memory carve-up, in doubles.
struct WarpSmem {
  double* hc;   // [7 nk][G]   harmonic constants of each group (component-major)
  double* up;   // [15][32]    bubble constants, lane-private columns
  double* ks;   // [6][4][32]  stage derivatives, lane-private columns
  double* xv;   // [2][32] double2 partner-state exchange records
  double* cm;   // [3][K-1][32] coupling coefficients of each lane's partners d = 1..K-1
  double* mat;  // implicit-coupling matrix rows (see mat_doubles), lane-private columns
  double* pv;   // [G][2K+1] pivot-row snapshot of each group (direct solve, K > 8)
};

constexpr int XV_DOUBLES = 4 * 32;

// Linear solvers of the implicit coupling system.
enum : int { LIN_RICHARDSON = 0, LIN_LU = 1 };

// Harmonic-constant region rounded up to an even count, so that every later
// region (and every warp's carve-up) stays 16-byte aligned for double2 access.
__host__ __device__ inline int hc_doubles(int K, int nk) { return (HC_PER_K * nk * (32 / K) + 1) & ~1; }

// Matrix region per warp:
//   Richardson, K <= 8: none (the partner coefficients live in registers);
//   Richardson, K > 8:  the partner coefficients as double2 records
//                       [K-1][(A,B), (C,D)][32] (kept out of registers: local
//                       memory would spill to L2);
//   direct, K <= 8:     staging of the four coefficient blocks by absolute
//                       column, [4][K][32], read back into register rows;
//   direct, K > 8:      the two augmented rows of every lane, [2][2K+1][32].
__host__ __device__ inline int mat_doubles(int K, int lin) {
  if (K <= 8) return lin == LIN_LU ? 4 * K * 32 : 0;
  return lin == LIN_LU ? 2 * (2 * K + 1) * 32 : 4 * (K - 1) * 32;
}
__host__ __device__ inline int pv_doubles(int K, int lin) {
  return (K > 8 && lin == LIN_LU) ? (((32 / K) * (2 * K + 1) + 1) & ~1) : 0;
}

__host__ __device__ inline int smem_doubles_per_warp(int K, int nk, int lin = LIN_RICHARDSON) {
  return hc_doubles(K, nk) + NUPS * 32 + 24 * 32 + XV_DOUBLES + 3 * (K - 1) * 32 + mat_doubles(K, lin) +
         pv_doubles(K, lin);
}

__device__ __forceinline__ WarpSmem warp_smem(double* base, int K, int nk, int lin = LIN_RICHARDSON) {
  WarpSmem w;
  double* p = base + (threadIdx.x >> 5) * smem_doubles_per_warp(K, nk, lin);
  w.hc = p;
  w.up = p + hc_doubles(K, nk);
  w.ks = w.up + NUPS * 32;
  w.xv = w.ks + 24 * 32;
  w.cm = w.xv + XV_DOUBLES;
  w.mat = w.cm + 3 * (K - 1) * 32;
  w.pv = w.mat + mat_doubles(K, lin);
  return w;
}

// Coupling matrices of this lane's system: M(c, j, i=this lane) = m[c*sc + j*sj]
struct MView {
  const double* __restrict__ m;  // points at M(0, 0, i)
  long long sc, sj;
};

// Copies this lane's coupling coefficients M(c, j, i) for its partners
// j = (i + d) mod K, d = 1..K-1, into shared memory: they are constant for the
// whole solve and are read every RHS evaluation.
__device__ __forceinline__ void store_coupling(const WarpSmem& w, const Geo& g, const MView& M) {
  for (int d = 1; d < g.K; ++d) {
    const int j = partner_lane(g, d) - g.base;
#pragma unroll
    for (int c = 0; c < 3; ++c) w.cm[(c * (g.K - 1) + d - 1) * 32 + g.lane] = M.m[c * M.sc + j * M.sj];
  }
}

__device__ __forceinline__ double cmv(const WarpSmem& w, const Geo& g, int c, int d) {
  return w.cm[(c * (g.K - 1) + d - 1) * 32 + g.lane];
}

// Per-lane integrator state (bubble + copies of the system scalars).
struct LaneState {
  double y[4];                 // R, X, U, V
  double sp0, sp3;             // 3 gamma, c
  double t, t_end, t_begin, h, g_old;
  double dnext, ddt;           // dense schedule (next sample time, spacing)
  int idx;                     // dense samples stored
  int status;
  bool active;
  int steps, rejected, conv_ok, conv_fail;
  long long lin_iters;
};

// Writes this lane's bubble constants (13 from the caller, 2 derived).
__device__ __forceinline__ void store_bubble_consts(const WarpSmem& w, const Geo& g, const double* up13,
                                                    long long stride) {
  double* u = w.up + g.lane;
#pragma unroll
  for (int p = 0; p < 13; ++p) u[p * 32] = up13[p * stride];
  u[13 * 32] = u[7 * 32] * (1.0 / 3.0);
  u[14 * 32] = u[4 * 32] * u[7 * 32];
}

__device__ __forceinline__ double upv(const WarpSmem& w, const Geo& g, int p) { return w.up[p * 32 + g.lane]; }

// Per-system harmonic constants, component-major: hc[(7k + c) * G + grp].
//   c = 0 w0*omega, 1 phase, 2 l0*wave, 3 PA, 4 PA*omega, 5 PA*wave, 6 PA*u0
// Written by lane 0 of the group from system parameters sp1 = 1/omega_ref,
// sp2 = lambda_ref/2pi, sp4 = 1/(rho c) and the control parameters
// cp[m * cp_stride], m = 0..4nk-1 (PA, omega, phase, wave number).
__device__ __forceinline__ void store_harmonics(const WarpSmem& w, const Geo& g, double sp1, double sp2,
                                                double sp4, const double* cp, int nk,
                                                long long cp_stride) {
  // acoustic_field_1d (ckm1d_def.py:95-97): w0 = 2pi sp[1], l0 = 2pi sp[2], u0 = sp[4]
  const double w0 = TWO_PI * sp1;
  const double l0 = TWO_PI * sp2;
  const double u0 = sp4;
  for (int k = 0; k < nk; ++k) {
    const double amps = cp[k * cp_stride], omega = cp[(nk + k) * cp_stride],
                 phase = cp[(2 * nk + k) * cp_stride], wave = cp[(3 * nk + k) * cp_stride];
    double* h = w.hc + (HC_PER_K * k) * g.G + g.grp;
    h[0 * g.G] = w0 * omega;
    h[1 * g.G] = phase;
    h[2 * g.G] = l0 * wave;
    h[3 * g.G] = amps;
    h[4 * g.G] = amps * omega;
    h[5 * g.G] = amps * wave;
    h[6 * g.G] = amps * u0;
  }
}

__device__ __forceinline__ double hcv(const WarpSmem& w, const Geo& g, int k, int c) {
  return w.hc[(HC_PER_K * k + c) * g.G + g.grp];
}

// Pairwise-tree sum of v over the group (next power of two, zero padded):
// every lane ends with ((v0 + v1) + (v2 + v3)) + ...  At level w each lane
// holds the sum of its aligned block of w bubbles; the partner block starts
// at q = (li ^ w) & ~(w - 1) and is read from its first lane (which exists
// unless the whole block is padding, then it contributes +0.0).  IEEE
// addition is commutative, so both blocks of a pair compute the same sum.
template <int KB>
__device__ __forceinline__ double group_sum(double v, const Geo& g) {
#pragma unroll
  for (int w = 1; w < KB; w <<= 1) {
    if (w < g.K) {
      const int q = (g.li ^ w) & ~(w - 1);
      double x = shfl(v, g.base + (q < g.K ? q : g.li));
      if (q >= g.K) x = 0.0;
      v = v + x;
    }
  }
  return v;
}

// Minimum over the group (order independent; NaN never wins).
template <int KB>
__device__ __forceinline__ double group_min(double v, const Geo& g) {
#pragma unroll
  for (int w = 1; w < KB; w <<= 1) {
    if (w < g.K) {
      const int q = (g.li ^ w) & ~(w - 1);
      const double x = shfl(v, g.base + (q < g.K ? q : g.li));
      if (q < g.K && x < v) v = x;
    }
  }
  return v;
}

// AND of a per-lane predicate over the group.
__device__ __forceinline__ bool group_all(bool p, const Geo& g) {
  const unsigned bad = __ballot_sync(FULL, !p);
  const unsigned gm = (g.K >= 32) ? FULL : (((1u << g.K) - 1u) << g.base);
  return (bad & gm) == 0u;
}

// event_fun (ckm1d_def.py:499-556): min over neighbours of
// |x_i - x_{i+1}| - (R_i R0_i + R_{i+1} R0_{i+1}) / lambda * (1 + threshold),
// 1e30 for a single bubble.
template <int KB>
__device__ __forceinline__ double group_event(const double y[4], double up12, const Geo& g, double col) {
  const double ri = y[0] * up12;
  const double rj = __shfl_down_sync(FULL, ri, 1);
  const double xj = __shfl_down_sync(FULL, y[1], 1);
  double gap = 1e30;
  if (g.li + 1 < g.K) gap = fabs(y[1] - xj) - (ri + rj) * col;
  // a sequential "if (gap < m) m = gap" scan from 1e30 ignores NaN and values
  // >= 1e30; clamp first so that the tree reduction agrees with it
  if (!(gap < 1e30)) gap = 1e30;
  return group_min<KB>(gap, g);
}

// RHS of the whole system, evaluated by its K lanes: dy of this lane's bubble.
// Returns via conv/iters the outcome of the implicit-coupling iteration.
// Group sum with butterfly shuffles, for groups of exactly KB lanes (KB a
// power of two, groups aligned to KB): the same pairwise tree as group_sum.
template <int KB>
__device__ __forceinline__ double group_sum_full(double v) {
#pragma unroll
  for (int w = 1; w < KB; w <<= 1) v = v + __shfl_xor_sync(FULL, v, w);
  return v;
}

// Residual r = b - A v of the implicit coupling system for this lane's bubble,
// A = I + off-diagonal partner blocks.  Partner distance d = 1..K-1 goes to
// accumulation chain (d - 1) mod 4 (increasing d within a chain); the chains
// are then combined by the open pairwise tree.  Coefficients from registers
// (K <= 8) or from the lane's shared-memory columns (K > 8).
template <int KB>
__device__ __forceinline__ void residual(const Geo& g, const double* Am, const double* Bm, const double* Cm,
                                         const double* Dm, double cpf0, double b0, double b1, double vr,
                                         double vt, double& r0, double& r1) {
  double ar[4] = {0.0, 0.0, 0.0, 0.0}, at[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 1; d < KB; ++d)
    if (d < g.K) {
      const int src = partner_lane(g, d);
      const double vrj = shfl(vr, src), vtj = shfl(vt, src);
      const int c = (d - 1) & 3;
      ar[c] = fma(Am[d], vrj, fma(Bm[d], vtj, ar[c]));
      at[c] = fma(Cm[d], vrj, fma(Dm[d], vtj, at[c]));
    }
  const int nc = g.K - 1 < 4 ? g.K - 1 : 4;
  const double sr = tree_open(ar, nc);
  const double st = tree_open(at, nc);
  r0 = b0 - fma(sr, cpf0, vr);
  r1 = b1 - (st + vt);
}

// The same for K > 8, from shared memory: the coefficients of partner
// distance d as two double2 records per lane, (A, B) at [(d - 1) 2][lane] and
// (C, D) at [(d - 1) 2 + 1][lane]; the partner iterates through the warp's
// exchange records (one 16-byte store per lane and one 16-byte load per
// partner, instead of two 64-bit shuffles per partner).  Same values and the
// same accumulation order as the register form.
template <int KB>
__device__ __forceinline__ void residual_smem(const Geo& g, const WarpSmem& W, double cpf0, double b0, double b1,
                                              double vr, double vt, double& r0, double& r1) {
  double ar[4] = {0.0, 0.0, 0.0, 0.0}, at[4] = {0.0, 0.0, 0.0, 0.0};
  const double2* m2 = reinterpret_cast<const double2*>(W.mat) + g.lane;
  double2* xr = reinterpret_cast<double2*>(W.xv);
  __syncwarp();
  xr[g.lane] = make_double2(vr, vt);
  __syncwarp();
#pragma unroll
  for (int d = 1; d < KB; ++d)
    if (d < g.K) {
      const double2 vj = xr[partner_rec(g, d)];
      const int c = (d - 1) & 3;
      const double2 ab = m2[(2 * (d - 1)) * 32], cd = m2[(2 * (d - 1) + 1) * 32];
      ar[c] = fma(ab.x, vj.x, fma(ab.y, vj.y, ar[c]));
      at[c] = fma(cd.x, vj.x, fma(cd.y, vj.y, at[c]));
    }
  const int nc = g.K - 1 < 4 ? g.K - 1 : 4;
  const double sr = tree_open(ar, nc);
  const double st = tree_open(at, nc);
  r0 = b0 - fma(sr, cpf0, vr);
  r1 = b1 - (st + vt);
}

// ---- direct solve of the implicit coupling system (lin_solver = LU) --------
// Unknowns x = (vr_0..vr_{K-1}, vt_0..vt_{K-1}); row R_i (index i) and row T_i
// (index K + i) are held by lane i:
//   R_i: x_i + cpf0_i sum_j (A_ij vr_j + B_ij vt_j) = b0_i
//   T_i: x_{K+i} + sum_j (C_ij vr_j + D_ij vt_j)    = b1_i
// Gauss-Jordan elimination with partial pivoting, column c = 0..2K-1:
//   p   = the not-yet-pivot row with the largest pivot key (piv_key32: |a[r][c]|
//         at 2^-13 relative resolution, NaN lowest, ties to the smaller row;
//         a warp-shuffle max-reduction over the system's lanes);
//   rp  = 1 / a[p][c];  pk[k] = a[p][k] for k = c+1..2K (k = 2K: right side);
//   every row r: l = (r == p) ? 0 : a[r][c] * rp,  a[r][k] = fma(-l, pk[k], a[r][k]).
// Pivot rows are eliminated too (Gauss-Jordan), so x_c = a[p_c][2K] * rp_c
// with no triangular back-substitution pass.  ok = every pivot nonzero and
// finite.  oracle/ckm1d_oracle.cpp (lu_solve) performs the same operations.
// Pivot key of row r (0 <= r < 128) for column c: the high 32 bits of
// |a[r][c]| (sign, exponent and 20 mantissa bits) with the low 7 bits replaced
// by 127 - r.  The pivot is the row with the largest key: the largest
// magnitude at 2^-13 relative resolution, ties to the smaller row; NaN ranks
// below every number and rows that are already pivots have key 0.  One 32-bit
// integer per row, so the argmax over a system's lanes is a max-reduction of
// single shuffles.
__host__ __device__ inline unsigned piv_key32(double v, int r, bool pivoted) {
  unsigned long long b;
  memcpy(&b, &v, sizeof b);
  b &= 0x7FFFFFFFFFFFFFFFull;
  unsigned hi = (unsigned)(b >> 32);
  if (b > 0x7FF0000000000000ull) hi = 0u;    // NaN
  return pivoted ? 0u : ((hi & ~127u) | (unsigned)(127 - r));
}

// Maximum of a key over the group (any K), the same in every lane.
template <int KB>
__device__ __forceinline__ unsigned group_max_u32(unsigned k, const Geo& g) {
#pragma unroll
  for (int w = 1; w < KB; w <<= 1) {
    if (w < g.K) {
      const int q = (g.li ^ w) & ~(w - 1);
      const unsigned o = __shfl_sync(FULL, k, g.base + (q < g.K ? q : g.li));
      if (q < g.K) k = o > k ? o : k;
    }
  }
  return k;
}

// Register rows, exact K <= 8 known at compile time (every index static: the
// column steps are expanded by template recursion, so the rows never leave
// registers).  The four coefficient blocks were staged by absolute column in
// W.mat.
struct LuTrack {
  bool pR, pT;       // this lane's rows R / T already pivot rows
  int srcR, srcT;    // pivot rows of columns li and K + li
  double rpR, rpT;   // their reciprocal pivots
  bool ok;
};

template <int KC, int C>
__device__ __forceinline__ void lu_column(const Geo& g, double (&rR)[2 * KC], double (&rT)[2 * KC], double& hR,
                                          double& hT, LuTrack& t) {
  constexpr int K = KC, N = 2 * KC;
  const int li = g.li;
  const unsigned kR = piv_key32(rR[C], li, t.pR), kT = piv_key32(rT[C], K + li, t.pT);
  const unsigned km = group_max_u32<(KC <= 2 ? 2 : (KC <= 4 ? 4 : 8))>(kR > kT ? kR : kT, g);
  const int p = 127 - (int)(km & 127u);
  const bool ps = p >= K;
  const int src = g.base + (ps ? p - K : p);
  const double piv = shfl(ps ? rT[C] : rR[C], src);
  t.ok = t.ok && (piv != 0.0) && cbcm::isfinite_(piv);
  const double rp = 1.0 / piv;
  const bool meR = (p == li), meT = (p == K + li);
  t.pR = t.pR || meR;
  t.pT = t.pT || meT;
  t.srcR = (C == li) ? p : t.srcR;
  t.rpR = (C == li) ? rp : t.rpR;
  t.srcT = (C == K + li) ? p : t.srcT;
  t.rpT = (C == K + li) ? rp : t.rpT;
  const double lR = meR ? 0.0 : rR[C] * rp;
  const double lT = meT ? 0.0 : rT[C] * rp;
  // The pivot row is almost always the diagonal row C (the matrix is the
  // identity plus the coupling terms): when it is for every system of the
  // warp, its owner lane and row are compile-time constants and the row is
  // broadcast without selects.  Both branches move the same values.
  if (__all_sync(FULL, (p == C) || !g.valid)) {
    constexpr bool DS = C >= K;
    const int dsrc = g.base + (DS ? C - K : C);
#pragma unroll
    for (int k = C + 1; k < N; ++k) {
      const double pk = shfl(DS ? rT[k] : rR[k], dsrc);
      rR[k] = fma(-lR, pk, rR[k]);
      rT[k] = fma(-lT, pk, rT[k]);
    }
    const double ph = shfl(DS ? hT : hR, dsrc);
    hR = fma(-lR, ph, hR);
    hT = fma(-lT, ph, hT);
  } else {
#pragma unroll
    for (int k = C + 1; k < N; ++k) {
      const double pk = shfl(ps ? rT[k] : rR[k], src);
      rR[k] = fma(-lR, pk, rR[k]);
      rT[k] = fma(-lT, pk, rT[k]);
    }
    const double ph = shfl(ps ? hT : hR, src);
    hR = fma(-lR, ph, hR);
    hT = fma(-lT, ph, hT);
  }
}

template <int KC, int... Cs>
__device__ __forceinline__ void lu_columns(const Geo& g, double (&rR)[2 * KC], double (&rT)[2 * KC], double& hR,
                                           double& hT, LuTrack& t, std::integer_sequence<int, Cs...>) {
  (lu_column<KC, Cs>(g, rR, rT, hR, hT, t), ...);
}

template <int KC>
__device__ __forceinline__ void lu_solve_reg(const Geo& g, const WarpSmem& W, double cpf0, double b0, double b1,
                                             double& xr, double& xt, bool& ok) {
  constexpr int K = KC, N = 2 * KC;
  const int li = g.li;
  const double* m = W.mat + g.lane;
  double rR[N], rT[N];
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const bool dg = (j == li);
    rR[j] = dg ? 1.0 : cpf0 * m[(0 * K + j) * 32];
    rR[K + j] = dg ? 0.0 : cpf0 * m[(1 * K + j) * 32];
    rT[j] = dg ? 0.0 : m[(2 * K + j) * 32];
    rT[K + j] = dg ? 1.0 : m[(3 * K + j) * 32];
  }
  double hR = b0, hT = b1;
  LuTrack t{false, false, 0, 0, 0.0, 0.0, true};
  lu_columns<KC>(g, rR, rT, hR, hT, t, std::make_integer_sequence<int, N>{});
  ok = t.ok;
  // x_c = h[p_c] * rp_c; this lane needs columns li and K + li
  const int oR = g.base + (t.srcR >= K ? t.srcR - K : t.srcR), oT = g.base + (t.srcT >= K ? t.srcT - K : t.srcT);
  const double aR = shfl(hR, oR), aT = shfl(hT, oR);
  const double cR = shfl(hR, oT), cT = shfl(hT, oT);
  xr = (t.srcR >= K ? aT : aR) * t.rpR;
  xt = (t.srcT >= K ? cT : cR) * t.rpT;
}

// Shared-memory rows for K > 8 (K read at run time): lane column k of row
// R at W.mat[k 32 + lane], of row T at W.mat[(RS + k) 32 + lane], RS = 2K + 1,
// right side at k = 2K.  The pivot row is first copied to the group's
// snapshot W.pv, so every row (the pivot row included) is updated from its
// values before the column, exactly as the register form reads them.
template <int KB>
__device__ __forceinline__ void lu_solve_smem(const Geo& g, const WarpSmem& W, double& xr, double& xt, bool& ok) {
  const int K = g.K, N = 2 * K, RS = N + 1;
  const int li = g.li;
  double* mR = W.mat + g.lane;
  double* mT = W.mat + RS * 32 + g.lane;
  double* pv = W.pv + g.grp * RS;
  bool pR = false, pT = false;
  int srcR = 0, srcT = 0;
  double rpR = 0.0, rpT = 0.0;
  ok = true;
#pragma unroll 1
  for (int c = 0; c < N; ++c) {
    __syncwarp();
    const double vR = mR[c * 32], vT = mT[c * 32];
    const unsigned kR = piv_key32(vR, li, pR), kT = piv_key32(vT, K + li, pT);
    const unsigned km = group_max_u32<KB>(kR > kT ? kR : kT, g);
    const int p = 127 - (int)(km & 127u);
    // the pivot value from its owner's column (lanes outside every group
    // read their own column)
    const int own = g.valid ? g.base + (p >= K ? p - K : p) : g.lane;
    const double piv = W.mat[(p >= K ? RS * 32 : 0) + c * 32 + own];
    ok = ok && (piv != 0.0) && cbcm::isfinite_(piv);
    const double rp = 1.0 / piv;
    const bool meR = (p == li), meT = (p == K + li);
    pR = pR || meR;
    pT = pT || meT;
    srcR = (c == li) ? p : srcR;
    rpR = (c == li) ? rp : rpR;
    srcT = (c == K + li) ? p : srcT;
    rpT = (c == K + li) ? rp : rpT;
    // snapshot of the pivot row (its owner copies it)
    if (g.valid && (meR || meT)) {
      const double* own = meR ? mR : mT;
      for (int k = c + 1; k <= N; ++k) pv[k] = own[k * 32];
    }
    __syncwarp();
    const double lR = meR ? 0.0 : vR * rp;
    const double lT = meT ? 0.0 : vT * rp;
#pragma unroll 4
    for (int k = c + 1; k <= N; ++k) {
      const double pk = pv[k];
      mR[k * 32] = fma(-lR, pk, mR[k * 32]);
      mT[k * 32] = fma(-lT, pk, mT[k * 32]);
    }
  }
  __syncwarp();
  // lanes outside every group read their own column (always in range)
  const int oR = g.valid ? g.base + (srcR >= K ? srcR - K : srcR) : g.lane;
  const int oT = g.valid ? g.base + (srcT >= K ? srcT - K : srcT) : g.lane;
  xr = W.mat[(srcR >= K ? RS * 32 : 0) + N * 32 + oR] * rpR;
  xt = W.mat[(srcT >= K ? RS * 32 : 0) + N * 32 + oT] * rpT;
}

// Right-hand side for one field form: NKC harmonics and field type ACC
// known at compile time (NKC = 0, ACC = -1: both read from P).  With both
// fixed the harmonic loops have no branches, so the independent sin/cos,
// log/exp and division chains of the bubble interleave.
template <int KB, int KC, int LIN, int NKC, int ACC>
__device__ __forceinline__ void rhs_form(const Geo& g, const Params& P, const WarpSmem& W, const MView& M,
                                         double sp0, double sp3, bool on, double t, const double y[4],
                                         double dy[4], bool& conv, int& iters) {
  const int nk = NKC > 0 ? NKC : P.nk;
  const int ac = ACC >= 0 ? ACC : P.ac;
  const int K = g.K;
  const int li = g.li;
  const double x0 = y[0], x1 = y[1], x2 = y[2], x3 = y[3];

  // ---- time harmonics (system-uniform): lane k computes harmonic k ----
  double st[NKMAX], ct[NKMAX];
  if (nk <= K) {
    const int k = li < nk ? li : 0;
    double s_, c_;
    cbcm::sincos(fma(hcv(W, g, k, 0), t, hcv(W, g, k, 1)), &s_, &c_);
#pragma unroll
    for (int kk = 0; kk < NKMAX; ++kk)
      if (kk < nk) {
        st[kk] = shfl(s_, g.base + kk);
        ct[kk] = shfl(c_, g.base + kk);
      }
  } else {
#pragma unroll
    for (int kk = 0; kk < NKMAX; ++kk)
      if (kk < nk) cbcm::sincos(fma(hcv(W, g, kk, 0), t, hcv(W, g, kk, 1)), &st[kk], &ct[kk]);
  }

  // ---- uncoupled Keller--Miksis + translation (ckm1d_def.py:418-447) ----
  const double rx0 = 1.0 / x0;
  const double p = cbcm::pow_pos(rx0, sp0);
  double pa = 0.0, pt = 0.0, px = 0.0, ux = 0.0;
#pragma unroll
  for (int k = 0; k < NKMAX; ++k) {
    if (k < nk) {
      const double a = hcv(W, g, k, 3), aw = hcv(W, g, k, 4);
      if (ac == 0) {  // CONST
        pa = fma(a, st[k], pa);
        pt = fma(aw, ct[k], pt);
      } else {
        double sx, cx;
        cbcm::sincos(fma(hcv(W, g, k, 2), x1, hcv(W, g, k, 1)), &sx, &cx);
        const double awv = hcv(W, g, k, 5), au = hcv(W, g, k, 6);
        if (ac == 1) {  // SW_N
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

  // ---- explicit coupling + matrix of the implicit system over partners ----
  // The partner coefficients A, B, C, D of the implicit system go to
  // registers (Richardson, K <= 8), to the lane's shared-memory columns by
  // partner distance (Richardson, K > 8) or by absolute partner column (the
  // direct solve: its staging area for K <= 8, its augmented rows for K > 8).
  constexpr bool REG = (KB <= 8) && (LIN == LIN_RICHARDSON);
  double g0 = 0.0, g1 = 0.0, tn = 0.0, tg2 = 0.0, tg3 = 0.0;
  double Am[REG ? KB : 1], Bm[REG ? KB : 1], Cm[REG ? KB : 1], Dm[REG ? KB : 1];
  double* mcol = W.mat + g.lane;
  const int RS = 2 * K + 1;
  // partner states through the exchange records
  double2* xv2 = reinterpret_cast<double2*>(W.xv);
  __syncwarp();
  xv2[g.lane] = make_double2(x0, x1);
  xv2[32 + g.lane] = make_double2(x2, x3);
  __syncwarp();
#pragma unroll
  for (int d = 1; d < KB; ++d) {
    if constexpr (REG) {
      Am[d] = 0.0;
      Bm[d] = 0.0;
      Cm[d] = 0.0;
      Dm[d] = 0.0;
    }
    if (d < K) {
      const int src = partner_rec(g, d);
      // partner state; its coupling terms are recomputed exactly as the
      // owning lane computes them (cheaper than exchanging seven terms)
      const double2 xa = xv2[src], xb = xv2[32 + src];
      const double xj0 = xa.x, xj1 = xa.y, xj2 = xb.x, xj3 = xb.y;
      // evaluated for every lane (no branch): lanes of finished systems
      // compute terms that are never used
      {
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
        const double m0 = cmv(W, g, 0, d);
        const double m1 = cmv(W, g, 1, d);
        const double m2 = cmv(W, g, 2, d);
        double t0 = fma(2.5 * srd2, h2j, rd3 * h4j);
        t0 = fma(2.0 * rd, h0j, t0);
        g0 = fma(-m0, t0, g0);
        const double t1 = fma(srd2, h1j, rd3 * h3j);
        g1 = fma(-0.5 * m0, t1, g1);
        const double t2 = fma(2.0 * srd2, h0j, (5.0 * rd3) * h2j);
        tn = fma(m1, t2, tn);
        tg2 = fma(m1, t1, tg2);
        tg3 = fma(m2, t1, tg3);
        const double a_ = (m0 * rd) * j02;
        const double b_ = ((0.5 * m0) * srd2) * j03;
        const double c_ = -((m1 * srd2) * j02);
        const double d_ = -((m1 * rd3) * j03);
        if constexpr (REG) {
          Am[d] = a_;
          Bm[d] = b_;
          Cm[d] = c_;
          Dm[d] = d_;
        } else if constexpr (LIN == LIN_RICHARDSON) {
          double2* mcol2 = reinterpret_cast<double2*>(W.mat) + g.lane;
          mcol2[(2 * (d - 1)) * 32] = make_double2(a_, b_);
          mcol2[(2 * (d - 1) + 1) * 32] = make_double2(c_, d_);
        } else {
          const int j = partner_lane(g, d) - g.base;   // absolute partner column
          if constexpr (KB <= 8) {
            mcol[(0 * K + j) * 32] = a_;
            mcol[(1 * K + j) * 32] = b_;
            mcol[(2 * K + j) * 32] = c_;
            mcol[(3 * K + j) * 32] = d_;
          } else {
            mcol[j * 32] = a_;              // row R (scaled by cpf0 below)
            mcol[(K + j) * 32] = b_;
            mcol[(RS + j) * 32] = c_;       // row T
            mcol[(RS + K + j) * 32] = d_;
          }
        }
      }
    }
  }
  // Keller--Miksis numerator / denominator of this bubble (after the partner
  // loop in program order, so that the division and log/exp chain feeding p
  // overlaps with the partner terms)
  const double u7 = upv(W, g, 7);
  const double q = fma(u7, x2, 1.0);
  double N = fma(upv(W, g, 1), x2, upv(W, g, 0)) * p;
  N = fma(-upv(W, g, 2), q, N);
  N = fma(-upv(W, g, 3), rx0, N);
  N = fma(-(upv(W, g, 4) * x2), rx0, N);
  const double w = fma(-upv(W, g, 13), x2, 1.0);
  N = fma((-1.5 * w) * x2, x2, N);
  N = fma(-(q * upv(W, g, 5)), pa, N);
  N = fma(-(upv(W, g, 6) * pt), x0, N);
  N = fma(upv(W, g, 8) * x3, x3, N);
  const double D = fma(-(u7 * x0), x2, x0) + upv(W, g, 14);
  const double rD = 1.0 / D;
  const double x02 = x0 * x0;
  const double x03 = x02 * x0;
  const double Fb1 = -(upv(W, g, 10) * x03) * px;
  const double Fd = -(upv(W, g, 11) * x0) * fma(x3, sp3, -ux);
  const double rx03 = (rx0 * rx0) * rx0;
  double b0 = N * rD;
  double b1 = fma((3.0 * (Fb1 + Fd)) * upv(W, g, 9), rx03, -(((3.0 * x2) * rx0) * x3));
  const double cpf0 = rD, cpf1 = x3 * rD, cpf2 = x2 * rx0, cpf3 = rx0 * rx0;
  b0 = fma(g0, cpf0, fma(g1, cpf1, b0));
  b1 = b1 + fma(tg2, cpf2, fma(tg3, cpf3, tn));

  if constexpr (LIN == LIN_LU) {
    // ---- implicit coupling: direct solve (Gauss-Jordan, partial pivoting) ----
    // (the exact K is a compile-time constant whenever K <= 8)
    static_assert(KB > 8 || KC > 0, "the register form needs the exact K");
    double xr, xt;
    bool okd;
    if constexpr (KB <= 8) {
      lu_solve_reg<(KC > 0 ? KC : 1)>(g, W, cpf0, b0, b1, xr, xt, okd);
    } else {
      // finish the augmented rows: scale row R by cpf0, diagonal, right sides
      for (int j = 0; j < K; ++j) {
        if (j == li) continue;
        mcol[j * 32] = cpf0 * mcol[j * 32];
        mcol[(K + j) * 32] = cpf0 * mcol[(K + j) * 32];
      }
      mcol[li * 32] = 1.0;
      mcol[(K + li) * 32] = 0.0;
      mcol[(2 * K) * 32] = b0;
      mcol[(RS + li) * 32] = 0.0;
      mcol[(RS + K + li) * 32] = 1.0;
      mcol[(RS + 2 * K) * 32] = b1;
      lu_solve_smem<KB>(g, W, xr, xt, okd);
    }
    iters = 1;
    conv = okd || !on;
    dy[0] = x2;
    dy[1] = x3;
    dy[2] = xr;
    dy[3] = xt;
    return;
  }

  // ---- implicit coupling: relaxed Richardson from v = b (ckm1d_def.py:303-404) ----
  const double bn = group_sum<KB>(fma(b0, b0, b1 * b1), g);
  const double rt = P.lin_rtol2 * bn;
  const double tol2 = rt > P.lin_atol2 ? rt : P.lin_atol2;
  double vr = b0, vt = b1;
  // Sweeps run in blocks of two with one warp vote per block.  The iterates
  // are advanced unconditionally and the answer is kept aside, so the
  // convergence tests (group norm, compare) of the block's two iterates are
  // off the dependency chain of the iteration (the norm of the first overlaps
  // the second sweep) and have no branch.  The count and the returned
  // iterate are those of the plain loop (test iterate it, then update, for
  // it = 0 .. lin_max_iter - 1): the first iterate whose residual norm is
  // below tol2, else the one after lin_max_iter updates.  A block may compute
  // one residual past the plain loop's exit; it changes no result.
  bool found = !on;
  double ans_r = vr, ans_t = vt;
  iters = 0;
  const bool full_groups = (g.K == KB);
  const int maxit = P.lin_max_iter;
  double r0, r1;
  if constexpr (REG) residual<KB>(g, Am, Bm, Cm, Dm, cpf0, b0, b1, vr, vt, r0, r1);
  else residual_smem<KB>(g, W, cpf0, b0, b1, vr, vt, r0, r1);
  for (int it = 0; it < maxit; it += 2) {
    if (__all_sync(FULL, found)) break;
    // iterate it: (vr, vt) with residual (r0, r1); iterate it + 1: (br, bt)
    const double br = fma(P.omega, r0, vr), bt = fma(P.omega, r1, vt);
    double q0, q1;
    if constexpr (REG) residual<KB>(g, Am, Bm, Cm, Dm, cpf0, b0, b1, br, bt, q0, q1);
    else residual_smem<KB>(g, W, cpf0, b0, b1, br, bt, q0, q1);
    const bool two = it + 1 < maxit;   // the plain loop also tests iterate it + 1
    const double wr = fma(P.omega, q0, br), wt = fma(P.omega, q1, bt);
    double s0, s1;
    if constexpr (REG) residual<KB>(g, Am, Bm, Cm, Dm, cpf0, b0, b1, wr, wt, s0, s1);
    else residual_smem<KB>(g, W, cpf0, b0, b1, wr, wt, s0, s1);
    const double rra = fma(r0, r0, r1 * r1), rrb = fma(q0, q0, q1 * q1);
    double rna, rnb;
    if (full_groups) {
      rna = group_sum_full<KB>(rra);
      rnb = group_sum_full<KB>(rrb);
    } else {
      rna = group_sum<KB>(rra, g);
      rnb = group_sum<KB>(rrb, g);
    }
    const bool hita = !found & (rna < tol2);
    iters = found ? iters : it + 1;
    ans_r = hita ? vr : ans_r;
    ans_t = hita ? vt : ans_t;
    found = found | hita;
    const bool hitb = two & !found & (rnb < tol2);
    iters = (found | !two) ? iters : it + 2;
    ans_r = hitb ? br : ans_r;
    ans_t = hitb ? bt : ans_t;
    found = found | hitb;
    // advance to iterate it + 2 (it + 1 when that was the last update)
    vr = two ? wr : br;
    vt = two ? wt : bt;
    r0 = s0;
    r1 = s1;
  }
  conv = found;
  if (found) {
    vr = ans_r;
    vt = ans_t;
  }
  if (!on) conv = true;
  dy[0] = x2;
  dy[1] = x3;
  dy[2] = vr;
  dy[3] = vt;
}

// Field forms with their own compiled right-hand side: two harmonics of a
// standing wave with the antinode (SW_A) or the node (SW_N) at x = 0, the
// forms of the benchmarked workloads; any other form uses the general one.
// P is uniform over a launch, so the branch never diverges.
template <int KB, int KC, int LIN>
__device__ __forceinline__ void rhs(const Geo& g, const Params& P, const WarpSmem& W, const MView& M,
                                    double sp0, double sp3, bool on, double t, const double y[4],
                                    double dy[4], bool& conv, int& iters) {
  if (P.nk == 2 && P.ac == 2)
    rhs_form<KB, KC, LIN, 2, 2>(g, P, W, M, sp0, sp3, on, t, y, dy, conv, iters);
  else if (P.nk == 2 && P.ac == 1)
    rhs_form<KB, KC, LIN, 2, 1>(g, P, W, M, sp0, sp3, on, t, y, dy, conv, iters);
  else
    rhs_form<KB, KC, LIN, 0, -1>(g, P, W, M, sp0, sp3, on, t, y, dy, conv, iters);
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

// State at Cash-Karp stage ST: y + h * sum_{m < ST} b[ST][m] k_m, the sum
// accumulated in increasing m (coefficients and loop fully compile-time).
template <int ST>
__device__ __forceinline__ void stage_state(const double* ks, double h, const double y[4], double ys[4]) {
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    double acc = kStageB[ST][0] * ks[c * 32];
#pragma unroll
    for (int m = 1; m < ST; ++m) acc = fma(kStageB[ST][m], ks[(m * 4 + c) * 32], acc);
    ys[c] = fma(h, acc, y[c]);
  }
}

// One adaptive Cash-Karp step for every active group of the warp
// (stepper.py:362-677).  Returns true (per lane) if a dense sample must be
// stored after this step; the caller writes it.
template <int KB, int KC, int LIN>
__device__ __forceinline__ bool step(const Geo& g, const Params& P, const WarpSmem& W, const MView& M,
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
  double* ks = W.ks + g.lane;   // ks[(st * 4 + c) * 32]
  int conv_fail_here = 0;

  // six Cash-Karp stages (stepper.py:379-480), one RHS call site
#pragma unroll 1
  for (int st = 0; st < 6; ++st) {
    double ys[4];
    switch (st) {
      case 0:
#pragma unroll
        for (int c = 0; c < 4; ++c) ys[c] = S.y[c];
        break;
      case 1: stage_state<1>(ks, h, S.y, ys); break;
      case 2: stage_state<2>(ks, h, S.y, ys); break;
      case 3: stage_state<3>(ks, h, S.y, ys); break;
      case 4: stage_state<4>(ks, h, S.y, ys); break;
      default: stage_state<5>(ks, h, S.y, ys); break;
    }
    const double ts = (st == 0) ? t : fma(kStageA[st], h, t);
    double kk[4];
    bool cv;
    int it;
    rhs<KB, KC, LIN>(g, P, W, M, S.sp0, S.sp3, on, ts, ys, kk, cv, it);
#pragma unroll
    for (int c = 0; c < 4; ++c) ks[(st * 4 + c) * 32] = kk[c];
    if (on) {
      S.lin_iters += it;
      if (cv) ++S.conv_ok;
      else {
        ++S.conv_fail;
        ++conv_fail_here;
      }
    }
  }

  // candidate (c2 = c5 = 0) and embedded error estimate (ce2 = 0)
  double yn[4];
  bool fin = true;
  double ratio_l = 1.0e30;
  bool ok_l = true;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const double k1 = ks[(0 * 4 + c) * 32], k3 = ks[(2 * 4 + c) * 32], k4 = ks[(3 * 4 + c) * 32],
                 k5 = ks[(4 * 4 + c) * 32], k6 = ks[(5 * 4 + c) * 32];
    const double acc = fma(C6, k6, fma(C4, k4, fma(C3, k3, C1 * k1)));
    yn[c] = fma(h, acc, S.y[c]);
    fin = fin && cbcm::isfinite_(yn[c]);
    const double es = fma(CE6, k6, fma(CE5, k5, fma(CE4, k4, fma(CE3, k3, CE1 * k1))));
    const double e = fabs(h * es) + 1.0e-18;
    const double ay = fabs(yn[c]), ao = fabs(S.y[c]);
    const double tl = P.rtol * (ay > ao ? ay : ao);
    const double tol = tl > P.atol ? tl : P.atol;
    const double r = tol / e;
    if (r < ratio_l) ratio_l = r;
    if (r < 1.0) ok_l = false;
  }
  const bool finite = group_all(fin, g);
  if (on) ++S.steps;

  const double g_new = group_event<KB>(yn, upv(W, g, 12), g, P.col);
  const bool crossing = (S.g_old * g_new < 0.0);
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
  }
  return store;
}

// After a dense store (if any): advance the schedule and test termination
// (stepper.py:651-662).
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
