// ckm1d_oracle.cpp -- CPU oracle for the CKM1D coupled-bubble integrator.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, serially and on the CPU, the
// algorithm of the reference's fused numba integrator
//   coupledbubble_control/backends/numba/rkck45_coupled_numba_stepper.py
//   coupledbubble_control/backends/numba/sysmtem_definitions/ckm1d_def.py
// It is used by tests/, by __graft_entry__.smoke() and by bench.py's CPU
// baseline leg as the checker.  The product (the CUDA library) never links or
// calls it.
//
// Parity contract with the CUDA kernels: every floating-point operation below
// is written in the same order, with the same explicit fma() calls, as the
// device code, and the elementary functions come from cbc_math.h.  Built with
// -ffp-contract=off (no implicit contraction) this makes the oracle and the
// GPU agree bit for bit.  Against the reference itself the oracle agrees to
// rounding level (the reference lets the compiler contract and uses libm);
// tests/golden holds vectors produced by running the reference numba kernel
// under numba's CUDA simulator.
//
// Deliberate differences from the reference (each one a defect fix):
//   * dense output: a stored slot is never overwritten by later steps
//     (reference store flag is never reset, stepper.py:71-112), and the sample
//     schedule continues across relaunches instead of forcing a sample at
//     every launch (stepper.py:196).  Optional "grid" mode clamps steps so
//     samples land exactly on t_begin + k (t_end - t_begin)/(NDO-1).
//     dense_mode 2 (oracle only, for pinning against the reference's own
//     dense output) replays the reference's behaviour, defect included.
//   * failure statuses that the reference defines but never sets
//     (stepper.py:27-33): -4 on a non-finite candidate state; -2 (or -3 when
//     the implicit coupling iteration failed in that step) when a step at the
//     minimum step size is rejected, where the reference would repeat the same
//     rejected step until its budget ran out; -1 when the step budget runs out.
//   * counters that the reference allocates but never fills
//     (models/model.py:212-216) are filled.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#include "../coupled-bubble-control_b200/csrc/cbc_math.h"

#include <atomic>
#include <thread>

extern "C" {

// Mirror of the solver/model specs (models/specs.py:6-72).
typedef struct cbo_spec {
  int32_t ns;         // number of systems
  int32_t ups;        // bubbles per system (K)
  int32_t tile;       // padded row width of the reference layout (>= ups)
  int32_t ndo;        // dense samples per system (0 = none)
  int32_t nk;         // harmonic components
  int32_t ac;         // 0 CONST, 1 SW_N, 2 SW_A
  int32_t dense_mode; // 0 reference schedule (fixed), 1 exact grid
  int32_t lin_max_iter;
  double atol, rtol, min_step, max_step;
  double lin_atol, lin_rtol, lin_relaxation;
  double etol;
  double col_threshold;  // collision threshold (0.1 in the numba kernel)
  int32_t lin_solver;    // 0 relaxed Richardson (the reference), 1 direct (Gauss-Jordan, partial pivoting)
  int32_t reserved;
} cbo_spec;

}  // extern "C"

namespace {

constexpr int KMAX = 64;
constexpr int NKMAX = 8;
constexpr double TWO_PI = 6.283185307179586;  // 2.0 * np.pi

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

struct Counters {
  int64_t steps = 0, rejected = 0, conv_ok = 0, conv_fail = 0, lin_iters = 0;
};

// One system, everything it needs, copied out of whatever layout the caller uses.
struct System {
  int K, NK, ac;
  double y[KMAX][4];  // R, X, U, V
  double up[KMAX][13];
  double c73[KMAX], c47[KMAX];
  double sp[5];
  double cp[4 * NKMAX];
  const double* M;  // M(c, j, i) = M[(c*K + j)*mstride_j ... ] via accessor
  // coupling matrices copied densely: Mc[c][j][i]
  std::vector<double> Mc;
  double m(int c, int j, int i) const { return Mc[((size_t)c * K + j) * K + i]; }
  // per-harmonic constants
  double wo[NKMAX], ph[NKMAX], lw[NKMAX], a[NKMAX], aw[NKMAX], awv[NKMAX], au[NKMAX];
};

void prepare(System& s) {
  // acoustic_field_1d (ckm1d_def.py:95-114): w0 = 2pi sp[1], l0 = 2pi sp[2], u0 = sp[4]
  const double w0 = TWO_PI * s.sp[1];
  const double l0 = TWO_PI * s.sp[2];
  const double u0 = s.sp[4];
  for (int k = 0; k < s.NK; ++k) {
    const double amps = s.cp[k], omega = s.cp[s.NK + k], phase = s.cp[2 * s.NK + k],
                 wave = s.cp[3 * s.NK + k];
    s.wo[k] = w0 * omega;
    s.ph[k] = phase;
    s.lw[k] = l0 * wave;
    s.a[k] = amps;
    s.aw[k] = amps * omega;
    s.awv[k] = amps * wave;
    s.au[k] = amps * u0;
  }
  for (int i = 0; i < s.K; ++i) {
    s.c73[i] = s.up[i][7] * (1.0 / 3.0);
    s.c47[i] = s.up[i][4] * s.up[i][7];
  }
}

struct Spec {
  double atol, rtol, min_step, max_step, lin_atol2, lin_rtol2, omega, etol, col;
  int lin_max_iter, ndo, dense_mode, lin_solver;
};

// Direct solve of the implicit coupling system (lin_solver = 1), the same
// operations as the device code (csrc/ckm1d_core.cuh, lu_solve_reg /
// lu_solve_smem).  Unknowns x = (vr_0..vr_{K-1}, vt_0..vt_{K-1}); a holds N =
// 2K rows of N + 1 entries (the right side last).  Gauss-Jordan elimination
// with partial pivoting: for column c the pivot is the not-yet-pivot row with
// the largest key (|a[r][c]| at 2^-13 relative resolution, NaN below every
// number, ties to the smaller row), rp = 1 / pivot, the pivot row's entries k > c are read before the column's
// updates, and every row r gets l = (r == p) ? 0 : a[r][c] * rp and
// a[r][k] = fma(-l, pivot_row[k], a[r][k]) for k = c+1..N.  Then
// x_c = a[p_c][N] * rp_c.  Returns false if a pivot is zero or not finite.
bool lu_solve(int K, std::vector<double>& a, double* x) {
  const int N = 2 * K, RS = N + 1;
  // pivot key: the high 32 bits of |a| with the low 7 bits replaced by
  // 127 - row (magnitude at 2^-13 relative resolution, ties to the smaller
  // row), NaN lowest (csrc/ckm1d_core.cuh, piv_key32)
  auto key = [](double v, int r) {
    uint64_t b;
    memcpy(&b, &v, sizeof b);
    b &= 0x7FFFFFFFFFFFFFFFull;
    uint32_t hi = (uint32_t)(b >> 32);
    if (b > 0x7FF0000000000000ull) hi = 0u;
    return (hi & ~127u) | (uint32_t)(127 - r);
  };
  bool pivoted[2 * KMAX] = {};
  int perm[2 * KMAX];
  double rps[2 * KMAX];
  double pk[2 * KMAX + 1];
  bool ok = true;
  for (int c = 0; c < N; ++c) {
    int p = -1;
    for (int r = 0; r < N; ++r) {
      if (pivoted[r]) continue;
      if (p < 0 || key(a[(size_t)r * RS + c], r) > key(a[(size_t)p * RS + c], p)) p = r;
    }
    const double piv = a[(size_t)p * RS + c];
    ok = ok && (piv != 0.0) && cbcm::isfinite_(piv);
    const double rp = 1.0 / piv;
    pivoted[p] = true;
    perm[c] = p;
    rps[c] = rp;
    for (int k = c + 1; k <= N; ++k) pk[k] = a[(size_t)p * RS + k];
    for (int r = 0; r < N; ++r) {
      const double l = (r == p) ? 0.0 : a[(size_t)r * RS + c] * rp;
      for (int k = c + 1; k <= N; ++k) a[(size_t)r * RS + k] = fma(-l, pk[k], a[(size_t)r * RS + k]);
    }
  }
  for (int c = 0; c < N; ++c) x[c] = a[(size_t)perm[c] * RS + N] * rps[c];
  return ok;
}

// Pairwise-tree sum over the next power of two (zero padded):
// ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + ...).
double tree_sum(const double* a, int K) {
  int P = 1;
  while (P < K) P <<= 1;
  double buf[2 * KMAX];
  for (int i = 0; i < P; ++i) buf[i] = i < K ? a[i] : 0.0;
  for (int w = 1; w < P; w <<= 1)
    for (int i = 0; i < P; i += 2 * w) buf[i] = buf[i] + buf[i + w];
  return buf[0];
}

// Pairwise tree without padding: at width w, a[i] += a[i + w] for every i a
// multiple of 2w with i + w < n, so a lone last element is carried up unchanged:
// ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + a6).  0.0 for n = 0.
double tree_sum_open(double* a, int n) {
  if (n <= 0) return 0.0;
  for (int w = 1; w < n; w <<= 1)
    for (int i = 0; i + w < n; i += 2 * w) a[i] = a[i] + a[i + w];
  return a[0];
}

// ode_fun + explicit_coupling + implicit_coupling for the whole system
// (ckm1d_def.py:408-497, :164-248, :250-300, :303-404).
void rhs(const System& s, const Spec& sp, double t, const double (*y)[4], double (*dy)[4],
         Counters& cnt) {
  const int K = s.K;
  // time harmonics (system-uniform part of acoustic_field_1d)
  double st[NKMAX], ct[NKMAX];
  for (int k = 0; k < s.NK; ++k) cbcm::sincos(cbcm::fma_(s.wo[k], t, s.ph[k]), &st[k], &ct[k]);

  double cpf0[KMAX], cpf1[KMAX], cpf2[KMAX], cpf3[KMAX];
  double h0[KMAX], h1[KMAX], h2[KMAX], h3[KMAX], h4[KMAX], h5[KMAX], h6[KMAX];
  double b0[KMAX], b1[KMAX];
  for (int i = 0; i < K; ++i) {
    const double x0 = y[i][0], x1 = y[i][1], x2 = y[i][2], x3 = y[i][3];
    const double* up = s.up[i];
    const double rx0 = 1.0 / x0;
    const double p = cbcm::pow_pos(rx0, s.sp[0]);
    double pa = 0.0, pt = 0.0, px = 0.0, ux = 0.0;
    for (int k = 0; k < s.NK; ++k) {
      if (s.ac == 0) {  // CONST
        pa = fma(s.a[k], st[k], pa);
        pt = fma(s.aw[k], ct[k], pt);
      } else {
        double sx, cx;
        cbcm::sincos(fma(s.lw[k], x1, s.ph[k]), &sx, &cx);
        if (s.ac == 1) {  // SW_N
          pa = fma(s.a[k] * sx, st[k], pa);
          pt = fma(s.aw[k] * sx, ct[k], pt);
          px = fma(s.awv[k] * cx, st[k], px);
          ux = fma(s.au[k] * cx, ct[k], ux);
        } else {  // SW_A
          pa = fma(s.a[k] * cx, st[k], pa);
          pt = fma(s.aw[k] * cx, ct[k], pt);
          px = fma(-(s.awv[k] * sx), st[k], px);
          ux = fma(-(s.au[k] * sx), ct[k], ux);
        }
      }
    }
    // Keller--Miksis numerator / denominator (ckm1d_def.py:429-438)
    const double q = fma(up[7], x2, 1.0);
    double N = fma(up[1], x2, up[0]) * p;
    N = fma(-up[2], q, N);
    N = fma(-up[3], rx0, N);
    N = fma(-(up[4] * x2), rx0, N);
    const double w = fma(-s.c73[i], x2, 1.0);
    N = fma((-1.5 * w) * x2, x2, N);
    N = fma(-(q * up[5]), pa, N);
    N = fma(-(up[6] * pt), x0, N);
    N = fma(up[8] * x3, x3, N);
    const double D = fma(-(up[7] * x0), x2, x0) + s.c47[i];
    const double rD = 1.0 / D;
    const double x02 = x0 * x0;
    const double x03 = x02 * x0;
    // primary Bjerknes and drag forces (ckm1d_def.py:441-447)
    const double Fb1 = -(up[10] * x03) * px;
    const double Fd = -(up[11] * x0) * fma(x3, s.sp[3], -ux);
    const double rx03 = (rx0 * rx0) * rx0;
    dy[i][0] = x2;
    dy[i][1] = x3;
    b0[i] = N * rD;
    b1[i] = fma((3.0 * (Fb1 + Fd)) * up[9], rx03, -(((3.0 * x2) * rx0) * x3));
    // coupling factors and terms (ckm1d_def.py:449-468)
    cpf0[i] = rD;
    cpf1[i] = x3 * rD;
    cpf2[i] = x2 * rx0;
    cpf3[i] = rx0 * rx0;
    h0[i] = x0 * (x2 * x2);
    h1[i] = x02 * x2;
    h2[i] = h1[i] * x3;
    h3[i] = x03 * x3;
    h4[i] = h3[i] * x3;
    h5[i] = x02;
    h6[i] = x03;
  }

  // explicit coupling (ckm1d_def.py:164-246) and the matrix of the implicit
  // system (mat_vec_product, ckm1d_def.py:250-299).  Canonical order: bubble i
  // sums over its partners j = (i + d) mod K, d = 1 .. K-1.
  static thread_local std::vector<double> Am, Bm, Cm, Dm;
  Am.resize((size_t)K * K);
  Bm.resize((size_t)K * K);
  Cm.resize((size_t)K * K);
  Dm.resize((size_t)K * K);
  for (int i = 0; i < K; ++i) {
    const double xi = y[i][1];
    double g0 = 0.0, g1 = 0.0, tn = 0.0, tg2 = 0.0, tg3 = 0.0;
    for (int d = 1; d < K; ++d) {
      const int j = (i + d) % K;
      const double delta = xi - y[j][1];
      const double sg = (double)((delta > 0.0) - (delta < 0.0));
      const double ad = fabs(delta);
      const double rd = 1.0 / (ad > 1e-30 ? ad : 1e-30);
      const double rd2 = rd * rd;
      const double srd2 = rd2 * sg;
      const double rd3 = rd2 * rd;
      const double m0 = s.m(0, j, i), m1 = s.m(1, j, i), m2 = s.m(2, j, i);
      double t0 = fma(2.5 * srd2, h2[j], rd3 * h4[j]);
      t0 = fma(2.0 * rd, h0[j], t0);
      g0 = fma(-m0, t0, g0);
      const double t1 = fma(srd2, h1[j], rd3 * h3[j]);
      g1 = fma(-0.5 * m0, t1, g1);
      const double t2 = fma(2.0 * srd2, h0[j], (5.0 * rd3) * h2[j]);
      tn = fma(m1, t2, tn);
      tg2 = fma(m1, t1, tg2);
      tg3 = fma(m2, t1, tg3);
      Am[(size_t)i * K + j] = (m0 * rd) * h5[j];
      Bm[(size_t)i * K + j] = ((0.5 * m0) * srd2) * h6[j];
      Cm[(size_t)i * K + j] = -((m1 * srd2) * h5[j]);
      Dm[(size_t)i * K + j] = -((m1 * rd3) * h6[j]);
    }
    b0[i] = fma(g0, cpf0[i], fma(g1, cpf1[i], b0[i]));
    b1[i] = b1[i] + fma(tg2, cpf2[i], fma(tg3, cpf3[i], tn));
  }

  if (sp.lin_solver == 1) {
    // direct solve: rows R_i (x_i + cpf0_i sum_j (A_ij vr_j + B_ij vt_j) = b0_i)
    // and T_i (x_{K+i} + sum_j (C_ij vr_j + D_ij vt_j) = b1_i)
    const int N = 2 * K, RS = N + 1;
    static thread_local std::vector<double> a;
    a.assign((size_t)N * RS, 0.0);
    for (int i = 0; i < K; ++i) {
      double* rR = &a[(size_t)i * RS];
      double* rT = &a[(size_t)(K + i) * RS];
      for (int j = 0; j < K; ++j) {
        if (j == i) {
          rR[j] = 1.0;
          rR[K + j] = 0.0;
          rT[j] = 0.0;
          rT[K + j] = 1.0;
        } else {
          rR[j] = cpf0[i] * Am[(size_t)i * K + j];
          rR[K + j] = cpf0[i] * Bm[(size_t)i * K + j];
          rT[j] = Cm[(size_t)i * K + j];
          rT[K + j] = Dm[(size_t)i * K + j];
        }
      }
      rR[N] = b0[i];
      rT[N] = b1[i];
    }
    double x[2 * KMAX];
    const bool ok = lu_solve(K, a, x);
    cnt.lin_iters += 1;
    if (ok) cnt.conv_ok += 1; else cnt.conv_fail += 1;
    for (int i = 0; i < K; ++i) {
      dy[i][2] = x[i];
      dy[i][3] = x[K + i];
    }
    return;
  }

  // implicit coupling: relaxed Richardson from v = b (ckm1d_def.py:303-404);
  // norms are pairwise-tree sums over the bubbles
  double acc[KMAX];
  for (int i = 0; i < K; ++i) acc[i] = fma(b0[i], b0[i], b1[i] * b1[i]);
  const double bn = tree_sum(acc, K);
  const double rt = sp.lin_rtol2 * bn;
  const double tol2 = rt > sp.lin_atol2 ? rt : sp.lin_atol2;
  double vr[KMAX], vt[KMAX], r0[KMAX], r1[KMAX];
  for (int i = 0; i < K; ++i) {
    vr[i] = b0[i];
    vt[i] = b1[i];
  }
  bool conv = false;
  for (int it = 0; it < sp.lin_max_iter; ++it) {
    for (int i = 0; i < K; ++i) {
      // partner distance d = 1..K-1 (j = (i + d) mod K) accumulates into
      // chain (d - 1) mod 4, increasing d within a chain; the chains are
      // combined by the open pairwise tree: the device kernel's order
      double cr[4] = {0.0, 0.0, 0.0, 0.0}, ct[4] = {0.0, 0.0, 0.0, 0.0};
      for (int d = 1; d < K; ++d) {
        const int j = (i + d) % K;
        const int c = (d - 1) & 3;
        cr[c] = fma(Am[(size_t)i * K + j], vr[j], fma(Bm[(size_t)i * K + j], vt[j], cr[c]));
        ct[c] = fma(Cm[(size_t)i * K + j], vr[j], fma(Dm[(size_t)i * K + j], vt[j], ct[c]));
      }
      const int nc = K - 1 < 4 ? K - 1 : 4;
      const double ar = tree_sum_open(cr, nc);
      const double at = tree_sum_open(ct, nc);
      const double ax0 = fma(ar, cpf0[i], vr[i]);
      const double ax1 = at + vt[i];
      r0[i] = b0[i] - ax0;
      r1[i] = b1[i] - ax1;
    }
    for (int i = 0; i < K; ++i) acc[i] = fma(r0[i], r0[i], r1[i] * r1[i]);
    const double rn = tree_sum(acc, K);
    cnt.lin_iters += 1;
    if (rn < tol2) {
      conv = true;
      break;
    }
    for (int i = 0; i < K; ++i) {
      vr[i] = fma(sp.omega, r0[i], vr[i]);
      vt[i] = fma(sp.omega, r1[i], vt[i]);
    }
  }
  if (conv) cnt.conv_ok += 1; else cnt.conv_fail += 1;
  for (int i = 0; i < K; ++i) {
    dy[i][2] = vr[i];
    dy[i][3] = vt[i];
  }
}

// event_fun (ckm1d_def.py:499-556): smallest gap between neighbours in the chain.
double event_g(const System& s, const Spec& sp, const double (*y)[4]) {
  double g = 1e30;
  for (int i = 0; i + 1 < s.K; ++i) {
    const double ri = y[i][0] * s.up[i][12];
    const double rj = y[i + 1][0] * s.up[i + 1][12];
    const double gap = fabs(y[i][1] - y[i + 1][1]) - (ri + rj) * sp.col;
    if (gap < g) g = gap;
  }
  return g;
}

struct Dense {
  int ndo = 0;
  int idx = 0;
  double t_begin = 0.0, t_end = 0.0, dt = 0.0;
  double next = 0.0;
  // store(slot, t, y) supplied by the layout front end
};

double grid_time(const Dense& d, int k) {
  if (k >= d.ndo - 1 && d.ndo > 1) return d.t_end;
  return fma((double)k, d.dt, d.t_begin);
}

enum : int {
  ACTIVE = 0, SUCCESS = 1, EVENT_TERMINAL = 2,
  MAX_STEPS = -1, STEP_LIMIT = -2, CONV_FAIL = -3, NONFINITE = -4
};

// Integrates one system for at most `budget` steps.  Mirrors the per-system
// control flow of the numba kernel (stepper.py:139-706) with launch
// boundaries made transparent.
template <class StoreFn>
void integrate(System& s, const Spec& sp, double& t, double t_end, double t_begin, double& h,
               double& g_store, int& status, int& dense_idx, const double* dense_time_prev,
               int64_t budget, Counters& cnt, StoreFn store) {
  // prologue (stepper.py:179-214); a stored failure status (-2, -3, -4) keeps
  // the system stopped, -1 (budget spent) resumes
  const int status_in = status;
  status = (t >= t_end) ? SUCCESS : ACTIVE;
  if (fabs(g_store) < sp.etol) status = EVENT_TERMINAL;
  if (status_in <= STEP_LIMIT) status = status_in;
  if (status != ACTIVE) return;

  const int K = s.K;
  double(*y)[4] = s.y;
  Dense d;
  d.ndo = sp.ndo;
  d.idx = dense_idx;
  d.t_begin = t_begin;
  d.t_end = t_end;
  d.dt = (sp.ndo == 1) ? (t_end - t_begin) : (sp.ndo > 1 ? (t_end - t_begin) / (double)(sp.ndo - 1) : 0.0);
  // slot the reference keeps overwriting (dense_mode 2 only; -1 = none)
  int defect_slot = -1;
  if (sp.dense_mode == 0 || sp.dense_mode == 2) {
    // reference schedule: next sample = previous stored time + dt, clipped to t_end;
    // the very first sample is taken at once.  The emulation of the reference
    // (mode 2) forces a sample at every launch, as its prologue does
    // (stepper.py:197-200: next sample time = actual time).
    if (d.idx == 0 || dense_time_prev == nullptr || sp.dense_mode == 2) d.next = t;
    else {
      const double nx = *dense_time_prev + d.dt;
      d.next = nx < t_end ? nx : t_end;
    }
    if (d.idx < d.ndo && d.next <= t) {
      store(d.idx, t, y, true);
      defect_slot = d.idx;
      d.idx += 1;
      const double nx = t + d.dt;
      d.next = nx < t_end ? nx : t_end;
    }
  } else if (d.ndo > 0) {
    if (d.idx < d.ndo && t >= grid_time(d, d.idx)) {
      store(d.idx, t, y, true);
      d.idx += 1;
    }
  }

  double g_old = event_g(s, sp, y);
  double k1[KMAX][4], k2[KMAX][4], k3[KMAX][4], k4[KMAX][4], k5[KMAX][4], k6[KMAX][4];
  double ys[KMAX][4], yn[KMAX][4];

  for (int64_t step = 0; step < budget; ++step) {
    // step-size clamps (stepper.py:366-373)
    if (h < sp.min_step) h = sp.min_step;
    if (h > sp.max_step) h = sp.max_step;
    const double rem = t_end - t;
    if (h > rem) h = rem;
    bool landing = false;
    double t_land = 0.0;
    if (sp.dense_mode == 1 && d.idx < d.ndo) {
      t_land = grid_time(d, d.idx);
      const double remk = t_land - t;
      if (h >= remk) {
        h = remk;
        landing = true;
      }
    }

    // six Cash-Karp stages (stepper.py:379-480)
    const int64_t conv_fail_before = cnt.conv_fail;
    rhs(s, sp, t, y, k1, cnt);
    for (int i = 0; i < K; ++i)
      for (int c = 0; c < 4; ++c) ys[i][c] = fma(h, B21 * k1[i][c], y[i][c]);
    rhs(s, sp, fma(A2, h, t), ys, k2, cnt);
    for (int i = 0; i < K; ++i)
      for (int c = 0; c < 4; ++c) ys[i][c] = fma(h, fma(B32, k2[i][c], B31 * k1[i][c]), y[i][c]);
    rhs(s, sp, fma(A3, h, t), ys, k3, cnt);
    for (int i = 0; i < K; ++i)
      for (int c = 0; c < 4; ++c)
        ys[i][c] = fma(h, fma(B43, k3[i][c], fma(B42, k2[i][c], B41 * k1[i][c])), y[i][c]);
    rhs(s, sp, fma(A4, h, t), ys, k4, cnt);
    for (int i = 0; i < K; ++i)
      for (int c = 0; c < 4; ++c)
        ys[i][c] = fma(h, fma(B54, k4[i][c], fma(B53, k3[i][c], fma(B52, k2[i][c], B51 * k1[i][c]))),
                       y[i][c]);
    rhs(s, sp, fma(A5, h, t), ys, k5, cnt);
    for (int i = 0; i < K; ++i)
      for (int c = 0; c < 4; ++c)
        ys[i][c] = fma(h,
                       fma(B65, k5[i][c],
                           fma(B64, k4[i][c], fma(B63, k3[i][c], fma(B62, k2[i][c], B61 * k1[i][c])))),
                       y[i][c]);
    rhs(s, sp, fma(A6, h, t), ys, k6, cnt);

    // candidate (stepper.py:483-484); c2 = c5 = 0
    bool finite = true;
    for (int i = 0; i < K; ++i)
      for (int c = 0; c < 4; ++c) {
        const double acc = fma(C6, k6[i][c], fma(C4, k4[i][c], fma(C3, k3[i][c], C1 * k1[i][c])));
        yn[i][c] = fma(h, acc, y[i][c]);
        if (!cbcm::isfinite_(yn[i][c])) finite = false;
      }

    cnt.steps += 1;
    const double g_new = event_g(s, sp, yn);
    bool ok;
    double h_next;
    const bool crossing = (g_old * g_new < 0.0);
    if (crossing) {
      // event bracketing (stepper.py:500-515, 575-581)
      const double abs_old = fabs(g_old);
      const double denom = abs_old + fabs(g_new);
      const double ratio = (abs_old / (denom + 1e-15)) * 0.99;
      h_next = h * ratio;
      ok = false;
    } else {
      if (!finite) {
        status = NONFINITE;
        cnt.rejected += 1;
        break;
      }
      // embedded error, max-norm of tol/err (stepper.py:521-536); ce2 = 0
      double ratio = 1.0e30;
      ok = true;
      for (int i = 0; i < K; ++i)
        for (int c = 0; c < 4; ++c) {
          const double es =
              fma(CE6, k6[i][c], fma(CE5, k5[i][c], fma(CE4, k4[i][c], fma(CE3, k3[i][c], CE1 * k1[i][c]))));
          const double e = fabs(h * es) + 1.0e-18;
          const double ay = fabs(yn[i][c]), ao = fabs(y[i][c]);
          const double tl = sp.rtol * (ay > ao ? ay : ao);
          const double tol = tl > sp.atol ? tl : sp.atol;
          const double r = tol / e;
          if (r < ratio) ratio = r;
          if (r < 1.0) ok = false;
        }
      // controller (stepper.py:610-614)
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
      t = landing ? t_land : t + h;
      for (int i = 0; i < K; ++i)
        for (int c = 0; c < 4; ++c) y[i][c] = yn[i][c];
      g_old = g_new;
    } else {
      cnt.rejected += 1;
      // a rejected step that cannot shrink any further: the reference loops here
      // until its step budget runs out; report it instead
      if (h <= sp.min_step) {
        status = (cnt.conv_fail > conv_fail_before) ? CONV_FAIL : STEP_LIMIT;
        h = h_next;
        break;
      }
    }
    h = h_next;

    // dense output (stepper.py:634-645, with the slot defect fixed)
    if (sp.dense_mode == 0) {
      if (d.idx < d.ndo && d.next <= t) {
        store(d.idx, t, y, true);
        d.idx += 1;
        const double nx = t + d.dt;
        d.next = nx < t_end ? nx : t_end;
      }
    } else if (sp.dense_mode == 2) {
      // the reference as it is (stepper.py:71-112): a new slot takes the time
      // and the state, and every later step rewrites the state of the last
      // slot taken, because its store flag is never reset
      if (d.idx < d.ndo && d.next <= t) {
        store(d.idx, t, y, true);
        defect_slot = d.idx;
        d.idx += 1;
        const double nx = t + d.dt;
        d.next = nx < t_end ? nx : t_end;
      } else if (defect_slot >= 0) {
        store(defect_slot, t, y, false);
      }
    } else if (ok && landing) {
      store(d.idx, t, y, true);
      d.idx += 1;
    }

    // termination (stepper.py:651-662)
    if (t >= t_end) {
      status = SUCCESS;
      break;
    }
    if (fabs(g_old) < sp.etol) {
      status = EVENT_TERMINAL;
      break;
    }
  }
  if (status == ACTIVE) status = MAX_STEPS;
  g_store = g_old;
  dense_idx = d.idx;
}

template <class F>
void run_parallel(F& worker, int nthreads) {
  int n = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
  if (n < 1) n = 1;
  if (n == 1) {
    worker();
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(n);
  for (int i = 0; i < n; ++i) pool.emplace_back([&worker]() { worker(); });
  for (auto& th : pool) th.join();
}

Spec make_spec(const cbo_spec* c) {
  Spec s;
  s.atol = c->atol;
  s.rtol = c->rtol;
  s.min_step = c->min_step;
  s.max_step = c->max_step;
  s.lin_atol2 = c->lin_atol * c->lin_atol;
  s.lin_rtol2 = c->lin_rtol * c->lin_rtol;
  s.omega = c->lin_relaxation;
  s.etol = c->etol;
  s.col = 1.0 + c->col_threshold;
  s.lin_max_iter = c->lin_max_iter;
  s.ndo = c->ndo;
  s.dense_mode = c->dense_mode;
  s.lin_solver = c->lin_solver;
  return s;
}

}  // namespace

extern "C" {

// Reference-layout front end: the same buffers, shapes and in-place update
// as the reference's solver (models/model.py:56-106, buffers.py:29-71):
//   actual_state (4, NS, TILE), unit_params (13, NS, TILE), system_params
//   (5, NS), control_params (4 NK, NS), coupling_matrices (3, UPS, NS, TILE),
//   dense_time (NDO, NS), dense_state (NDO, 4, NS, TILE), per-system vectors.
// Counter pointers may be NULL.  `budget` = maximum steps per system.
// Returns 0, or a negative value on bad arguments.
int cbo_solve_ref_layout(const cbo_spec* spec, double* actual_time, const double* time_end,
                         const double* time_begin, double* time_step, double* actual_state,
                         const double* unit_params, const double* system_params,
                         const double* control_params, const double* coupling_matrices,
                         int32_t* dense_index, double* dense_time, double* dense_state,
                         double* actual_event, int32_t* status_flags, int32_t* total_steps,
                         int32_t* rejected_steps, int32_t* conv_success, int32_t* conv_failures,
                         int64_t* lin_iters, int64_t budget, int32_t nthreads) {
  if (!spec || spec->ups < 1 || spec->ups > KMAX || spec->nk < 1 || spec->nk > NKMAX || spec->ns < 1 ||
      spec->tile < spec->ups || spec->lin_solver < 0 || spec->lin_solver > 1)
    return -1;
  const Spec sp = make_spec(spec);
  const int NS = spec->ns, K = spec->ups, T = spec->tile, NK = spec->nk, NDO = spec->ndo;
  const size_t NST = (size_t)NS * T;
  // dynamic schedule over systems on `nthreads` host threads (<= 0: all cores)
  std::atomic<int> next_sys(0);
  auto worker = [&]() {
  for (int g = next_sys.fetch_add(1); g < NS; g = next_sys.fetch_add(1)) {
    System s;
    s.K = K;
    s.NK = NK;
    s.ac = spec->ac;
    for (int i = 0; i < K; ++i) {
      for (int c = 0; c < 4; ++c) s.y[i][c] = actual_state[c * NST + (size_t)g * T + i];
      for (int p = 0; p < 13; ++p) s.up[i][p] = unit_params[p * NST + (size_t)g * T + i];
    }
    for (int p = 0; p < 5; ++p) s.sp[p] = system_params[(size_t)p * NS + g];
    for (int p = 0; p < 4 * NK; ++p) s.cp[p] = control_params[(size_t)p * NS + g];
    s.Mc.resize((size_t)3 * K * K);
    for (int c = 0; c < 3; ++c)
      for (int j = 0; j < K; ++j)
        for (int i = 0; i < K; ++i)
          s.Mc[((size_t)c * K + j) * K + i] = coupling_matrices[((size_t)c * K + j) * NST + (size_t)g * T + i];
    prepare(s);
    double t = actual_time[g], h = time_step[g], ge = actual_event[g];
    int status = status_flags[g];
    int didx = dense_index ? dense_index[g] : 0;
    const double* prev = (dense_time && didx > 0) ? &dense_time[(size_t)(didx - 1) * NS + g] : nullptr;
    Counters cnt;
    auto store = [&](int slot, double ts, const double (*yy)[4], bool write_time) {
      if (!dense_time || !dense_state) return;
      if (write_time) dense_time[(size_t)slot * NS + g] = ts;
      for (int c = 0; c < 4; ++c)
        for (int i = 0; i < K; ++i) dense_state[((size_t)slot * 4 + c) * NST + (size_t)g * T + i] = yy[i][c];
    };
    Spec spl = sp;
    if (!dense_time || !dense_state || !dense_index) spl.ndo = 0;
    integrate(s, spl, t, time_end[g], time_begin[g], h, ge, status, didx, prev, budget, cnt, store);
    for (int i = 0; i < K; ++i)
      for (int c = 0; c < 4; ++c) actual_state[c * NST + (size_t)g * T + i] = s.y[i][c];
    actual_time[g] = t;
    time_step[g] = h;
    actual_event[g] = ge;
    status_flags[g] = status;
    if (dense_index) dense_index[g] = didx;
    if (total_steps) total_steps[g] += (int32_t)cnt.steps;
    if (rejected_steps) rejected_steps[g] += (int32_t)cnt.rejected;
    if (conv_success) conv_success[g] += (int32_t)cnt.conv_ok;
    if (conv_failures) conv_failures[g] += (int32_t)cnt.conv_fail;
    if (lin_iters) lin_iters[g] += cnt.lin_iters;
  }
  };
  run_parallel(worker, nthreads);
  return 0;
}

// The direct solver alone, for its unit tests: a holds the 2K x (2K + 1)
// augmented matrix row-major (overwritten), x receives the 2K unknowns.
// Returns 1 if every pivot was nonzero and finite, 0 if not, -1 on bad K.
int cbo_lu_solve(int32_t K, double* a, double* x) {
  if (K < 1 || K > KMAX) return -1;
  std::vector<double> v(a, a + (size_t)2 * K * (2 * K + 1));
  const bool ok = lu_solve(K, v, x);
  std::copy(v.begin(), v.end(), a);
  return ok ? 1 : 0;
}

// Elementary-function evaluator used by the unit tests of cbc_math.h.
// kind: 0 sin, 1 cos, 2 exp, 3 log, 4 pow(x, y[i])
void cbo_math_eval(int kind, int64_t n, const double* x, const double* y, double* out) {
  for (int64_t i = 0; i < n; ++i) {
    double s, c;
    switch (kind) {
      case 0: cbcm::sincos(x[i], &s, &c); out[i] = s; break;
      case 1: cbcm::sincos(x[i], &s, &c); out[i] = c; break;
      case 2: out[i] = cbcm::exp(x[i]); break;
      case 3: out[i] = cbcm::log(x[i]); break;
      default: out[i] = cbcm::pow_pos(x[i], y[i]); break;
    }
  }
}

}  // extern "C"
