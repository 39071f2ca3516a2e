"""An independent check of the tight-tolerance reference used for the
accuracy statements: the oracle's Cash-Karp integrator at rtol = atol =
1e-12 with the direct coupling solve, against scipy's DOP853 (a different
Runge-Kutta pair and step controller) at rtol = 1e-12 over a numpy
restatement of the right-hand side with an exact dense solve of the implicit
coupling system.  Both start from the model's own host buffers (the
precomputed bubble, system, control and coupling constants), so they agree
only if the integrations do.

The right-hand side follows the kernels' formulas (radial Keller-Miksis with
the translational forces, the pair terms over the partners and the 2K x 2K
implicit system for the accelerations; acoustic_field_1d, ode_fun,
explicit_coupling and implicit_coupling of
backends/numba/sysmtem_definitions/ckm1d_def.py), written as plain numpy
expressions in natural order: it shares no code and no operation order with
the kernels or the oracle.

Observed (3 systems each: plain study K = 2 and mixed-K K = 4 over half a
period, SW_A; K = 8 SW_N over 0.3 period; K = 3 CONST over half a period;
3,000-13,200 oracle steps, dR/dt changing by up to 41 on the way): R within
2.3e-12, x within 1.7e-14, dR/dt within 9.3e-10, dx/dt within 5.4e-13
(relative, with the floors below).  The bound asserted is 1e-8.
"""
import copy

import numpy as np
import pytest

from cbc_b200 import scenes
from cbc_b200.models import SolverSpec
from oracle import oracle

scipy_integrate = pytest.importorskip("scipy.integrate")

FLOOR = np.array([1.0, 1e-3, 1e-2, 1e-3])     # R, x, dR/dt, dx/dt


def _rhs_factory(buf, s, K, nk, ac):
    """dy/dt of system s (state ordered R[K], X[K], U[K], V[K])."""
    up = buf["unit_params"][:, s, :K]                       # (13, K)
    sp = buf["system_params"][:, s]
    cp = buf["control_params"][:, s]
    M = buf["coupling_matrices"][:, :K, s, :K]              # M[c, j, i]
    gamma3, w0, l0, c_, u0 = sp[0], 2 * np.pi * sp[1], 2 * np.pi * sp[2], sp[3], sp[4]
    PA, om, ph, wv = cp[:nk], cp[nk:2 * nk], cp[2 * nk:3 * nk], cp[3 * nk:4 * nk]
    eye = np.eye(K, dtype=bool)

    def f(t, y):
        R, X, U, V = y[:K], y[K:2 * K], y[2 * K:3 * K], y[3 * K:]
        st = np.sin(w0 * om * t + ph)[:, None]              # (nk, 1)
        ct = np.cos(w0 * om * t + ph)[:, None]
        arg = l0 * wv[:, None] * X[None, :] + ph[:, None]   # (nk, K)
        sx, cx = np.sin(arg), np.cos(arg)
        A_ = PA[:, None]
        if ac == "SW_A":
            pa = np.sum(A_ * cx * st, 0)
            pt = np.sum(A_ * om[:, None] * cx * ct, 0)
            px = np.sum(-A_ * wv[:, None] * sx * st, 0)
            ux = np.sum(-A_ * u0 * sx * ct, 0)
        elif ac == "SW_N":
            pa = np.sum(A_ * sx * st, 0)
            pt = np.sum(A_ * om[:, None] * sx * ct, 0)
            px = np.sum(A_ * wv[:, None] * cx * st, 0)
            ux = np.sum(A_ * u0 * cx * ct, 0)
        else:
            pa = np.sum(A_ * st, 0) * np.ones(K)
            pt = np.sum(A_ * om[:, None] * ct, 0) * np.ones(K)
            px = np.zeros(K)
            ux = np.zeros(K)
        # pair terms: receiving bubble i (rows), partner j (columns)
        Rj, Uj, Vj = R[None, :], U[None, :], V[None, :]
        delta = X[:, None] - X[None, :]
        sg = np.sign(delta)
        rd = 1.0 / np.maximum(np.abs(delta), 1e-30)
        rd2, rd3 = rd * rd, rd * rd * rd
        m0, m1, m2 = M[0].T, M[1].T, M[2].T                 # [i, j]
        h0, h1 = Rj * Uj ** 2, Rj ** 2 * Uj
        h2, h3 = h1 * Vj, Rj ** 3 * Vj
        h4 = h3 * Vj
        t0 = 2.5 * sg * rd2 * h2 + rd3 * h4 + 2.0 * rd * h0
        t1 = sg * rd2 * h1 + rd3 * h3
        t2 = 2.0 * sg * rd2 * h0 + 5.0 * rd3 * h2
        off = ~eye
        g0 = -np.sum(np.where(off, m0 * t0, 0.0), 1)
        g1 = -0.5 * np.sum(np.where(off, m0 * t1, 0.0), 1)
        tn = np.sum(np.where(off, m1 * t2, 0.0), 1)
        tg2 = np.sum(np.where(off, m1 * t1, 0.0), 1)
        tg3 = np.sum(np.where(off, m2 * t1, 0.0), 1)
        Am = np.where(off, m0 * rd * Rj ** 2, 0.0)
        Bm = np.where(off, 0.5 * m0 * sg * rd2 * Rj ** 3, 0.0)
        Cm = np.where(off, -m1 * sg * rd2 * Rj ** 2, 0.0)
        Dm = np.where(off, -m1 * rd3 * Rj ** 3, 0.0)
        # uncoupled Keller-Miksis and translation
        p = (1.0 / R) ** gamma3
        q = 1.0 + up[7] * U
        N = ((up[0] + up[1] * U) * p - up[2] * q - up[3] / R - up[4] * U / R
             - 1.5 * (1.0 - up[7] / 3.0 * U) * U ** 2 - q * up[5] * pa - up[6] * pt * R + up[8] * V ** 2)
        D = R - up[7] * R * U + up[4] * up[7]
        Fb = -up[10] * R ** 3 * px
        Fd = -up[11] * R * (V * c_ - ux)
        b0 = N / D + g0 / D + g1 * V / D
        b1 = 3.0 * (Fb + Fd) * up[9] / R ** 3 - 3.0 * U * V / R + tn + tg2 * U / R + tg3 / R ** 2
        # implicit system for the accelerations, solved exactly
        A = np.block([[np.eye(K) + Am / D[:, None], Bm / D[:, None]], [Cm, np.eye(K) + Dm]])
        acc = np.linalg.solve(A, np.concatenate([b0, b1]))
        return np.concatenate([U, V, acc])

    return f


def _oracle_tight(scene):
    spec_s = SolverSpec(rtol=1e-12, atol=1e-12, lin_rtol=1e-12, lin_atol=1e-12, lin_solver="lu")
    m = scenes.build_model(scene, solver_spec=spec_s, ndo=0)
    start = copy.deepcopy(oracle.model_buffers(m))
    buf = copy.deepcopy(start)
    es, ms = m._execution_spec, m._model_spec
    spec = oracle.make_spec(es.ns, es.ups, es.tile, 0, ms.nk, ms.ac, spec_s)
    oracle.solve_ref_layout(spec, buf, 5_000_000)
    return start, buf, ms.nk, ms.ac


@pytest.mark.parametrize("case", ["plain_K2", "mixed_K4", "swn_K8", "const_K3"])
def test_tight_reference_agrees_with_dop853(case):
    if case == "plain_K2":
        sc = scenes.subset(scenes.plain_study(ns=1024, periods=0.5, seed=0), np.arange(3))
    elif case == "mixed_K4":
        mk = scenes.mixed_k(ns=65536, seed=1)
        sc = scenes.subset(mk, np.nonzero(mk.K == 4)[0][:3])
        sc.t_end = np.minimum(sc.t_end, 0.5)
    elif case == "swn_K8":
        sc = scenes.uniform(8, ns=3, periods=0.3, seed=21, ac="SW_N")
    else:
        sc = scenes.uniform(3, ns=3, periods=0.5, seed=22, ac="CONST")
    start, tight, nk, ac = _oracle_tight(sc)
    K = int(sc.K[0])
    checked = 0
    for s in range(sc.ns):
        if tight["status_flags"][s] != 1:
            continue
        y0 = np.concatenate([start["actual_state"][c, s, :K] for c in range(4)])
        f = _rhs_factory(start, s, K, nk, ac)
        sol = scipy_integrate.solve_ivp(f, (0.0, float(start["time_end"][s])), y0, method="DOP853",
                                        rtol=1e-12, atol=1e-13)
        assert sol.success
        want = sol.y[:, -1].reshape(4, K)
        got = tight["actual_state"][:, s, :K]
        err = np.max(np.abs(got - want) / np.maximum(np.abs(want), FLOOR[:, None]), axis=1)
        assert np.all(err < 1e-8), (case, s, err)
        checked += 1
    assert checked >= 2
