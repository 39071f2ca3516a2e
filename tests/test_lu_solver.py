"""The direct implicit-coupling solve (lin_solver = "lu") of the oracle,
which the CUDA kernels reproduce bit for bit (tests/test_parity_lu.py).

* On random augmented systems of the coupling's shape (unit diagonal, rows
  R_i / T_i) it matches numpy's LAPACK solve to 1e-12 relative.
* Partial pivoting: a system whose diagonal is zero is solved (the pivot
  search exchanges rows), and a singular one reports failure.
* In whole integrations it removes the Richardson iteration's convergence
  failures.  The two solvers are different algorithms (Richardson stops at a
  1e-9 relative residual), so their trajectories agree to the integrator's
  own tolerance-level error, not bit for bit: over the first tenth of a
  period every sample agrees to 1e-6 relative (observed 4.4e-7 on dR/dt).
  Against a tight solution both are equally accurate
  (tests/test_accuracy_rtol12.py).
"""
import numpy as np
import pytest

from cbc_b200 import scenes
from cbc_b200.models import SolverSpec
from oracle import oracle


def _coupling_like(K, rng, scale=0.3):
    n = 2 * K
    a = rng.uniform(-scale / K, scale / K, size=(n, n))
    for i in range(K):
        a[i, i] = 1.0
        a[i, K + i] = 0.0
        a[K + i, i] = 0.0
        a[K + i, K + i] = 1.0
    b = rng.normal(size=n)
    return np.hstack([a, b[:, None]])


@pytest.mark.parametrize("K", [1, 2, 3, 4, 5, 8, 16, 32])
def test_matches_lapack(K):
    rng = np.random.default_rng(100 + K)
    for _ in range(20):
        aug = _coupling_like(K, rng)
        x, ok, _ = oracle.lu_solve(aug)
        assert ok
        ref = np.linalg.solve(aug[:, :-1], aug[:, -1])
        assert np.max(np.abs(x - ref) / np.maximum(np.abs(ref), 1e-12)) < 1e-12


def test_pivoting_exchanges_rows():
    # zero diagonal: elimination without row exchanges would divide by zero
    K = 2
    a = np.array([[0.0, 2.0, 1.0, 0.0],
                  [3.0, 0.0, 0.0, 1.0],
                  [1.0, 1.0, 0.0, 0.0],
                  [0.0, 1.0, 2.0, 0.5]])
    b = np.array([1.0, 2.0, 3.0, 4.0])
    x, ok, _ = oracle.lu_solve(np.hstack([a, b[:, None]]))
    assert ok
    np.testing.assert_allclose(x, np.linalg.solve(a, b), rtol=1e-13)


def test_equal_magnitude_candidates_solve():
    # column 0 has |a| = 2 in rows 1 and 3 (the pivot search takes row 1,
    # the smaller index, on the CPU and the GPU alike)
    a = np.array([[1.0, 0.0, 0.0, 0.0, 1.0],
                  [2.0, 1.0, 0.0, 0.0, 1.0],
                  [0.0, 0.0, 1.0, 0.0, 1.0],
                  [-2.0, 1.0, 0.0, 1.0, 1.0]])
    x, ok, _ = oracle.lu_solve(a)
    assert ok
    np.testing.assert_allclose(x, np.linalg.solve(a[:, :4], a[:, 4]), rtol=1e-14)


def test_singular_reports_failure():
    K = 2
    a = np.zeros((4, 5))
    a[:, :4] = np.outer(np.arange(1.0, 5.0), np.ones(4))
    _, ok, _ = oracle.lu_solve(a)
    assert not ok


def _solve(scene, lin, ndo=None):
    m = scenes.build_model(scene, solver_spec=SolverSpec(lin_solver=lin, dense_mode="grid"), ndo=ndo)
    return oracle.solve_model(m, max_steps=1_000_000, kernel_steps=1_000_000)


def test_integration_agrees_with_richardson_early():
    """First tenth of a period of the plain study (before any collapse),
    10 dense samples: every sample within 1e-6 relative (floors at the
    components' typical sizes)."""
    sc = scenes.subset(scenes.plain_study(ns=1024, periods=0.1, samples_per_period=90, seed=0), np.arange(64))
    a, b = _solve(sc, "richardson"), _solve(sc, "lu")
    assert np.all(a["status_flags"] == 1) and np.all(b["status_flags"] == 1)
    floor = np.array([1.0, 1e-3, 1e-2, 1e-3])[None, :, None, None]
    da, db = a["dense_state"][:, :, :, :2], b["dense_state"][:, :, :, :2]
    err = np.abs(da - db) / np.maximum(np.abs(da), floor)
    assert np.max(err) < 1e-6, np.max(err, axis=(0, 2, 3))
    assert int(b["convergence_failures"].sum()) == 0
    assert np.all(b["lin_iters"] == 6 * b["total_steps"])     # one direct solve per RHS


def test_direct_solve_has_no_convergence_failures():
    """Systems of the mixed-K workload whose Richardson iteration fails
    (status -3) integrate on with the direct solve."""
    mk = scenes.mixed_k(ns=65536, seed=1)
    sel = np.nonzero(mk.K == 8)[0][:48]
    sc = scenes.subset(mk, sel)
    sc.t_end = np.minimum(sc.t_end, 3.0)
    a, b = _solve(sc, "richardson", ndo=0), _solve(sc, "lu", ndo=0)
    assert int(b["convergence_failures"].sum()) == 0
    assert not np.any(b["status_flags"] == -3)
