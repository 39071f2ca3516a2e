"""GPU parity of the direct implicit-coupling solve (lin_solver = "lu")
against the oracle's restatement of it, bit for bit: the register form
(K <= 8: rows in registers, pivot search and pivot-row broadcast by warp
shuffles) and the shared-memory form (K = 16, 32), through the
reference-layout path and the batched mixed-K path."""
import numpy as np
import pytest

from cbc_b200 import scenes
from cbc_b200.models import SolverSpec

from _parity import assert_bit_exact, run_pair

pytestmark = pytest.mark.gpu

LU = SolverSpec(lin_solver="lu")


@pytest.mark.parametrize("K", [1, 2, 3, 4, 5, 6, 7, 8])
def test_lu_bit_exact_small_k(cuda, K):
    sc = scenes.uniform(K, ns=48, periods=0.5, seed=40 + K, samples_per_period=16)
    gpu, ref = run_pair(sc, solver_spec=LU)
    assert_bit_exact(gpu, ref)
    assert np.all(gpu["status_flags"] != 0)
    assert int(gpu["convergence_failures"].sum()) == 0


@pytest.mark.parametrize("K", [12, 16, 24, 32])
def test_lu_bit_exact_large_k(cuda, K):
    sc = scenes.uniform(K, ns=6, periods=0.05, seed=50 + K, pa_hi=1.2, x_range=(-0.5, 0.5), samples_per_period=40)
    gpu, ref = run_pair(sc, solver_spec=LU)
    assert_bit_exact(gpu, ref)


def test_lu_grid_dense_plain_study(cuda):
    sc = scenes.subset(scenes.plain_study(ns=1024, periods=1.0, samples_per_period=32, seed=0), np.arange(256))
    gpu, ref = run_pair(sc, solver_spec=SolverSpec(lin_solver="lu", dense_mode="grid"))
    assert_bit_exact(gpu, ref)


def test_lu_mixed_k_ensemble_bit_exact(cuda):
    import torch
    from cbc_b200.ensemble import Ensemble
    from test_parity_ensemble import compare, oracle_ragged
    sc = scenes.mixed_k(ns=300, span=(0.2, 0.6), seed=41)
    ens, models = Ensemble.from_scene(sc, solver_spec=LU, return_models=True)
    ens.to_device()
    plan = ens.plan(200_000)
    plan.launch()
    torch.cuda.synchronize()
    gpu = ens.to_host()
    ref = oracle_ragged(models, ens.host, 200_000, ens.solver_spec)
    compare(gpu, ref)
    assert int(gpu["conv_fail"].sum()) == 0
    plan.close()


def test_lu_ensemble_large_k_bit_exact(cuda):
    """K = 16 and 32 buckets of the batched path (blocks cut to the warps
    whose shared memory fits)."""
    import torch
    from cbc_b200.ensemble import Ensemble
    from test_parity_ensemble import compare, oracle_ragged
    a = scenes.uniform(16, ns=5, periods=0.04, seed=42, pa_hi=1.2, x_range=(-0.5, 0.5))
    b = scenes.uniform(32, ns=4, periods=0.04, seed=43, pa_hi=1.2, x_range=(-0.5, 0.5))
    sc = scenes.Scene(K=np.concatenate([a.K, b.K]), R0=a.R0 + b.R0, PA=np.hstack([a.PA, b.PA]),
                      FR=np.hstack([a.FR, b.FR]), PS=np.hstack([a.PS, b.PS]), X0=a.X0 + b.X0,
                      t_end=np.concatenate([a.t_end, b.t_end]), ac="SW_A", ndo=0)
    for spec in (LU, SolverSpec()):
        ens, models = Ensemble.from_scene(sc, solver_spec=spec, return_models=True)
        ens.to_device()
        ens.solve(200_000)
        torch.cuda.synchronize()
        compare(ens.to_host(), oracle_ragged(models, ens.host, 200_000, ens.solver_spec))
