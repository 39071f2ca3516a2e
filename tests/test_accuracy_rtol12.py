"""Accuracy of the integrator at the benchmark tolerance (rtol = atol = 1e-9)
against the same integrator at rtol = atol = 1e-12, on small seeded samples
of each workload.  The CUDA kernels are bit-identical to the oracle used
here (the -m gpu parity tests), so these are the errors of the GPU results.

Errors are relative, with floors at the typical size of each component
(R/R0: 1, x/lambda: 1e-3, dR/dt: 1e-2, dx/dt: 1e-3), taken over every dense
sample (configs with dense output) or the end state, for the systems that
complete at both tolerances.  Observed maxima:

  plain study, K=2, 2 periods, 65 samples:   R 3.4e-7  x 1.4e-10  U 9.1e-6  V 1.2e-6
  mixed-K, K=2/4/8, end state (<= 2 periods): R 4.7e-8  x 5.7e-10  U 5.7e-6  V 4.3e-8
  vec-env like, K=4 SW_N, 5 periods:          R 1.3e-6  x 5.1e-8   U 2.1e-6  V 2.2e-6
  served like, K=16, 1 period:                R 7.9e-10 x 1.4e-11  U 2.5e-8  V 2.4e-11
  large-K dense, K=32, 0.5 period, 33 samples: R 6.6e-10 x 2.0e-12 U 6.3e-6  V 1.3e-9

(medians 3e-12 .. 1e-10; the maxima come from the collapse phase, where
dR/dt changes by orders of magnitude within a few steps).  The bounds below
guard against regressions with a margin.

The direct coupling solve (lin_solver = "lu") at rtol = atol = 1e-9 against
the tight direct-solve solution, same cases:

  plain study:  R 3.4e-7  x 1.5e-10  U 7.4e-6  V 1.2e-6
  mixed-K:      R <= 3.1e-8  x <= 2.0e-10  U <= 4.2e-6  V <= 6.3e-9
  vec-env like: R 1.0e-7  x 1.2e-8   U 1.5e-7  V 1.8e-7
  served like:  R 1.5e-9  x 3.9e-12  U 6.6e-8  V 1.8e-11
  large-K:      R 6.3e-10 x 2.4e-14  U 8.7e-7  V 1.2e-9

-- as accurate as the Richardson path or more (the iteration's 1e-9 residual
is one more error source), and the tight Richardson and tight direct
solutions agree to the digits above.
"""
import copy

import numpy as np
import pytest

from cbc_b200 import scenes
from cbc_b200.models import SolverSpec
from oracle import oracle

FLOOR = np.array([1.0, 1e-3, 1e-2, 1e-3])     # R, x, dR/dt, dx/dt
BOUND = np.array([1e-5, 1e-6, 1e-4, 1e-4])


def _run(scene, rtol, ndo, lin="richardson"):
    spec_s = SolverSpec(rtol=rtol, atol=rtol, lin_rtol=min(1e-9, rtol), lin_atol=min(1e-9, rtol),
                        dense_mode="grid", lin_solver=lin)
    m = scenes.build_model(scene, solver_spec=spec_s, ndo=ndo)
    buf = copy.deepcopy(oracle.model_buffers(m))
    es, ms = m._execution_spec, m._model_spec
    spec = oracle.make_spec(es.ns, es.ups, es.tile, ndo, ms.nk, ms.ac, spec_s)
    buf["lin_iters"] = np.zeros(es.ns, np.int64)
    oracle.solve_ref_layout(spec, buf, 5_000_000)
    return buf


def _max_errors(scene, ndo, lin="richardson"):
    a, b = _run(scene, 1e-9, ndo, lin), _run(scene, 1e-12, ndo, lin)
    K = int(scene.K[0])
    ok = (a["status_flags"] == 1) & (b["status_flags"] == 1)
    assert np.any(ok)
    if ndo > 0:
        sa, sb = a["dense_state"][:, :, ok, :K], b["dense_state"][:, :, ok, :K]   # (ndo, 4, ns, K)
        err = np.abs(sa - sb) / np.maximum(np.abs(sb), FLOOR[None, :, None, None])
        return np.max(err, axis=(0, 2, 3))
    sa, sb = a["actual_state"][:, ok, :K], b["actual_state"][:, ok, :K]
    err = np.abs(sa - sb) / np.maximum(np.abs(sb), FLOOR[:, None, None])
    return np.max(err, axis=(1, 2))


def _cases():
    sc0 = scenes.subset(scenes.plain_study(ns=1024, periods=2.0, samples_per_period=32, seed=0), np.arange(16))
    yield "plain_K2_dense", sc0, sc0.ndo
    mk = scenes.mixed_k(ns=65536, seed=1)
    for k in (2, 4, 8):
        s = scenes.subset(mk, np.nonzero(mk.K == k)[0][:8])
        s.t_end = np.minimum(s.t_end, 2.0)
        yield f"mixed_K{k}", s, 0
    yield "env_K4_SWN", scenes.uniform(4, 8, 5.0, seed=2, ac="SW_N"), 0
    yield "served_K16", scenes.uniform(16, 2, 1.0, seed=3), 0
    s4 = scenes.large_k(ns=2, K=32, periods=0.5, samples_per_period=64, seed=4)
    yield "large_K32_dense", s4, s4.ndo


@pytest.mark.parametrize("name,scene,ndo", list(_cases()), ids=lambda v: v if isinstance(v, str) else "")
def test_error_against_tight_tolerance(name, scene, ndo):
    e = _max_errors(scene, ndo)
    assert np.all(e <= BOUND), f"{name}: max rel err (R, x, U, V) = {e}"


@pytest.mark.parametrize("name,scene,ndo", list(_cases()), ids=lambda v: v if isinstance(v, str) else "")
def test_direct_solve_error_against_tight_tolerance(name, scene, ndo):
    e = _max_errors(scene, ndo, lin="lu")
    assert np.all(e <= BOUND), f"{name}: max rel err (R, x, U, V) = {e}"
