"""Accuracy of the shared FP64 elementary functions (cbc_math.h) against
numpy/glibc.  The CUDA kernels and the oracle both use these routines, so
this is the independent check of their accuracy."""
import numpy as np

from oracle import oracle


def _ulps(a, b):
    scale = np.spacing(np.maximum(np.abs(b), np.finfo(np.float64).tiny))
    return np.abs(a - b) / scale


def test_sincos():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(-4, 4, 200_000), rng.uniform(-3e3, 3e3, 200_000),
                        rng.uniform(-2e5, 2e5, 50_000), [0.0, -0.0, np.pi / 4, np.pi / 2, np.pi]])
    s = oracle.math_eval(0, x)
    c = oracle.math_eval(1, x)
    # absolute error in units of ulp(1) near zeros of sin/cos, relative elsewhere
    es = np.abs(s - np.sin(x)) / np.maximum(np.spacing(np.abs(np.sin(x))), np.spacing(1.0) * 1e-3)
    ec = np.abs(c - np.cos(x)) / np.maximum(np.spacing(np.abs(np.cos(x))), np.spacing(1.0) * 1e-3)
    big = np.abs(x) < 4e3
    assert np.max(es[big]) <= 2.0 and np.max(ec[big]) <= 2.0
    assert np.max(np.abs(s - np.sin(x))) < 1e-11 and np.max(np.abs(c - np.cos(x))) < 1e-11
    assert np.all(np.isnan(oracle.math_eval(0, np.array([np.inf, -np.inf, np.nan]))))


def test_exp_log_pow():
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(-700, 700, 200_000), rng.uniform(-3, 3, 200_000), [0.0, 1.0, -1.0]])
    assert np.max(_ulps(oracle.math_eval(2, x), np.exp(x))) <= 2.0
    z = np.concatenate([np.exp(rng.uniform(-700, 700, 200_000)), rng.uniform(0.5, 2.0, 200_000),
                        [1.0, 2.0, 1e-310, 5e-324]])
    assert np.max(_ulps(oracle.math_eval(3, z), np.log(z))) <= 2.0
    b = np.exp(rng.uniform(-5, 5, 200_000))
    y = np.full_like(b, 4.2)
    rel = np.abs(oracle.math_eval(4, b, y) - b ** 4.2) / b ** 4.2
    assert np.max(rel) < 1e-14
    assert oracle.math_eval(3, np.array([0.0]))[0] == -np.inf
    assert np.isnan(oracle.math_eval(3, np.array([-1.0]))[0])
    assert oracle.math_eval(2, np.array([800.0]))[0] == np.inf
    assert oracle.math_eval(2, np.array([-800.0]))[0] == 0.0


def test_special_values():
    """Non-finite, zero, subnormal and range-edge arguments (the routines
    select these results instead of branching)."""
    inf, nan = np.inf, np.nan
    e = oracle.math_eval(2, np.array([nan, inf, -inf, 709.7, -745.1, -740.0, -1e-320, 0.0, -0.0]))
    assert np.isnan(e[0]) and e[1] == inf and e[2] == 0.0
    ref = np.exp(np.array([709.7, -745.1, -740.0]))
    assert np.all(_ulps(e[3:6], ref) <= 2.0)
    assert e[6] == 1.0 and e[7] == 1.0 and e[8] == 1.0
    lg = oracle.math_eval(3, np.array([nan, inf, -inf, -0.0, 0.0, 5e-324, 2.2e-308, 1.7e308, -2.0]))
    assert np.isnan(lg[0]) and lg[1] == inf and np.isnan(lg[2]) and lg[3] == -inf and lg[4] == -inf
    assert np.all(_ulps(lg[5:8], np.log(np.array([5e-324, 2.2e-308, 1.7e308]))) <= 2.0)
    assert np.isnan(lg[8])
    for kind in (0, 1):
        v = oracle.math_eval(kind, np.array([inf, -inf, nan, 0.0, -0.0]))
        assert np.all(np.isnan(v[:3]))
    assert oracle.math_eval(0, np.array([0.0]))[0] == 0.0 and oracle.math_eval(1, np.array([0.0]))[0] == 1.0
