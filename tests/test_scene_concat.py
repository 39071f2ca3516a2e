"""scenes.concat keeps every system's inputs in order."""
import numpy as np
import pytest

from cbc_b200 import scenes


def test_concat_orders_systems():
    a = scenes.uniform(2, ns=3, periods=1.0, seed=1)
    b = scenes.uniform(5, ns=2, periods=2.0, seed=2)
    c = scenes.concat(a, b)
    assert list(c.K) == [2, 2, 2, 5, 5]
    assert c.PA.shape == (a.nk, 5)
    assert np.array_equal(c.R0[3], b.R0[0]) and np.array_equal(c.X0[2], a.X0[2])
    assert np.array_equal(c.t_end, np.concatenate([a.t_end, b.t_end]))
    sub = scenes.subset(c, [3, 4])
    assert np.array_equal(sub.PS, b.PS)


def test_concat_rejects_mixed_fields():
    a = scenes.uniform(2, ns=1, periods=1.0, seed=1, ac="SW_A")
    b = scenes.uniform(2, ns=1, periods=1.0, seed=1, ac="SW_N")
    with pytest.raises(ValueError):
        scenes.concat(a, b)
