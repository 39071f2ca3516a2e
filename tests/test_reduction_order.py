"""The canonical sum order shared by the kernels and the oracle.

Sums over the bubbles of a system (the norms of the implicit-coupling
iteration) are pairwise trees over the next power of two with zero padding.
The kernels evaluate them with warp shuffles: at level w every lane adds the
partial sum of the block starting at (li ^ w) & ~(w - 1).  This test emulates
that lane program on the CPU and checks that every lane ends with exactly the
oracle's tree_sum, for every group size the kernels support."""
import numpy as np
import pytest


def oracle_tree(a):
    K = len(a)
    P = 1
    while P < K:
        P <<= 1
    buf = list(a) + [0.0] * (P - K)
    w = 1
    while w < P:
        for i in range(0, P, 2 * w):
            buf[i] = buf[i] + buf[i + w]
        w <<= 1
    return buf[0]


def lanes_tree(a, KB):
    K = len(a)
    v = list(a)
    w = 1
    while w < KB:
        if w < K:
            v = [v[li] + (v[(li ^ w) & ~(w - 1)] if ((li ^ w) & ~(w - 1)) < K else 0.0) for li in range(K)]
        w <<= 1
    return v


@pytest.mark.parametrize("K", list(range(1, 33)))
def test_lane_tree_equals_oracle_tree(K):
    KB = 2
    while KB < K:
        KB <<= 1
    rng = np.random.default_rng(K)
    for _ in range(100):
        a = list(rng.standard_normal(K) * 10.0 ** rng.integers(-6, 6, K))
        ref = oracle_tree(a)
        assert all(x == ref for x in lanes_tree(a, KB))


def test_tree_differs_from_sequential_for_some_inputs():
    # the order matters: a sequential sum is not an acceptable substitute
    a = [1.0, 1e-16, 1e-16, 1e-16]
    seq = ((a[0] + a[1]) + a[2]) + a[3]
    assert seq == 1.0
    assert oracle_tree(a) == 1.0 + 2e-16 != seq


def open_tree(a, N):
    """The kernels' tree_open over an N-slot register array holding n = len(a)
    values (unrolled loops over the compile-time N, predicated on n)."""
    n = len(a)
    s = list(a) + [0.0] * (N - n)
    w = 1
    while w < N:
        for i in range(0, N - w, 2 * w):
            if i + w < n:
                s[i] = s[i] + s[i + w]
        w <<= 1
    return s[0] if n > 0 else 0.0


def oracle_open(a):
    """oracle tree_sum_open: at width w < n, a[i] += a[i + w] for i + w < n."""
    s = list(a)
    n = len(s)
    if n == 0:
        return 0.0
    w = 1
    while w < n:
        for i in range(0, n - w, 2 * w):
            s[i] = s[i] + s[i + w]
        w <<= 1
    return s[0]


@pytest.mark.parametrize("KB", [2, 4, 8, 16, 32])
def test_open_tree_matches_oracle_and_padded_for_norms(KB):
    rng = np.random.default_rng(KB)
    for n in range(0, KB + 1):
        a = (rng.standard_normal(n) * 10.0 ** rng.integers(-8, 8, n)).tolist()
        assert open_tree(a, KB) == oracle_open(a)
        nonneg = [x * x for x in a]
        if n:
            assert open_tree(nonneg, KB) == oracle_tree(nonneg)
