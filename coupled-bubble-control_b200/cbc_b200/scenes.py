"""Seeded synthetic workloads of the CKM1D parameter studies.

The reference publishes no benchmark dataset; these generators produce the
parameter distributions its study and benchmark scripts use
(``scripts/benchmarks/kernel_prof.py:65-145``, ``scripts/verify_CKM1D_paramstudy.py``)
at the sizes of the headline workloads:

* ``plain_study``   1024 systems, K=2, 10 periods, 32 dense samples/period
* ``mixed_k``       65,536 systems, K in {2,3,4,6,8} (p .4/.2/.2/.1/.1),
                    spans U[5,50] periods, no dense output
* ``vec_env``       1024 envs, K=4, R0 = 60 um, SW_N, 5 periods per env step
* ``served``        Poisson request stream, K in {2,4,8,16}, spans U[1,50]
* ``large_k``       16,384 systems, K=32, 200 periods, 64 samples/period

Physics shared by all: water (rho 998, c 1497, sigma 0.0728, mu 1e-3,
P_inf 1 bar, p_v 2.33 kPa, gamma 1.4), standing wave SW_A with two
harmonics at 25 and 50 kHz, reference frequency 25 kHz (one dimensionless
time unit = one period of 25 kHz, positions in units of lambda_1 = c/25 kHz).

Draw order from ``np.random.default_rng(seed)``: K per system (mixed
workloads) -> R0 (um) -> PA (bar, shape (NK, NS)) -> phase phi (rad) ->
positions -> spans.  Positions use exact uniform spacings: K sorted uniform
draws on a range shortened by (K-1) * gap_min, then the i-th point is shifted
by i * gap_min, so every neighbour gap is >= 20 * max(R0) / lambda_1.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

REF_FREQ_KHZ = 25.0
FREQS_KHZ = (25.0, 50.0)
C_WATER = 1497.0
LAMBDA1 = C_WATER / (REF_FREQ_KHZ * 1e3)   # m


@dataclass
class Scene:
    """One batch of independent systems (ragged in K when mixed)."""
    K: np.ndarray            # (NS,) int32 bubbles per system
    R0: List[np.ndarray]     # per system, (K_s,) um
    PA: np.ndarray           # (NK, NS) bar
    FR: np.ndarray           # (NK, NS) kHz
    PS: np.ndarray           # (NK, NS) phase in units of pi (reference convention)
    X0: List[np.ndarray]     # per system, (K_s,) dimensionless positions x / lambda_1
    t_end: np.ndarray        # (NS,) dimensionless spans (periods of 25 kHz)
    ac: str = "SW_A"
    ndo: int = 0
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def ns(self) -> int:
        return int(self.K.shape[0])

    @property
    def nk(self) -> int:
        return int(self.PA.shape[0])

    def system_periods(self) -> float:
        return float(np.sum(self.t_end))


def _positions(rng, K: int, r0max_um: float, lo: float, hi: float) -> np.ndarray:
    gmin = 20.0 * r0max_um * 1e-6 / LAMBDA1
    span = (hi - lo) - (K - 1) * gmin
    if span <= 0:
        raise ValueError(f"cannot place {K} bubbles with gap {gmin:.3g} in [{lo}, {hi}]")
    u = np.sort(rng.uniform(0.0, span, size=K))
    return lo + u + np.arange(K) * gmin


def _scene(rng, Ks: np.ndarray, pa_hi: float, x_lo: float, x_hi: float, spans: Optional[np.ndarray],
           t_fixed: float, ndo: int, name: str, r0=(2.0, 8.0)) -> Scene:
    NS = Ks.shape[0]
    NK = len(FREQS_KHZ)
    R0 = [rng.uniform(r0[0], r0[1], size=int(k)) for k in Ks]
    PA = rng.uniform(0.0, pa_hi, size=(NK, NS))
    phi = rng.uniform(0.0, 2.0 * np.pi, size=(NK, NS))
    X0 = [_positions(rng, int(k), float(np.max(R0[s])), x_lo, x_hi) for s, k in enumerate(Ks)]
    if spans is None:
        t_end = np.full(NS, float(t_fixed))
    else:
        t_end = spans
    FR = np.tile(np.asarray(FREQS_KHZ, dtype=np.float64)[:, None], (1, NS))
    return Scene(K=Ks.astype(np.int32), R0=R0, PA=PA, FR=FR, PS=phi / np.pi, X0=X0,
                 t_end=np.asarray(t_end, dtype=np.float64), ac="SW_A", ndo=ndo, name=name)


def plain_study(ns: int = 1024, periods: float = 10.0, samples_per_period: int = 32, seed: int = 0) -> Scene:
    rng = np.random.default_rng(seed)
    Ks = np.full(ns, 2, dtype=np.int32)
    ndo = int(round(periods * samples_per_period)) + 1 if samples_per_period > 0 else 0
    return _scene(rng, Ks, 1.5, -0.25, 0.25, None, periods, ndo, "plain_study")


def uniform(K: int, ns: int, periods: float, seed: int = 0, pa_hi: float = 1.5, ac: str = "SW_A",
            samples_per_period: int = 0, x_range=(-0.25, 0.25)) -> Scene:
    """Parameter-study scene with a fixed number of bubbles per system."""
    rng = np.random.default_rng(seed)
    Ks = np.full(ns, K, dtype=np.int32)
    ndo = int(round(periods * samples_per_period)) + 1 if samples_per_period > 0 else 0
    sc = _scene(rng, Ks, pa_hi, x_range[0], x_range[1], None, periods, ndo, f"uniform_K{K}")
    sc.ac = ac
    return sc


MIXED_K = (2, 3, 4, 6, 8)
MIXED_P = (0.4, 0.2, 0.2, 0.1, 0.1)


def mixed_k(ns: int = 65536, span=(5.0, 50.0), seed: int = 1) -> Scene:
    rng = np.random.default_rng(seed)
    Ks = rng.choice(np.asarray(MIXED_K, dtype=np.int32), size=ns, p=np.asarray(MIXED_P))
    sc = _scene(rng, Ks, 1.5, -0.25, 0.25, None, 0.0, 0, "mixed_k")
    sc.t_end = rng.uniform(span[0], span[1], size=ns)
    return sc


def large_k(ns: int = 16384, K: int = 32, periods: float = 200.0, samples_per_period: int = 64,
            seed: int = 4) -> Scene:
    rng = np.random.default_rng(seed)
    Ks = np.full(ns, K, dtype=np.int32)
    ndo = int(round(periods * samples_per_period)) + 1
    return _scene(rng, Ks, 1.2, -0.5, 0.5, None, periods, ndo, "large_k")


def served_stream(duration_s: float = 60.0, rate_hz: float = 20000.0, seed: int = 3, max_requests=None):
    """Arrival times (s) and the scene of all requests of a Poisson stream."""
    rng = np.random.default_rng(seed)
    n = int(rng.poisson(rate_hz * duration_s)) if max_requests is None else int(max_requests)
    Ks = rng.choice(np.asarray((2, 4, 8, 16), dtype=np.int32), size=n)
    sc = _scene(rng, Ks, 1.5, -0.25, 0.25, None, 0.0, 0, "served")
    sc.t_end = rng.uniform(1.0, 50.0, size=n)
    gaps = rng.exponential(1.0 / rate_hz, size=n)
    return np.cumsum(gaps), sc


def to_padded(scene: Scene):
    """(R0, X0) as (NS, K) arrays for a uniform-K scene (reference layout inputs)."""
    K = int(scene.K[0])
    if not np.all(scene.K == K):
        raise ValueError("scene is ragged; split it by K first")
    return np.stack(scene.R0), np.stack(scene.X0)


def subset(scene: Scene, idx) -> Scene:
    idx = np.asarray(idx)
    return Scene(K=scene.K[idx], R0=[scene.R0[i] for i in idx], PA=scene.PA[:, idx], FR=scene.FR[:, idx],
                 PS=scene.PS[:, idx], X0=[scene.X0[i] for i in idx], t_end=scene.t_end[idx], ac=scene.ac,
                 ndo=scene.ndo, name=scene.name, meta=dict(scene.meta))


def concat(*parts: Scene) -> Scene:
    """One scene holding the systems of `parts` in order (same field type)."""
    if not parts:
        raise ValueError("nothing to concatenate")
    if len({p.ac for p in parts}) != 1 or len({p.nk for p in parts}) != 1:
        raise ValueError("scenes differ in field type or harmonics count")
    return Scene(K=np.concatenate([p.K for p in parts]), R0=[r for p in parts for r in p.R0],
                 PA=np.hstack([p.PA for p in parts]), FR=np.hstack([p.FR for p in parts]),
                 PS=np.hstack([p.PS for p in parts]), X0=[x for p in parts for x in p.X0],
                 t_end=np.concatenate([p.t_end for p in parts]), ac=parts[0].ac, ndo=max(p.ndo for p in parts),
                 name="+".join(p.name for p in parts if p.name))


def build_model(scene: Scene, solver_spec=None, backend=None, ndo: Optional[int] = None):
    """A ``CKM1D`` model (uniform K) whose host buffers hold the scene.

    Mirrors how the reference's study scripts set up a run
    (``scripts/benchmarks/kernel_prof.py:304-335``): construct, then write
    ``time_end`` and the initial positions into the host buffers.
    """
    from .models import CKM1D, water
    from .backends import BackendName
    R0, X0 = to_padded(scene)
    ns, K = R0.shape
    model = CKM1D(num_systems=ns, systems_per_block=1, units_per_system=K, R0=R0, PA=scene.PA,
                  FR=scene.FR, PS=scene.PS, REF_FREQ=REF_FREQ_KHZ, num_components=scene.nk,
                  acoustic_field=scene.ac, mat_props=water(),
                  backend=backend if backend is not None else BackendName.B200,
                  num_stored_points=scene.ndo if ndo is None else ndo, solver_spec=solver_spec)
    hb = model.runtime.host_buffers
    hb.state.time_end[:] = scene.t_end
    hb.state.actual_state[1, :, :K] = X0
    return model
