"""Device-side admission of solve requests: packing raw requests for
``cbc_admit`` (the GPU parameter precompute) and the range allocator that
gives each admitted request its rows of a preallocated ragged ensemble.

A request is raw physics: K radii (um), positions (units of the reference
wavelength), the drive (PA in bar, frequencies in kHz, phases in units of
pi) and a span in periods.  The host only packs these numbers (one fixed-size
record of float64 per request, CBC_ADMIT_RECORD(nk) doubles) and copies the
batch to the device in one transfer; the precompute of the reference's
``CKM1D.build_parameters`` (models/ckm1d.py:133-202) runs on the GPU and is
bit-identical to the host version (cbc_b200.models.ckm1d).
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from .models.ckm1d import precompute_constants, system_constants


def consts_struct(mat_props, ref_freq_khz: float) -> _lib.cbc_precompute_consts:
    """The scalar constants of the precompute, evaluated on the host exactly
    as the host precompute evaluates them."""
    c = precompute_constants(mat_props, ref_freq_khz * 1000.0)
    out = _lib.cbc_precompute_consts()
    out.two_pi, out.pi = c["two_pi"], np.pi
    out.w_ref, out.l_ref = c["w_ref"], c["l_ref"]
    out.rho, out.cl, out.p0, out.pv = c["RHO"], c["CL"], c["P0"], c["PV"]
    for k in ("st2", "k1", "p0pv", "k4", "tw", "k6", "hl", "k9", "k10", "k11", "km2"):
        setattr(out, k, c[k])
    for i, v in enumerate(system_constants(c)):
        out.system_params[i] = v
    return out


def pack_records(K: Sequence[int], slot: Sequence[int], bubble_offset: Sequence[int],
                 coupling_offset: Sequence[int], span: Sequence[float], PA: np.ndarray, FR: np.ndarray,
                 PS: np.ndarray, R0: List[np.ndarray], X0: List[np.ndarray], out: Optional[np.ndarray] = None):
    """(n, CBC_ADMIT_RECORD(nk)) float64 records; PA / FR / PS are (n, nk)."""
    n = len(K)
    PA, FR, PS = (np.asarray(a, dtype=np.float64).reshape(n, -1) for a in (PA, FR, PS))
    nk = PA.shape[1]
    rl = _lib.admit_record_len(nk)
    rec = out[:n] if out is not None else np.zeros((n, rl))
    rec[:, 0] = K
    rec[:, 1] = slot
    rec[:, 2] = bubble_offset
    rec[:, 3] = coupling_offset
    rec[:, 4] = span
    rec[:, 5:5 + nk] = PA
    rec[:, 5 + nk:5 + 2 * nk] = FR
    rec[:, 5 + 2 * nk:5 + 3 * nk] = PS
    base = 5 + 3 * nk
    rec[:, base:] = 0.0
    Ka = np.asarray(K, np.int64)
    for k in np.unique(Ka):                    # one stacked copy per bubble count
        idx = np.nonzero(Ka == k)[0]
        rec[idx, base:base + k] = np.stack([R0[i] for i in idx])
        rec[idx, base + 32:base + 32 + k] = np.stack([X0[i] for i in idx])
    return rec


class RangeAllocator:
    """First-fit allocator of contiguous index ranges in [0, capacity)
    (rows of the bubble arrays, elements of the coupling array).  Freed
    ranges are merged with their neighbours."""

    def __init__(self, capacity: int):
        self.capacity = int(capacity)
        self.free_list = [(0, self.capacity)] if capacity > 0 else []   # sorted (start, length)
        self.used = 0

    def alloc(self, n: int) -> Optional[int]:
        n = int(n)
        for i, (start, length) in enumerate(self.free_list):
            if length >= n:
                if length == n:
                    self.free_list.pop(i)
                else:
                    self.free_list[i] = (start + n, length - n)
                self.used += n
                return start
        return None

    def free(self, start: int, n: int) -> None:
        start, n = int(start), int(n)
        fl = self.free_list
        lo, hi = 0, len(fl)
        while lo < hi:
            mid = (lo + hi) // 2
            if fl[mid][0] < start:
                lo = mid + 1
            else:
                hi = mid
        fl.insert(lo, (start, n))
        # merge with the next and the previous range
        if lo + 1 < len(fl) and fl[lo][0] + fl[lo][1] == fl[lo + 1][0]:
            fl[lo] = (fl[lo][0], fl[lo][1] + fl[lo + 1][1])
            fl.pop(lo + 1)
        if lo > 0 and fl[lo - 1][0] + fl[lo - 1][1] == fl[lo][0]:
            fl[lo - 1] = (fl[lo - 1][0], fl[lo - 1][1] + fl[lo][1])
            fl.pop(lo)
        self.used -= n

    @property
    def largest_free(self) -> int:
        return max((l for _, l in self.free_list), default=0)
