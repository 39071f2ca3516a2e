"""Device-side admission (cbc_admit): the GPU parameter precompute of raw
requests into slots of a preallocated ensemble, bit-identical to the host
precompute (Ensemble.from_scene -> CKM1D.build_parameters); and the range
allocator and record packing it relies on (CPU)."""
import ctypes

import numpy as np
import pytest

from cbc_b200 import _lib, admission, scenes
from cbc_b200.admission import RangeAllocator
from cbc_b200.ensemble import Ensemble
from cbc_b200.models import CKM1D, water


def test_range_allocator_first_fit_and_merge():
    a = RangeAllocator(100)
    x = a.alloc(30)
    y = a.alloc(30)
    z = a.alloc(30)
    assert (x, y, z) == (0, 30, 60) and a.alloc(20) is None and a.used == 90
    a.free(y, 30)
    assert a.alloc(40) is None and a.largest_free == 30
    a.free(x, 30)
    assert a.largest_free == 60            # [0, 60) merged
    assert a.alloc(50) == 0
    a.free(0, 50)
    a.free(z, 30)
    assert a.free_list == [(0, 100)] and a.used == 0


def test_pack_records_layout():
    K = [2, 3]
    rec = admission.pack_records(K, [5, 9], [10, 20], [100, 200], [3.5, 7.0], PA=[[1.0, 0.5], [0.2, 0.3]],
                                 FR=[[25.0, 50.0]] * 2, PS=[[0.1, 0.2], [0.3, 0.4]],
                                 R0=[np.array([4.0, 5.0]), np.array([2.0, 3.0, 6.0])],
                                 X0=[np.array([-0.1, 0.1]), np.array([-0.2, 0.0, 0.2])])
    assert rec.shape == (2, _lib.admit_record_len(2))
    assert list(rec[1, :5]) == [3, 9, 20, 200, 7.0]
    assert list(rec[1, 5:11]) == [0.2, 0.3, 25.0, 50.0, 0.3, 0.4]
    assert list(rec[1, 11:14]) == [2.0, 3.0, 6.0] and rec[1, 14] == 0.0
    assert list(rec[1, 43:46]) == [-0.2, 0.0, 0.2]


def test_explicit_cubes_stay_within_an_ulp_of_pow():
    """The precompute's cubes are (x * x) * x (reproducible on the GPU); the
    reference writes x ** 3.  They differ by at most one ulp."""
    rng = np.random.default_rng(7)
    x = rng.uniform(2e-6, 8e-6, 100000)
    d = np.abs((x * x) * x - x ** 3) / np.spacing(x ** 3)
    assert d.max() <= 1.0


def _ensemble_with_slots(sc):
    """A host-precomputed ensemble of `sc` and an empty one of the same
    shape into which cbc_admit writes the same requests."""
    ref = Ensemble.from_scene(sc)
    blank = Ensemble.from_scene(sc)
    for k in ("state", "unit_params", "system_params", "control_params", "coupling", "t", "t_end", "h", "event"):
        blank.host[k][...] = 0.0
    for k in ("bubble_offset", "coupling_offset"):
        blank.host[k][...] = -1
    blank.host["status"][...] = 7
    blank.host["steps"][...] = 5
    return ref, blank


@pytest.mark.gpu
def test_admit_is_bit_identical_to_host_precompute(cuda):
    import torch
    sc = scenes.mixed_k(ns=300, span=(1.0, 50.0), seed=70)
    extra = scenes.uniform(16, ns=4, periods=3.0, seed=71, x_range=(-0.5, 0.5))
    big = scenes.uniform(32, ns=3, periods=2.0, seed=72, pa_hi=1.2, x_range=(-0.5, 0.5))
    sc = scenes.Scene(K=np.concatenate([sc.K, extra.K, big.K]), R0=sc.R0 + extra.R0 + big.R0,
                      PA=np.hstack([sc.PA, extra.PA, big.PA]), FR=np.hstack([sc.FR, extra.FR, big.FR]),
                      PS=np.hstack([sc.PS, extra.PS, big.PS]), X0=sc.X0 + extra.X0 + big.X0,
                      t_end=np.concatenate([sc.t_end, extra.t_end, big.t_end]), ac="SW_A")
    ref, blank = _ensemble_with_slots(sc)
    blank.to_device()
    h = ref.host
    n = sc.ns
    perm = np.random.default_rng(1).permutation(n)          # any order of requests
    rec = admission.pack_records(sc.K[perm], perm, h["bubble_offset"][perm], h["coupling_offset"][perm],
                                 sc.t_end[perm], sc.PA.T[perm], sc.FR.T[perm], sc.PS.T[perm],
                                 [sc.R0[i] for i in perm], [sc.X0[i] for i in perm])
    d_rec = torch.from_numpy(np.ascontiguousarray(rec)).cuda()
    ctx = _lib.default_context(0)
    consts = admission.consts_struct(water(), scenes.REF_FREQ_KHZ)
    e = blank.abi()
    ctx.check(_lib.lib().cbc_admit(ctx.handle, ctypes.byref(e), ctypes.byref(consts), d_rec.data_ptr(), n,
                                   sc.nk, int(blank.dev["coupling"].numel()), None))
    torch.cuda.synchronize()
    got = blank.to_host()
    for k in ("bubble_offset", "coupling_offset", "state", "system_params", "control_params", "coupling", "t",
              "t_end", "t_begin", "h", "event", "status", "steps", "rejected", "conv_ok", "conv_fail", "lin_iters"):
        assert np.array_equal(got[k], h[k]), k
    assert np.array_equal(got["unit_params"][:, :13], h["unit_params"][:, :13])


@pytest.mark.gpu
def test_admit_skips_records_outside_the_ensemble(cuda):
    import torch
    sc = scenes.mixed_k(ns=20, span=(1.0, 2.0), seed=73)
    ref, blank = _ensemble_with_slots(sc)
    blank.to_device()
    h = ref.host
    rec = admission.pack_records(sc.K[:3], [0, 25, 1], [h["bubble_offset"][0], 0, 10 ** 9],
                                 [h["coupling_offset"][0], 0, 0], [1.0] * 3, sc.PA.T[:3], sc.FR.T[:3],
                                 sc.PS.T[:3], sc.R0[:3], sc.X0[:3])
    d_rec = torch.from_numpy(rec).cuda()
    ctx = _lib.default_context(0)
    consts = admission.consts_struct(water(), scenes.REF_FREQ_KHZ)
    e = blank.abi()
    ctx.check(_lib.lib().cbc_admit(ctx.handle, ctypes.byref(e), ctypes.byref(consts), d_rec.data_ptr(), 3,
                                   sc.nk, int(blank.dev["coupling"].numel()), None))
    torch.cuda.synchronize()
    got = blank.to_host()
    assert got["status"][0] == 0 and got["status"][1] == 7          # slot 1's record had a bad bubble offset
    assert np.all(got["status"][2:] == 7)
