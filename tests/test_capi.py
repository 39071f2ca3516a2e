"""The C-ABI library loads on a machine without a GPU and exports every
symbol that include/*.h declares (no compute calls are made here)."""
import ctypes
import glob
import os
import re

import pytest

from cbc_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s+\**\s*(cbc_[a-z0-9_]+)\s*\(",
                             text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_declared_symbols():
    L = _lib.lib()
    names = declared_symbols()
    assert {"cbc_create", "cbc_destroy", "cbc_solve", "cbc_last_error", "cbc_version"} <= names
    for n in sorted(names):
        assert hasattr(L, n), f"{n} declared in include/ but not exported"


def test_version_and_errors_without_gpu():
    L = _lib.lib()
    assert L.cbc_version() >= 100
    # invalid argument path needs no device
    assert L.cbc_create(None, 0) == -1
    assert b"NULL" in L.cbc_last_error(None)


def test_python_solver_rejects_bad_shapes():
    from cbc_b200.backends import b200_solver
    from cbc_b200.models import ExecutionSpec, ModelSpec, SolverSpec
    ms = ModelSpec(name="CKM1D", sd=4, nup=13, nsp=5, ncm=3, nk=2, ne=1, ncf=4, nct=8, ac="SW_A")
    es = ExecutionSpec(ups=3, ns=10, spb=1, ndo=0)
    spec = b200_solver.make_cbc_spec(ms, es, SolverSpec())
    assert (spec.ns, spec.ups, spec.tile, spec.nk, spec.ac) == (10, 3, 4, 2, 2)
    assert abs(spec.lin_relaxation - 2.0 / 3.0) < 1e-16
