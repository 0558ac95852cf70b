"""The C-ABI library loads and exports what include/cugmres.h declares (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT
import cugmres_b200 as cg
from cugmres_b200 import _lib

HEADER = os.path.join(ROOT, "include", "cugmres.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cugmres_\w+)\s*\(", src)))


def test_header_and_binding_agree():
    assert declared() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    for name in declared():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    syms = set(l.split()[-1] for l in out.splitlines() if l.strip())
    for name in declared():
        assert name in syms, name


def test_strerror_and_defaults():
    lib = _lib.lib()
    assert lib.cugmres_strerror(0).decode() == "ok"
    assert "not converged" in lib.cugmres_strerror(3).decode()
    o = _lib.CgOpts()
    lib.cugmres_default_opts(ctypes.byref(o))
    assert o.restart == 100 and o.tol == 1e-10 and o.precision == 0 and o.givens == 0


def test_green_block_host_path(oracle):
    g = cg.green_block("reference", 32)
    assert np.array_equal(g, oracle.green_block_reference(32, True))
    h = cg.green_block("helmholtz", 16, 2 * np.pi, 0.05)
    assert np.abs(h - oracle.green_block_helmholtz(16, 2 * np.pi, 0.05)).max() < 1e-15
    with pytest.raises(cg.CugmresError):
        cg.green_block("helmholtz", 16, -1.0, 0.05)


def test_invalid_arguments_return_codes():
    lib = _lib.lib()
    assert lib.cugmres_create(None, 0) == _lib.CG_ERR_INVALID
    assert lib.cugmres_solve(None, None, None, None, None, 0, None) == _lib.CG_ERR_INVALID
    assert lib.cugmres_matvec(None, None, None, 0) == _lib.CG_ERR_INVALID
    assert lib.cugmres_green_block(7, 4, 1.0, 1.0, None) == _lib.CG_ERR_INVALID
