"""The C-ABI library: it loads without a GPU, exports every symbol that
include/edge_b200.h declares, and rejects bad arguments before touching the
device (no compute calls here)."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

from edgeb200 import _native as N


def test_header_symbols_exported():
    sig = N.parse_header()
    assert len(sig) >= 39
    lib = N.load()
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIBPATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (edge_\w+)", out))
    missing = sorted(set(sig) - exported)
    assert not missing, f"declared but not exported: {missing}"
    for name in sig:
        assert hasattr(lib, name)


def test_no_undeclared_exports():
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIBPATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (edge_\w+)", out))
    assert exported <= set(N.parse_header())


def test_version_and_errors():
    lib = N.load()
    assert lib.edge_version() >= 10000
    for code in (N.EDGE_OK, N.EDGE_EINVAL, N.EDGE_EALIGN, N.EDGE_ENOCONV, N.EDGE_ENAN, N.EDGE_ESTALL):
        assert lib.edge_error_string(code)


def test_argument_validation_without_device():
    """Null pointers / bad sizes / aliasing fail with EDGE_EINVAL before any
    CUDA call, so these run on a machine without a GPU."""
    lib = N.load()
    null = ctypes.c_void_p(0)
    f = ctypes.c_float
    assert lib.edge_march_edge(64, 32, 32, f(1 / 32), f(0.01), f(1e-4), null, null, null, null, null, null, null,
                               null, null, null, null, null, null, null, null, null, null, 0, null) == N.EDGE_EINVAL
    # a 3-cell axis is below the Hermite stencil
    p = ctypes.c_void_p(16)
    assert lib.edge_advect_u_sl(3, 8, 8, f(0.1), f(0.01), p, p, p, ctypes.c_void_p(32), ctypes.c_void_p(48),
                                ctypes.c_void_p(64), null) == N.EDGE_EINVAL
    # output aliasing its input is refused
    assert lib.edge_advect_u_sl(8, 8, 8, f(0.1), f(0.01), p, p, p, p, p, p, null) == N.EDGE_EINVAL
    # vec4 dye pointers must be 16-byte aligned
    q = ctypes.c_void_p(20)
    assert lib.edge_pullback_dye(8, 8, 8, f(0.1), q, p, p, p, null, f(1), null, null, 0, ctypes.c_void_p(64),
                                 null) == N.EDGE_EALIGN
    # multigrid: every level must halve exactly (restrict writes r[l+1][I//2])
    h = ctypes.c_void_p()
    bt = (ctypes.c_int * 6)(2, 2, 2, 2, 2, 2)
    assert lib.edge_mgpcg_create(ctypes.byref(h), 10, 8, 8, 1, bt, null, null, 0) == N.EDGE_EINVAL
    assert lib.edge_mgpcg_create(ctypes.byref(h), 16, 8, 8, 1, bt, null, null, 7) == N.EDGE_EINVAL
    # the allocation-free projection refuses grids beyond its static scratch
    # (64^3 cells) before any CUDA call
    assert lib.edge_mgpcg_poisson_noalloc(128, 64, 64, 2, bt, p, p, p, ctypes.c_double(1e-12),
                                          ctypes.c_double(1e-12), 400, null, null, null, null) == N.EDGE_EINVAL


def test_python_side_has_no_fallback(monkeypatch):
    """The host package refuses to run when the library is missing."""
    monkeypatch.setattr(N, "_lib", None)
    monkeypatch.setattr(N, "LIBPATH", os.path.join(ROOT, "does-not-exist.so"))
    with pytest.raises(RuntimeError):
        N.load()
