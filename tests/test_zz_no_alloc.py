"""The allocation-free projection entry point (edge_mgpcg_poisson_noalloc),
called through the C ABI, against the regular solver (edge_mgpcg_poisson) on
the same input, twice in a row (the shared scratch keeps the previous call's
contents, which must not leak into the next result).

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _rel(a, b):
    a = a.double()
    b = b.double()
    return float((a - b).norm() / b.norm().clamp_min(1e-30))


def test_noalloc_matches_regular_solver_twice():
    from edgeb200 import _native as N
    from edgeb200.projection import Projection

    lib = N.load()
    torch.cuda.set_device(0)
    res = (32, 32, 16)
    base_level = 2
    bt = (ctypes.c_int * 6)(2, 2, 2, 2, 2, 2)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(123)
    shapes = [(res[0] + 1, res[1], res[2]), (res[0], res[1] + 1, res[2]), (res[0], res[1], res[2] + 1)]
    P = Projection(res, base_level=base_level)
    for call in range(2):
        u0 = [torch.from_numpy(rng.normal(size=s).astype(np.float32)).cuda() for s in shapes]
        ref = [t.clone() for t in u0]
        P.poisson(*ref)
        it_ref, rtr_ref, st_ref = P.result()
        got = [t.clone() for t in u0]
        it = ctypes.c_int(-1)
        rtr = ctypes.c_double(-1.0)
        st = ctypes.c_int(-99)
        rc = lib.edge_mgpcg_poisson_noalloc(*res, base_level, bt, *[_ptr(t) for t in got], ctypes.c_double(1e-12),
                                            ctypes.c_double(1e-12), 400, ctypes.byref(it), ctypes.byref(rtr),
                                            ctypes.byref(st), stream)
        torch.cuda.synchronize()
        assert rc == N.EDGE_OK
        assert st.value == N.EDGE_OK == st_ref
        assert it.value == it_ref
        for a, b in zip(got, ref):
            assert _rel(a, b) < 1e-5, call


def test_noalloc_rejects_grids_beyond_its_scratch():
    from edgeb200 import _native as N
    lib = N.load()
    bt = (ctypes.c_int * 6)(2, 2, 2, 2, 2, 2)
    p = ctypes.c_void_p(256)
    null = ctypes.c_void_p(0)
    rc = lib.edge_mgpcg_poisson_noalloc(128, 64, 64, 2, bt, p, p, p, ctypes.c_double(1e-12), ctypes.c_double(1e-12),
                                        400, null, null, null, null)
    assert rc == N.EDGE_EINVAL
