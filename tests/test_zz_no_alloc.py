"""The allocation-free projection entry point (edge_mgpcg_poisson_noalloc),
called through the C ABI, against the regular solver (edge_mgpcg_poisson) on
the same input.  Some callers cannot allocate device memory while they run
(a host runtime that owns the whole device heap, an engine that forbids
cudaMalloc after warm-up); this entry point serves them from static scratch.

The calls come in a row on two shapes: the shared scratch keeps the previous
call's contents, which must not leak into the next result, and the second
shape (five levels down to an odd 3^3 grid, whose colour planes carry padding
slots) places its levels at other offsets than the first.

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


@pytest.mark.parametrize("cases", [[((32, 32, 16), 2), ((32, 32, 16), 2), ((48, 48, 48), 1), ((32, 32, 16), 2)]])
def test_noalloc_matches_regular_solver_in_a_row(cases):
    from edgeb200 import _native as N
    from edgeb200.projection import Projection

    lib = N.load()
    torch.cuda.set_device(0)
    bt = (ctypes.c_int * 6)(2, 2, 2, 2, 2, 2)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(123)
    for call, (res, base_level) in enumerate(cases):
        shapes = [(res[0] + 1, res[1], res[2]), (res[0], res[1] + 1, res[2]), (res[0], res[1], res[2] + 1)]
        P = Projection(res, base_level=base_level)
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
        assert it.value == it_ref, (call, res)
        for a, b in zip(got, ref):
            assert _rel(a, b) < 1e-5, (call, res)
