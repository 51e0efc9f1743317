"""The allocation-free triangular solve (bem_lu_solve_tiled_static).

Some callers cannot allocate device memory once they run -- their device
memory belongs to another allocator, or cudaMalloc's implicit device
synchronisation is not acceptable in their loop -- so they cannot create the
workspace that bem_lu_solve_tiled keeps in its context.  The static variant
takes no context and keeps its scratch in a device array compiled into the
library.  These checks call it directly through the C ABI and compare it with
the context-based solve on the same factors, on two calls in a row (the
shared array keeps the previous call's contents, which must not leak into the
next result).  This file is collected last, and also runs alone in a fresh
process.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-11  # same as the context-based tiled solve tests


def _factors(engine, n, cplx, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    A = A + 3 * n ** 0.5 * np.eye(n)
    LU = torch.as_tensor(A, device="cuda").contiguous()
    piv, dinv, info = engine.lu_factor_tiled(LU)
    assert int(info.item()) == 0
    return A, LU, piv, dinv


def _static_solve(lib, LU, piv, dinv, b):
    from bem_b200._lib import C128, F64
    from bem_b200.engine import _dtype_code
    n = LU.shape[0]
    rc = lib.bem_lu_solve_tiled_static(_dtype_code(LU), ctypes.c_void_p(LU.data_ptr()), n, LU.stride(0),
                                       ctypes.c_void_p(piv.data_ptr()), ctypes.c_void_p(dinv.data_ptr()),
                                       ctypes.c_void_p(b.data_ptr()),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, rc
    return b


@pytest.mark.parametrize("cplx", [False, True])
def test_static_solve_matches_context_solve_twice(cplx):
    from bem_b200.engine import Engine
    eng = Engine()
    lib = eng.lib
    n = 700
    A, LU, piv, dinv = _factors(eng, n, cplx, 17)
    rng = np.random.default_rng(5)
    for call in range(2):
        b = rng.standard_normal(n) + (1j * rng.standard_normal(n) if cplx else 0)
        ref = torch.as_tensor(b, device="cuda").contiguous()
        eng.lu_solve_tiled(LU, piv, dinv, ref)
        got = _static_solve(lib, LU, piv, dinv, torch.as_tensor(b, device="cuda").contiguous())
        torch.cuda.synchronize()
        r, g = ref.cpu().numpy(), got.cpu().numpy()
        assert np.abs(g - r).max() / np.abs(r).max() < TOL, call
        assert np.abs(g - np.linalg.solve(A, b)).max() / np.abs(r).max() < TOL, call
    eng.close()


def test_static_solve_rejects_sizes_beyond_its_array():
    from bem_b200 import _lib
    lib = _lib.load()
    t = torch.zeros(4, dtype=torch.float64, device="cuda")
    p = torch.zeros(4, dtype=torch.int32, device="cuda")
    n = _lib.STATIC_SOLVE_MAX_N + 1
    rc = lib.bem_lu_solve_tiled_static(_lib.F64, ctypes.c_void_p(t.data_ptr()), n, n, ctypes.c_void_p(p.data_ptr()),
                                       ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(t.data_ptr()), None)
    assert rc == -1  # BEM_ERR_INVALID, nothing launched
