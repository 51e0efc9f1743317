"""Cholesky factor in tile-LU form (bem_chol_factor) against numpy on the
same Hermitian positive definite matrices."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from bem_b200.engine import Engine
    e = Engine()
    yield e
    e.close()


def _hpd(n, cplx, seed):
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((2 * n, n))
    if cplx:
        G = G + 1j * rng.standard_normal((2 * n, n))
    N = G.conj().T @ G / n
    d = 1.0 / np.sqrt(np.real(np.diag(N)))
    return N * d[:, None] * d[None, :]


@pytest.mark.parametrize("tensor_cores", [False, True])
@pytest.mark.parametrize("cplx", [True, False])
@pytest.mark.parametrize("n", [37, 300, 777])
def test_chol_solve_matches_numpy(engine, n, cplx, tensor_cores):
    """The factor solves N x = b: to 1e-11 with FP64 updates; with the
    tensor-core updates (FP16-split products, FP64 Schur complement) within
    1e-5 (it preconditions the FP64 iteration of the least squares)."""
    N = _hpd(n, cplx, n)
    dt = torch.complex128 if cplx else torch.float64
    A = torch.as_tensor(N, dtype=dt, device="cuda")
    F = A.clone()
    piv, dinv, info = engine.chol_factor(F, tensor_cores=tensor_cores)
    assert int(info.item()) == 0
    rng = np.random.default_rng(1)
    b = rng.standard_normal(n) + (1j * rng.standard_normal(n) if cplx else 0)
    x = torch.as_tensor(b, dtype=dt, device="cuda").contiguous()
    engine.lu_solve_tiled(F, piv, dinv, x)
    ref = np.linalg.solve(N, b)
    err = np.linalg.norm(x.cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err < (1e-5 if tensor_cores else 1e-11), err


@pytest.mark.parametrize("nb", [256, 512, 1024])
def test_chol_panels_and_subpanels(engine, nb):
    """Several panels (BEM_TUNE_CHOL_NB) with partial sub-panels of 256
    columns and a partial last panel, FP64 updates: to 1e-11."""
    from bem_b200 import _lib as L
    n = 1333
    N = _hpd(n, True, 7)
    A = torch.as_tensor(N, device="cuda")
    F = A.clone()
    engine.set_tuning(L.TUNE_CHOL_NB, nb)
    try:
        piv, dinv, info = engine.chol_factor(F, tensor_cores=False)
    finally:
        engine.set_tuning(L.TUNE_CHOL_NB, 0)
    assert int(info.item()) == 0
    b = np.random.default_rng(2).standard_normal(n) + 0j
    x = torch.as_tensor(b, device="cuda").contiguous()
    engine.lu_solve_tiled(F, piv, dinv, x)
    ref = np.linalg.solve(N, b)
    assert np.linalg.norm(x.cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-11


def test_chol_reports_indefinite(engine):
    """A matrix with a negative pivot sets info to 1 + that column."""
    N = _hpd(130, True, 3)
    N[70, 70] = -1.0
    F = torch.as_tensor(N, device="cuda")
    _, _, info = engine.chol_factor(F, tensor_cores=False)
    assert int(info.item()) > 0
