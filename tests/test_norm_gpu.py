"""The FP64 building blocks of the operator-norm analysis (the reference's
compute_inv_norm, BEM_manager.py:874-920) on this library's kernels:
bem_gemm (DMMA products, split K for thin ones) and bem_chol_inverse
(Cholesky plus triangular inverse), against numpy in FP64."""
import numpy as np
import pytest
import torch

from tests._util import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from bem_b200.engine import Engine
    e = Engine()
    yield e
    e.close()


def _rand(rng, shape, cplx):
    a = rng.standard_normal(shape)
    if cplx:
        a = a + 1j * rng.standard_normal(shape)
    return a


@pytest.mark.parametrize("cplx", [True, False])
@pytest.mark.parametrize("conj_a,conj_b", [(False, False), (True, False), (False, True), (True, True)])
@pytest.mark.parametrize("m,n,k", [(300, 200, 129), (200, 8, 5000), (70, 70, 70)])
def test_gemm_matches_numpy(engine, cplx, conj_a, conj_b, m, n, k):
    rng = np.random.default_rng(m + n + k)
    A = _rand(rng, (k, m) if conj_a else (m, k), cplx)
    B = _rand(rng, (n, k) if conj_b else (k, n), cplx)
    C0 = _rand(rng, (m, n), cplx)
    opa = A.conj().T if conj_a else A
    opb = B.conj().T if conj_b else B
    ref = C0 - 0.5 * (opa @ opb)
    C = torch.as_tensor(C0, device="cuda").contiguous()
    engine.gemm(torch.as_tensor(A, device="cuda"), torch.as_tensor(B, device="cuda"), C, alpha=-0.5, conj_a=conj_a,
                conj_b=conj_b)
    assert rel_err(C.cpu().numpy(), ref) < 1e-13


@pytest.mark.parametrize("conj_b", [False, True])
@pytest.mark.parametrize("m,n,k", [(200, 150, 300), (300, 8, 300), (77, 77, 77)])
def test_gemm_triangular_operands(engine, conj_b, m, n, k):
    """tri flags: op(A) lower and op(B) upper triangular.  Zeros on the
    other side of the diagonal within the 64-wide diagonal tiles, and
    garbage (1e300) beyond them, where the product must not read."""
    rng = np.random.default_rng(m * n + k)
    i, c = np.indices((m, k))
    A = np.where(c <= i, _rand(rng, (m, k), True), 0.0)
    Ag = np.where(c >= (i // 64 + 1) * 64, 1e300, A)
    r, j = np.indices((k, n))
    Bop = np.where(r <= j, _rand(rng, (k, n), True), 0.0)
    Bg = np.where(r >= (j // 64 + 1) * 64, 1e300, Bop)
    ref = A @ Bop
    B = Bg.conj().T.copy() if conj_b else Bg
    C = torch.zeros(m, n, dtype=torch.complex128, device="cuda")
    engine.gemm(torch.as_tensor(Ag, device="cuda"), torch.as_tensor(B, device="cuda"), C, conj_b=conj_b,
                a_lower=True, b_upper=True)
    assert rel_err(C.cpu().numpy(), ref) < 1e-13


@pytest.mark.parametrize("cplx", [True, False])
@pytest.mark.parametrize("n", [37, 300, 777])
def test_chol_inverse(engine, cplx, n):
    rng = np.random.default_rng(n)
    B = _rand(rng, (n, n), cplx)
    M = B @ B.conj().T + n * np.eye(n)
    A = torch.as_tensor(M, device="cuda").contiguous()
    X, info = engine.chol_inverse(A)
    assert int(info.item()) == 0
    Xh = X.cpu().numpy()
    Lref = np.linalg.cholesky(M)
    assert np.all(np.triu(Xh, 1) == 0)
    assert rel_err(Xh, np.linalg.inv(Lref)) < 1e-12
    assert rel_err(np.tril(A.cpu().numpy()), Lref) < 1e-12


def test_chol_inverse_reports_indefinite(engine):
    M = np.eye(200)
    M[150, 150] = -1.0
    X, info = engine.chol_inverse(torch.as_tensor(M, device="cuda").contiguous())
    assert int(info.item()) == 151
