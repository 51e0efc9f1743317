"""Dense LU / triangular solves / refinement (libbem_b200) against numpy
(LAPACK) on the same inputs."""
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


def _mat(n, cplx, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n))
    if cplx:
        A = A + 1j * rng.standard_normal((n, n))
    return A + n ** 0.5 * np.eye(n) * 0.5


@pytest.mark.parametrize("n", [1, 37, 64, 200, 321])
@pytest.mark.parametrize("cplx", [False, True])
def test_lu_fp64_solve(engine, n, cplx):
    A = _mat(n, cplx, n)
    rng = np.random.default_rng(7)
    b = rng.standard_normal((n, 2)) + (1j * rng.standard_normal((n, 2)) if cplx else 0)
    x_ref = np.linalg.solve(A, b)
    Ad = torch.as_tensor(A, device="cuda").contiguous()
    piv, info = engine.lu_factor(Ad)
    assert int(info.item()) == 0
    bd = torch.as_tensor(b, device="cuda").contiguous()
    engine.lu_solve(Ad, piv, bd)
    assert rel_err(bd.cpu().numpy(), x_ref) < 1e-11


@pytest.mark.parametrize("cplx", [False, True])
def test_lu_matches_lapack_factors(engine, cplx):
    import scipy.linalg
    n = 150
    A = _mat(n, cplx, 3)
    Ad = torch.as_tensor(A, device="cuda").contiguous()
    piv, info = engine.lu_factor(Ad)
    lu, piv_ref = scipy.linalg.lu_factor(A)
    assert (piv.cpu().numpy() == piv_ref).all()
    assert rel_err(Ad.cpu().numpy(), lu) < 1e-12


def test_lu_singular_reports_info(engine):
    A = np.ones((10, 10))
    Ad = torch.as_tensor(A, device="cuda").contiguous()
    piv, info = engine.lu_factor(Ad)
    assert int(info.item()) > 0


@pytest.mark.parametrize("cplx", [False, True])
def test_fp32_factor_with_fp64_refinement(engine, cplx):
    n = 300
    A = _mat(n, cplx, 11)
    rng = np.random.default_rng(5)
    b = rng.standard_normal(n) + (1j * rng.standard_normal(n) if cplx else 0)
    x_ref = np.linalg.solve(A, b)
    A_hi = torch.as_tensor(A, device="cuda").contiguous()
    LU = A_hi.to(torch.complex64 if cplx else torch.float32).contiguous()
    piv, info = engine.lu_factor(LU)
    assert int(info.item()) == 0
    bd = torch.as_tensor(b, device="cuda").contiguous()
    xd = torch.zeros_like(bd)
    it, rr = engine.refine_solve(A_hi, LU, piv, bd, xd, tol=1e-13, maxit=30)
    assert rr <= 1e-13 and it >= 1
    assert rel_err(xd.cpu().numpy(), x_ref) < 1e-11


def test_gemv(engine):
    rng = np.random.default_rng(2)
    A = rng.standard_normal((70, 50)) + 1j * rng.standard_normal((70, 50))
    x = rng.standard_normal(50) + 1j * rng.standard_normal(50)
    y0 = rng.standard_normal(70) + 1j * rng.standard_normal(70)
    Ad = torch.as_tensor(A, device="cuda")
    yd = torch.as_tensor(y0.copy(), device="cuda")
    engine.gemv(Ad, torch.as_tensor(x, device="cuda"), yd, alpha=-2.0, beta=0.5)
    assert rel_err(yd.cpu().numpy(), 0.5 * y0 - 2.0 * A @ x) < 1e-13


@pytest.mark.parametrize("n", [5, 64, 200, 333])
@pytest.mark.parametrize("cplx", [False, True])
def test_tiled_factor_and_dataflow_solve(engine, n, cplx):
    """Tile-pivoted FP64 factor + barrier-free solve reproduce numpy's solve on
    a diagonally dominant matrix (tile pivoting needs no cross-tile swaps)."""
    A = _mat(n, cplx, 2 * n) + 3 * n ** 0.5 * np.eye(n)
    rng = np.random.default_rng(9)
    b = rng.standard_normal(n) + (1j * rng.standard_normal(n) if cplx else 0)
    LU = torch.as_tensor(A, device="cuda").contiguous()
    piv, dinv, info = engine.lu_factor_tiled(LU)
    assert int(info.item()) == 0
    x = torch.as_tensor(b, device="cuda").contiguous()
    engine.lu_solve_tiled(LU, piv, dinv, x)
    assert rel_err(x.cpu().numpy(), np.linalg.solve(A, b)) < 1e-11


@pytest.mark.parametrize("cplx", [False, True])
def test_tiled_fp32_factor_with_refinement(engine, cplx):
    n = 500
    A = _mat(n, cplx, 21) + 2 * n ** 0.5 * np.eye(n)
    rng = np.random.default_rng(4)
    b = rng.standard_normal(n) + (1j * rng.standard_normal(n) if cplx else 0)
    A_hi = torch.as_tensor(A, device="cuda").contiguous()
    LU = A_hi.to(torch.complex64 if cplx else torch.float32).contiguous()
    piv, dinv, info = engine.lu_factor_tiled(LU)
    bd = torch.as_tensor(b, device="cuda").contiguous()
    xd = torch.zeros_like(bd)
    it, rr = engine.refine_solve(A_hi, LU, piv, bd, xd, tol=1e-13, maxit=30, dinv=dinv)
    assert rr <= 1e-13
    assert rel_err(xd.cpu().numpy(), np.linalg.solve(A, b)) < 1e-11


@pytest.mark.parametrize("cplx", [False, True])
def test_async_refinement_stopping_rules(engine, cplx):
    """The device-side stopping test of the tiled refinement: b = 0 returns
    x = 0 after no iteration; an iteration cap below the needed count reports
    BEM_ERR_NOCONVERGE with the residual reached; a later call on the same
    factor converges (the state of a call does not leak into the next); and
    the iteration count matches the synchronous loop's rule (stop at the
    first residual below tol)."""
    from bem_b200._lib import BemError
    n = 300
    A = _mat(n, cplx, 5) + 2 * n ** 0.5 * np.eye(n)
    A_hi = torch.as_tensor(A, device="cuda").contiguous()
    LU = A_hi.to(torch.complex64 if cplx else torch.float32).contiguous()
    piv, dinv, _ = engine.lu_factor_tiled(LU)
    zero = torch.zeros(n, dtype=A_hi.dtype, device="cuda")
    x = torch.full_like(zero, 7.0)
    it, rr = engine.refine_solve(A_hi, LU, piv, zero, x, tol=1e-12, maxit=10, dinv=dinv)
    assert it == 0 and rr == 0.0 and float(x.abs().max()) == 0.0
    rng = np.random.default_rng(8)
    b = rng.standard_normal(n) + (1j * rng.standard_normal(n) if cplx else 0)
    bd = torch.as_tensor(b, device="cuda").contiguous()
    with pytest.raises(BemError) as exc:
        engine.refine_solve(A_hi, LU, piv, bd, torch.zeros_like(bd), tol=1e-14, maxit=1, dinv=dinv)
    assert exc.value.code == -4
    xd = torch.zeros_like(bd)
    it, rr = engine.refine_solve(A_hi, LU, piv, bd, xd, tol=1e-12, maxit=20, dinv=dinv)
    assert rr <= 1e-12 and 1 <= it <= 6
    # the same stopping point as solving to a looser tolerance and counting
    xl = torch.zeros_like(bd)
    it_loose, rr_loose = engine.refine_solve(A_hi, LU, piv, bd, xl, tol=1e-6, maxit=20, dinv=dinv)
    assert it_loose <= it and rr_loose <= 1e-6
    assert rel_err(xd.cpu().numpy(), np.linalg.solve(A, b)) < 1e-10


def _illcond(n, cplx, cond, seed):
    """Q diag(s) Q^H with singular values log-spaced from 1 to 1/cond."""
    rng = np.random.default_rng(seed)
    Z = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    Q, _ = np.linalg.qr(Z)
    s = np.logspace(0, -np.log10(cond), n)
    return (Q * s) @ Q.conj().T


@pytest.mark.parametrize("tiled", [False, True])
@pytest.mark.parametrize("cplx", [False, True])
def test_gmres_ir(engine, cplx, tiled):
    """bem_gmres_ir on a system with cond(A) = 1e6, where the FP32 factor's
    refinement contracts slowly (cond * u_fp32 ~ 0.06): the solution against
    numpy's FP64 solve, b = 0, and the iteration cap."""
    from bem_b200._lib import BemError
    n = 256
    A = _illcond(n, cplx, 1e6, 31)
    rng = np.random.default_rng(6)
    b = rng.standard_normal(n) + (1j * rng.standard_normal(n) if cplx else 0)
    A_hi = torch.as_tensor(A, device="cuda").contiguous()
    LU = A_hi.to(torch.complex64 if cplx else torch.float32).contiguous()
    if tiled:
        piv, dinv, _ = engine.lu_factor_tiled(LU)
    else:
        piv, _ = engine.lu_factor(LU)
        dinv = None
    bd = torch.as_tensor(b, device="cuda").contiguous()
    xd = torch.zeros_like(bd)
    # the FP64 residual of this system bottoms out near eps * cond(A) = 1e-10
    it, rr = engine.gmres_solve(A_hi, LU, piv, bd, xd, tol=1e-10, maxit=200, restart=30, dinv=dinv)
    assert rr <= 1e-10 and it >= 1
    assert rel_err(xd.cpu().numpy(), np.linalg.solve(A, b)) < 1e-7
    zero = torch.zeros_like(bd)
    x0 = torch.zeros_like(bd)
    it0, rr0 = engine.gmres_solve(A_hi, LU, piv, zero, x0, tol=1e-12, maxit=10, restart=5, dinv=dinv)
    assert it0 == 0 and rr0 == 0.0 and float(x0.abs().max()) == 0.0
    with pytest.raises(BemError) as exc:
        engine.gmres_solve(A_hi, LU, piv, bd, torch.zeros_like(bd), tol=1e-15, maxit=1, restart=1, dinv=dinv,
                           accept=0.0)
    assert exc.value.code == -4


def test_device_code_is_sm100a():
    """The device code the runtime loaded is the sm_100a build (binaryVersion 100)."""
    import ctypes
    from bem_b200 import _lib
    L = _lib.load()
    torch.zeros(1, device="cuda")
    v = ctypes.c_int(0)
    assert L.bem_binary_version(ctypes.byref(v)) == 0
    assert v.value == 100


def test_factor_status_after_tiled_factor(engine):
    """bem_lu_factor_status reads (and clears) the tiled factorisation's
    tensor-core wait status: BEM_OK for a factor that completed."""
    from bem_b200 import _lib
    n = 256
    A = torch.as_tensor(_mat(n, True, 5), dtype=torch.complex64, device="cuda")
    engine.lu_factor_tiled(A)
    L = _lib.load()
    assert L.bem_lu_factor_status(engine.ctx, ctypes_stream()) == 0


def ctypes_stream():
    return torch.cuda.current_stream().cuda_stream
