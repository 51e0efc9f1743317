"""Least squares of the stacked transmission system [A; P+_i] x = rhs (the
reference's torch.linalg.lstsq, BEM_manager.py:1039-1050) on this library's
kernels, against numpy's QR-based lstsq on the same matrices and against the
oracle's assembly."""
import numpy as np
import pytest
import torch

from tests._util import rel_err

pytestmark = pytest.mark.gpu


def _system(subdiv, precision, Q=4, kernel="Helmholtz_Transmission"):
    from bem_b200 import icosphere
    from bem_b200.managers import CoreManager
    from bem_b200.workloads import PlaneWave, plane_wave_direction
    v, f = icosphere(subdiv)
    pw = PlaneWave(5.0, plane_wave_direction(0))
    params = dict(dim=3, vertices=v, panels=f, GaussQR=Q, kernel=kernel, boundary="Full", k=5.0, n_i=2.25,
                  n_o=1.0, scope="Exterior", Q_Neumann=0, Q_Dirichlet=1, precision=precision)
    core = CoreManager(params)
    core.initialization(pw.fD, pw.fN)
    return core, core._BEM_manager, v, f


@pytest.mark.parametrize("tensor_cores", [True, False])
@pytest.mark.parametrize("out_dtype", [torch.complex64, torch.complex128])
def test_gram_matrix(out_dtype, tensor_cores):
    """bem_gram: N = D (A^H A + P^H P) D with D the power-of-two column
    equilibration; FP16-split tensor-core products within 1e-6 (normwise),
    FP64 products to 1e-13 (to the output's precision for complex64)."""
    core, b, *_ = _system(2, "fp64")
    b.assemble_system()
    A, P = b._mat_A, b._mat_P
    n = A.shape[0]
    Nm = torch.empty(n, n, dtype=out_dtype, device="cuda")
    d = torch.empty(n, dtype=torch.float64, device="cuda")
    b.engine.gram(A, P, Nm, d, tensor_cores=tensor_cores)
    An, Pn = A.cpu().numpy(), P.cpu().numpy()
    cn = np.sqrt((np.abs(An) ** 2).sum(0) + (np.abs(Pn) ** 2).sum(0))
    dref = 2.0 ** (-np.rint(np.log2(cn)))
    assert np.array_equal(d.cpu().numpy(), dref)
    G = np.concatenate([An, Pn], 0) * dref
    Nref = G.conj().T @ G
    got = Nm.cpu().numpy().astype(np.complex128)
    err = np.linalg.norm(got - Nref) / np.linalg.norm(Nref)
    tol = 1e-6 if tensor_cores else (1e-7 if out_dtype == torch.complex64 else 1e-13)
    assert err < tol, err
    assert np.array_equal(got, got.conj().T)  # exactly Hermitian
    core.kill()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("subdiv", [2, 3])
def test_lstsq_matches_qr(subdiv, precision):
    """The driver's transmission solve equals numpy.linalg.lstsq (QR) of the
    same [A; P] and right-hand side to 1e-9, whichever precision assembled
    them (the solver itself is FP64-accurate on both paths)."""
    core, b, *_ = _system(subdiv, precision)
    b.run()
    A, P = b._mat_A.cpu().numpy(), b._mat_P.cpu().numpy()
    rhs = b.rhs.cpu().numpy()
    ref = np.linalg.lstsq(np.concatenate([A, P], 0), rhs, rcond=None)[0]
    assert rel_err(b.raw_solved.cpu().numpy(), ref) < 1e-9
    assert np.linalg.norm(b.raw_solved.cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-9
    core.kill()


def test_lstsq_against_oracle_assembly():
    """End to end on icosphere s2 (GaussQR 5): the mixed-precision solution
    (FP32 far field, FP16-split normal matrix, FP64 refinement) within 1e-6
    of numpy's lstsq of the oracle's FP64 [A; P+_i] system (the reference's
    solve, BEM_manager.py:1039-1050), and the plain FP64 solution within
    1e-10."""
    from oracle import oracle as O
    from bem_b200.workloads import plane_wave_direction
    dvec = plane_wave_direction(0)
    k = 5.0

    def fD(x, s=1.0):
        return np.exp(1j * k * s * (x @ dvec))

    def fN(x, n, s=1.0):
        return 1j * k * s * (n @ dvec) * np.exp(1j * k * s * (x @ dvec))
    res = {}
    for prec in ("mixed", "fp64"):
        core, b, v, f = _system(2, prec, Q=5)
        b.run()
        res[prec] = b.raw_solved.cpu().numpy()
        core.kill()
    params = dict(dim=3, kernel="Helmholtz_Transmission", boundary="Full", k=k, n_i=2.25, n_o=1.0, GaussQR=5,
                  scope="Exterior", Q_Neumann=0, Q_Dirichlet=1)
    ref = O.Problem(v, f, params, fD, fN, quirk=True).run()["raw_solved"]
    assert np.linalg.norm(res["fp64"] - ref) / np.linalg.norm(ref) < 1e-10
    assert rel_err(res["fp64"], ref) < 1e-10
    assert np.linalg.norm(res["mixed"] - ref) / np.linalg.norm(ref) < 1e-6
    assert rel_err(res["mixed"], ref) < 1e-6


def test_lstsq_real_system():
    """A real (Laplace "Full") stacked system through the same kernels, against
    numpy's lstsq."""
    core, b, *_ = _system(2, "mixed", Q=3, kernel="Laplace")
    b.run()
    A, P = b._mat_A.cpu().numpy(), b._mat_P.cpu().numpy()
    ref = np.linalg.lstsq(np.concatenate([A, P], 0), b.rhs.cpu().numpy(), rcond=None)[0]
    assert rel_err(b.raw_solved.cpu().numpy(), ref) < 1e-9
    core.kill()
