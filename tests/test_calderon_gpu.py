"""Fused Calderon-block assembly of the transmission operator
(bem_assemble_calderon) against the CPU oracle's per-operator assembly and
against this library's own per-operator path, on the same inputs."""
import numpy as np
import pytest

from tests._util import rel_err

pytestmark = pytest.mark.gpu


def _problem(subdiv, precision, Q=4, k=5.0, n_i=2.25, fuse=True, kernel="Helmholtz_Transmission"):
    from bem_b200 import icosphere
    from bem_b200.managers import CoreManager
    from bem_b200.workloads import PlaneWave, plane_wave_direction
    v, f = icosphere(subdiv)
    pw = PlaneWave(k, plane_wave_direction(0))
    params = dict(dim=3, vertices=v, panels=f, GaussQR=Q, kernel=kernel, boundary="Full", k=k, n_i=n_i, n_o=1.0,
                  scope="Exterior", Q_Neumann=0, Q_Dirichlet=1, precision=precision, fuse_calderon=fuse)
    core = CoreManager(params)
    core.initialization(pw.fD, pw.fN)
    return core, core._BEM_manager, v, f


def _oracle(v, f, Q, k=5.0, n_i=2.25, kernel="Helmholtz_Transmission"):
    """A = P-_o + P+_i and P = P+_i by the oracle's per-operator assembly."""
    from oracle import oracle as O
    params = dict(dim=3, kernel=kernel, boundary="Full", k=k, n_i=n_i, n_o=1.0, GaussQR=Q, scope="Exterior",
                  Q_Neumann=0, Q_Dirichlet=1)
    pb = O.Problem(v, f, params, None, None, quirk=True)
    A = np.zeros((pb.n, pb.n), pb.dtype)
    pb.add_identity(A, 0.5)
    pb.add_M(A, pb.forward(pb.sqrt_no), -1.0)
    P = np.zeros_like(A)
    pb.add_identity(P, 0.5)
    pb.add_M(P, pb.forward(pb.sqrt_ni), 1.0)
    return A + P, P


@pytest.mark.parametrize("subdiv", [1, 2])
def test_fused_fp64_matches_oracle(subdiv):
    """A and P in FP64 equal the oracle's per-operator assembly
    (BEM_manager.py:995-1006, 1039-1045) to 1e-12."""
    Q = 4
    core, b, v, f = _problem(subdiv, "fp64", Q=Q)
    b.assemble_system()
    A_ref, P_ref = _oracle(v, f, Q)
    assert rel_err(b._mat_P.cpu().numpy(), P_ref) < 1e-12
    assert rel_err(b._mat_A.cpu().numpy(), A_ref) < 1e-12
    core.kill()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_matches_per_operator_path(precision):
    """The fused sweep and the per-operator kernels (matrix_layer_forward +
    assemble_matA) give the same A, P and right-hand side: to 1e-12 in FP64;
    in mixed precision each within 2e-6 of the FP64 blocks."""
    from bem_b200.utils.types import AssembleType
    core, b, *_ = _problem(3, precision)
    b.assemble_system()
    A_f, P_f, rhs_f = b._mat_A.clone(), b._mat_P.clone(), b.rhs.clone()
    core.kill()
    core, b, *_ = _problem(3, precision, fuse=False)
    b.assemble_system()
    A_u, rhs_u = b._mat_A.clone(), b.rhs.clone()
    b._mat_A.zero_()
    b.assemble_matA(assemble_type=int(AssembleType.ADD_P_PLUS), multiplier=1.0)
    P_u = b._mat_A.clone()
    core.kill()
    tol = 1e-12 if precision == "fp64" else 2e-6
    for x, y in ((A_f, A_u), (P_f, P_u), (rhs_f, rhs_u)):
        assert rel_err(x.cpu().numpy(), y.cpu().numpy()) < tol
    if precision == "mixed":
        core, b, *_ = _problem(3, "fp64")
        b.assemble_system()
        assert rel_err(A_f.cpu().numpy(), b._mat_A.cpu().numpy()) < 2e-6
        assert rel_err(P_f.cpu().numpy(), b._mat_P.cpu().numpy()) < 2e-6
        core.kill()


def test_laplace_full_and_grouped_wavenumbers():
    """Laplace "Full" problems take the same path (k = 0), and the forms of the
    sweep agree: one launch with both wavenumbers (tuning group 2), one per
    wavenumber (1), and the packed FP32x2 sweeps (3: over test points, one
    wavenumber per launch; 4: the two wavenumbers in the two lanes; mixed
    precision)."""
    from bem_b200 import _lib as L
    core, b, v, f = _problem(2, "fp64", Q=3, kernel="Laplace")
    b.assemble_system()
    A_ref, _ = _oracle(v, f, 3, k=0.0, kernel="Laplace")
    assert rel_err(b._mat_A.cpu().numpy(), A_ref) < 1e-12
    core.kill()
    for prec in ("fp64", "mixed"):
        outs = []
        for group in ((1, 2) if prec == "fp64" else (1, 2, 3, 4, 5)):
            core, b, *_ = _problem(2, prec)
            b.engine.set_tuning(L.TUNE_CALDERON_GROUP, group)
            b.assemble_system()
            outs.append((b._mat_A.clone(), b._mat_P.clone()))
            core.kill()
        tol = 1e-13 if prec == "fp64" else 1e-6
        for o in outs[1:]:
            assert rel_err(outs[0][0].cpu().numpy(), o[0].cpu().numpy()) < tol
            assert rel_err(outs[0][1].cpu().numpy(), o[1].cpu().numpy()) < tol
