"""The k-derivative of the Helmholtz operators (bem_assemble with deriv_k)
and dJ/dk of the transmission problem through the adjoint
(managers/kderiv.py).

- Operator blocks: the derivative kernels (FP64) against the central
  difference in k (fixed k2) of the oracle's FP64 blocks, h = 1e-4
  (truncation ~h^2, cancellation ~1e-16/h): tolerance 1e-7 of the largest
  entry.
- dJ/dk of J = ||x||^2 on the icosphere of subdivision 2 (320 panels) for
  the square system and for the reference's least squares, FP64, against the
  fourth-order central difference of J (delta = 5e-3): tolerance 1e-6.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests._util import full_spaces, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from bem_b200.engine import Engine
    e = Engine()
    yield e
    e.close()


@pytest.mark.parametrize("op,nbx,nby", [(O.OP_V, 1, 1), (O.OP_K, 1, 3), (O.OP_KP, 3, 1), (O.OP_W, 3, 3),
                                        (O.OP_V, 3, 3)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_operator_k_derivative(engine, op, nbx, nby, precision):
    from bem_b200 import _lib as L
    from bem_b200 import icosphere
    from bem_b200.engine import DeviceSpace
    v, f = icosphere(2)
    Q, k, k2, h = 4, 2.5, 6.25, 1e-4
    engine.set_mesh(v, f, Q)
    ts, rs = full_spaces(len(v), f, nbx), full_spaces(len(v), f, nby)
    nrow = len(f) if nbx == 1 else len(v)
    ncol = len(f) if nby == 1 else len(v)
    ref = np.zeros((nrow, ncol), np.complex128)
    tmp = np.zeros_like(ref)
    O.assemble(v, f, op, True, k + h, k2, Q, True, ts, rs, out=ref)
    O.assemble(v, f, op, True, k - h, k2, Q, True, ts, rs, out=tmp)
    ref = (ref - tmp) / (2 * h)
    out = torch.zeros(nrow, ncol, dtype=torch.complex128, device="cuda")
    prec = L.PREC_MIXED if precision == "mixed" else L.PREC_FP64
    engine.assemble(engine.op_desc(op, True, k, k2, precision=prec, deriv_k=True),
                    DeviceSpace.from_numpy(*ts, engine.device), DeviceSpace.from_numpy(*rs, engine.device), out)
    assert rel_err(out.cpu().numpy(), ref) < (1e-7 if precision == "fp64" else 2e-6)


def test_deriv_k_rejected_where_unsupported(engine):
    from bem_b200 import icosphere
    from bem_b200._lib import BemError
    from bem_b200.engine import DeviceSpace
    v, f = icosphere(1)
    engine.set_mesh(v, f, 3)
    sp = DeviceSpace.from_numpy(*full_spaces(len(v), f, 1), engine.device)
    out = torch.zeros(len(f), len(f), dtype=torch.float64, device="cuda")
    with pytest.raises(BemError):
        engine.assemble(engine.op_desc(O.OP_V, False, 0.0, 0.0, deriv_k=True), sp, sp, out)


@pytest.mark.parametrize("solver", ["square", "lstsq"])
def test_dJdk_matches_central_difference(solver):
    from bem_b200.managers import CoreManager
    from bem_b200.managers.kderiv import solution_norm_k_gradient
    from bem_b200.workloads import transmission_s5
    params, pw = transmission_s5("fp64", 2, solver)
    if solver == "square":
        params.update(solve_precision="mixed", refine_tol=1e-13)
    core = CoreManager(params)
    core.initialization(pw.fD, pw.fN)
    g = solution_norm_k_gradient(core._BEM_manager, pw, check=True, delta=1e-3)
    core.kill()
    cd = g["dJdk_central_difference"]
    assert abs(g["dJdk"] - cd) <= 1e-6 * abs(cd), (g["dJdk"], cd)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_media_derivative_equals_per_medium(precision):
    """dM/dk of both media assembled together (k_derivative_M_media:
    bem_assemble_batch with the derivative kernels, dW/dk2 as two batched W
    terms) equals the per-medium assembly (k_derivative_M): 1e-12 in FP64,
    2e-6 of the largest entry in mixed precision."""
    from bem_b200.managers import CoreManager
    from bem_b200.managers.kderiv import k_derivative_M, k_derivative_M_media
    from bem_b200.utils.types import ScopeType
    from bem_b200.workloads import transmission_s5
    params, pw = transmission_s5(precision, 2, "lstsq")
    core = CoreManager(params)
    core.initialization(pw.fD, pw.fN)
    bm = core._BEM_manager
    n = bm.N_Neumann + bm.M_Dirichlet
    k = float(bm._k)
    ref_o = torch.zeros(n, n, dtype=torch.complex128, device="cuda")
    ref_i = torch.zeros_like(ref_o)
    k_derivative_M(bm, k, bm._sqrt_no, int(ScopeType.EXTERIOR), ref_o, -1.0)
    k_derivative_M(bm, k, bm._sqrt_ni, int(ScopeType.INTERIOR), ref_i, 1.0)
    got_o = torch.zeros_like(ref_o)
    got_i = torch.zeros_like(ref_o)
    k_derivative_M_media(bm, k, [(bm._sqrt_no, got_o, -1.0), (bm._sqrt_ni, got_i, 1.0)])
    core.kill()
    tol = 1e-12 if precision == "fp64" else 2e-6
    assert rel_err(got_o.cpu().numpy(), ref_o.cpu().numpy()) < tol
    assert rel_err(got_i.cpu().numpy(), ref_i.cpu().numpy()) < tol
