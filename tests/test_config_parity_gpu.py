"""Parity at the benchmark configurations' own sizes, against the FP64 C
oracle (the restatement of the reference's loops, pinned to the reference's
outputs by the golden fixtures).

- Laplace interior Dirichlet on the icosphere of subdivision 3 (1280 panels,
  642 vertices), GaussQR 5, u = 1/|x - x0|: the full V block and K g of the
  fused sweep entrywise, and the whole driver (A, right-hand side, solution)
  against the oracle's driver.
- Helmholtz interior Dirichlet, k = 3, subdivision 4 (5120 panels), GaussQR
  5, plane wave: 64 seeded rows of V and of K g, FP64 and mixed precision,
  and the mixed driver's solution against the FP64 driver's.

Tolerances: FP64 1e-12 of the block's largest entry (summation order only);
mixed 2e-6 for entries (FP32 separate pairs); 1e-6 for solutions.
"""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests._util import data_callbacks, full_spaces, rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 2e-6
SOLUTION_TOL = 1e-6


@pytest.fixture(scope="module")
def engine():
    from bem_b200.engine import Engine
    O.set_threads(os.cpu_count() or 1)
    e = Engine()
    yield e
    e.close()


def _spaces(engine, v, f):
    from bem_b200.engine import DeviceSpace
    p0 = full_spaces(len(v), f, 1)
    p1 = full_spaces(len(v), f, 3)
    return p0, p1, DeviceSpace.from_numpy(*p0, engine.device), DeviceSpace.from_numpy(*p1, engine.device)


def _fused(engine, v, f, Q, helm, k, g, precision):
    """V and K g of one fused symmetric sweep (the call the driver makes for
    a Dirichlet problem), with the reference's conj(g) for Helmholtz."""
    from bem_b200 import _lib as L
    engine.set_mesh(v, f, Q)
    p0, p1, s0, s1 = _spaces(engine, v, f)
    dt = torch.complex128 if helm else torch.float64
    V = torch.zeros(len(f), len(f), dtype=dt, device="cuda")
    y = torch.zeros(len(f), dtype=dt, device="cuda")
    desc = engine.op_desc(O.OP_V, helm, k, k * k, precision=L.PREC_MIXED if precision == "mixed" else L.PREC_FP64)
    engine.assemble_dirichlet(desc, s0, s0, V, s0, s1, torch.as_tensor(g, device="cuda"), y, scale=1.0,
                              scale_k=1.0, conj_g=helm)
    return V, y, p0, p1


def test_laplace_s3_full_V_and_Kg(engine):
    from bem_b200 import icosphere
    v, f = icosphere(3)
    assert (len(v), len(f)) == (642, 1280)
    fD, _ = data_callbacks("laplace_point")
    g = fD(np.asarray(v, np.float64))
    V, y, p0, p1 = _fused(engine, v, f, 5, False, 0.0, g, "fp64")
    Vref = np.zeros((len(f), len(f)))
    O.assemble(v, f, O.OP_V, False, 0.0, 0.0, 5, True, p0, p0, out=Vref)
    yref = np.zeros(len(f))
    O.assemble(v, f, O.OP_K, False, 0.0, 0.0, 5, True, p0, p1, x=g, y=yref)
    assert rel_err(V.cpu().numpy(), Vref) < FP64_TOL
    assert rel_err(y.cpu().numpy(), yref) < FP64_TOL


def test_laplace_s3_driver_against_oracle_driver():
    """The whole plain FP64 driver (CoreManager) on the 1280-panel problem
    against the oracle's driver: A, right-hand side and the Neumann trace;
    the trace also against the analytic du/dn, in both quadrature modes."""
    from bem_b200 import icosphere
    from bem_b200.managers import CoreManager
    from bem_b200.workloads import laplace_dirichlet_s3
    params, fD, fN = laplace_dirichlet_s3("fp64")
    core = CoreManager(params)
    core.initialization(fD, fN)
    b = core._BEM_manager
    b.run()
    v, f = icosphere(3)
    r = O.Problem(v, f, params, *data_callbacks("laplace_point")).run()
    assert rel_err(b._mat_A.cpu().numpy(), r["A"]) < FP64_TOL
    assert rel_err(b.rhs.cpu().numpy(), r["rhs"]) < FP64_TOL
    got = b.raw_solved.cpu().numpy()
    assert rel_err(got, r["raw_solved"]) < 1e-10
    ana = b.raw_analytical_solved.cpu().numpy()
    core.kill()
    # the Neumann trace against the analytic du/dn: with the reference's
    # near-pair quadrature (the default) the error is the reference's own,
    # about 0.4 and not shrinking with the mesh; the corrected quadrature
    # (quirk = 0) converges (5.2e-3 on these 1280 panels)
    assert 0.2 < np.linalg.norm(got - ana) / np.linalg.norm(ana) < 0.5
    params["quirk"] = 0
    core = CoreManager(params)
    core.initialization(fD, fN)
    core._BEM_manager.run()
    got0 = core._BEM_manager.raw_solved.cpu().numpy()
    ana0 = core._BEM_manager.raw_analytical_solved.cpu().numpy()
    core.kill()
    assert np.linalg.norm(got0 - ana0) / np.linalg.norm(ana0) < 1e-2


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_helmholtz_s4_sampled_rows(engine, precision):
    from bem_b200 import icosphere
    from bem_b200.workloads import plane_wave_direction
    v, f = icosphere(4)
    assert (len(v), len(f)) == (2562, 5120)
    k = 3.0
    fD, _ = data_callbacks("plane_wave", k, plane_wave_direction(0))
    g = fD(np.asarray(v, np.float64))
    V, y, p0, p1 = _fused(engine, v, f, 5, True, k, g, precision)
    rows = np.sort(np.random.default_rng(2024).choice(len(f), 64, replace=False)).astype(np.int32)
    sub = (rows, 1, np.arange(64, dtype=np.int32))
    Vref = np.zeros((64, len(f)), np.complex128)
    O.assemble(v, f, O.OP_V, True, k, k * k, 5, True, sub, p0, out=Vref)
    yref = np.zeros(64, np.complex128)
    O.assemble(v, f, O.OP_K, True, k, k * k, 5, True, sub, p1, x=g, y=yref, conj_x=True)
    tol = FP64_TOL if precision == "fp64" else MIXED_TOL
    idx = torch.as_tensor(rows.astype(np.int64), device="cuda")
    assert rel_err(V.index_select(0, idx).cpu().numpy(), Vref) < tol
    assert rel_err(y.index_select(0, idx).cpu().numpy(), yref) < tol


def test_helmholtz_s4_mixed_driver_solution():
    """The mixed driver (FP32 far field, FP32 tile LU, FP64 refinement) on the
    5120-panel problem against the FP64 driver, whose blocks the sampled-row
    test pins to the oracle."""
    from bem_b200.managers import CoreManager
    from bem_b200.workloads import helmholtz_dirichlet_s4
    sols = {}
    for precision in ("fp64", "mixed"):
        params, fD, fN = helmholtz_dirichlet_s4(precision)
        core = CoreManager(params)
        core.initialization(fD, fN)
        core._BEM_manager.run()
        sols[precision] = core._BEM_manager.raw_solved.cpu().numpy()
        core.kill()
    assert rel_err(sols["mixed"], sols["fp64"]) < SOLUTION_TOL
