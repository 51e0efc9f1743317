"""BEMManager methods outside run(): block readers and writers
(BEM_manager.py:846-872), the plain getters (:205-221) and Jacobian_solver
(:803-821), on the golden cases' managers."""
import numpy as np
import pytest
import torch

from tests._util import load_fixture, torch_callbacks

pytestmark = pytest.mark.gpu


def _manager(name):
    from bem_b200.managers import CoreManager
    d = load_fixture(name)
    params = eval(str(d["params"]))
    params.update(vertices=d["vertices"], panels=d["panels"])
    fD, fN = torch_callbacks(str(d["data_kind"]), float(params.get("k", 0.0)), d["direction"])
    core = CoreManager(params)
    core.initialization(fD, fN)
    return core, core._BEM_manager


def test_block_parts_tile_the_matrix():
    core, b = _manager("cube_helm_mix_ext_q4")  # both Neumann and Dirichlet unknowns
    mm = core._mesh_manager
    assert b.get_num_of_panels_Neumann() == mm.get_num_of_panels_Neumann()
    assert b.get_num_of_panels_Dirichlet() == mm.get_num_of_panels_Dirichlet()
    assert b.get_shape_func_degree_Neumann() == mm.get_shape_func_degree_Neumann()
    assert b.get_shape_func_degree_Dirichlet() == mm.get_shape_func_degree_Dirichlet()
    N, M = b.N_Neumann, b.M_Dirichlet
    assert N > 0 and M > 0
    T = torch.zeros_like(b._mat_A)
    blocks = {"V": (N, N, 1.0), "K": (N, M, 2.0), "adj_K": (M, N, 3.0), "W": (M, M, 4.0)}
    for part, (r, c, v) in blocks.items():
        getattr(b, f"set_{part}_part")(T, torch.full((r, c), v, dtype=T.dtype, device=T.device))
    for part, (r, c, v) in blocks.items():
        got = getattr(b, f"get_{part}_part")(T)
        assert got.shape == (r, c) and bool((got == v).all())
    assert bool((T != 0).all())  # the four blocks cover the matrix exactly once
    core.kill()


@pytest.mark.parametrize("name", ["cube_lap_dir_q5", "ico1_helm_dir_p1_q3"])
def test_jacobian_solver_sweeps(name):
    core, b = _manager(name)
    n = b.N_Neumann + b.M_Dirichlet
    rng = np.random.default_rng(3)
    cplx = b._mat_A.is_complex()
    A = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    A += np.diag(2.0 * np.abs(A).sum(1))  # |a_ii| > 2 sum_j |a_ij|: Jacobi contracts by 1/2 or better
    rhs = rng.standard_normal(n) + (1j * rng.standard_normal(n) if cplx else 0)
    b._mat_A.copy_(torch.as_tensor(A))
    b.rhs[:n].copy_(torch.as_tensor(rhs))
    b.raw_solved.zero_()
    u = np.zeros(n, A.dtype)
    res = []
    for _ in range(4):
        res.append(b.Jacobian_solver())
        u = u + (rhs - A @ u) / np.diag(A)
        want = np.sqrt((np.abs(rhs - A @ u) ** 2).sum() / n)
        assert abs(res[-1] - want) <= 1e-10 * max(want, 1e-300)
        assert np.abs(b.raw_solved.cpu().numpy() - u).max() <= 1e-12 * np.abs(u).max()
    assert res[-1] < res[0]
    core.kill()
