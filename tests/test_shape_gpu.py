"""Shape gradient of the Laplace interior Dirichlet problem through the
adjoint kernels (bem_adjoint_vertices) against central finite differences of
the FP64 forward solve, J = ||t - t_target||^2 with t_target from the
unperturbed sphere."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup(precision, subdiv=2, Q=3):
    from bem_b200 import icosphere
    from bem_b200.meshes import perturbed_sphere
    from bem_b200.shape import DirichletShape, point_source
    v0, f = icosphere(subdiv)
    v, _ = perturbed_sphere(subdiv, lmax=6, amplitude=0.05, seed=0)
    u, gu = point_source()
    prob = DirichletShape(f, u, gu, gauss_qr=Q, precision=precision)
    dev = prob.device
    t_target = prob.forward(torch.as_tensor(v0, device=dev)).clone()
    return prob, torch.as_tensor(v, device=dev), t_target


def _J(prob, X, t_target):
    t = prob.forward(X)
    return float(((t - t_target) ** 2).sum())


def _adjoint_grad(prob, X, t_target):
    from bem_b200.shape import DirichletShapeSolve
    Xg = X.clone().requires_grad_(True)
    t = DirichletShapeSolve.apply(Xg, prob)
    J = ((t - t_target) ** 2).sum()
    J.backward()
    return Xg.grad


def test_adjoint_matches_central_differences():
    prob, X, t_target = _setup("fp64")
    G = _adjoint_grad(prob, X, t_target)
    rng = np.random.default_rng(3)
    h = 1e-6
    gmax = float(G.abs().max())
    for _ in range(8):
        v = int(rng.integers(0, X.shape[0]))
        c = int(rng.integers(0, 3))
        Xp, Xm = X.clone(), X.clone()
        Xp[v, c] += h
        Xm[v, c] -= h
        fd = (_J(prob, Xp, t_target) - _J(prob, Xm, t_target)) / (2 * h)
        assert abs(float(G[v, c]) - fd) <= 1e-5 * gmax, (v, c, float(G[v, c]), fd, gmax)


def test_mixed_gradient_matches_fp64():
    p64, X, t64 = _setup("fp64")
    g64 = _adjoint_grad(p64, X, t64)
    pmx, X2, tmx = _setup("mixed")
    gmx = _adjoint_grad(pmx, X2, tmx)
    assert float((gmx - g64).norm() / g64.norm()) < 1e-4


def test_adjoint_matches_central_differences_s3_32_coordinates():
    """The same check on the 1280-panel perturbed sphere (GaussQR = 4) at 32
    seeded vertex coordinates, h = 1e-6 as in the shape workload: every
    coordinate within 1e-5 of the gradient's largest entry, and the median
    relative difference below 1e-4."""
    prob, X, t_target = _setup("fp64", subdiv=3, Q=4)
    G = _adjoint_grad(prob, X, t_target)
    rng = np.random.default_rng(11)
    h = 1e-6
    gmax = float(G.abs().max())
    rel = []
    for _ in range(32):
        v = int(rng.integers(0, X.shape[0]))
        c = int(rng.integers(0, 3))
        Xp, Xm = X.clone(), X.clone()
        Xp[v, c] += h
        Xm[v, c] -= h
        fd = (_J(prob, Xp, t_target) - _J(prob, Xm, t_target)) / (2 * h)
        g = float(G[v, c])
        assert abs(g - fd) <= 1e-5 * gmax, (v, c, g, fd, gmax)
        rel.append(abs(g - fd) / max(abs(fd), 1e-3 * gmax))
    assert float(np.median(rel)) < 1e-4, np.median(rel)
