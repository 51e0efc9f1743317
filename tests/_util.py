"""Shared helpers for the test-suite (fixtures, data callbacks, spaces)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES_3D = ["cube_lap_dir_q5", "cube_lap_neu_q5", "cube_helm_mix_ext_q4", "cube_trans_q3", "ico1_lap_full_q3",
               "ico1_helm_dir_p1_q3"]
# the reference's 2D path on its analytical disk (N segments)
FIXTURES_2D = ["disk32_lap_dir_q4", "disk32_lap_neu_q4", "disk24_helm_mix_ext_q3", "disk24_helm_dir_p1_q3",
               "disk256_lap_dir_q3"]
FIXTURES = FIXTURES_3D + FIXTURES_2D


def load_fixture(name):
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        import pytest
        pytest.skip(f"golden fixture {name} not generated")
    d = np.load(path)
    return {k: d[k] for k in d.files}


def to_complex(a):
    a = np.asarray(a)
    if a.shape[-1] == 2:
        return a[..., 0] + 1j * a[..., 1]
    return a[..., 0]


def data_callbacks(kind, k=0.0, direction=None):
    """Boundary data of the golden cases as vectorised numpy callables:
    fD(x[m,3], sqrt_n) and fN(x[m,3], n[m,3], sqrt_n)."""
    if kind == "laplace_point":
        x0 = np.array([2.0, 2.0, 2.0])

        def fD(x, s=1.0):
            return 1.0 / np.linalg.norm(x - x0, axis=1)

        def fN(x, n, s=1.0):
            return -np.sum((x - x0) * n, 1) / np.linalg.norm(x - x0, axis=1) ** 3
        return fD, fN
    if kind == "laplace_2d":
        # u = (x^2 - y^2) / 2 (the 2D data of the reference's Laplace demo)
        def fD(x, s=1.0):
            return 0.5 * x[:, 0] ** 2 - 0.5 * x[:, 1] ** 2

        def fN(x, n, s=1.0):
            return x[:, 0] * n[:, 0] - x[:, 1] * n[:, 1]
        return fD, fN
    d = np.asarray(direction, dtype=np.float64)

    def fD(x, s=1.0):
        return np.exp(1j * k * s * (x @ d))

    def fN(x, n, s=1.0):
        return 1j * k * s * (n @ d) * np.exp(1j * k * s * (x @ d))
    return fD, fN


def full_spaces(nv, tris, nb):
    """(panels, nb, dof) covering every panel: P0 dof = panel, P1 dof = vertex."""
    nt = len(tris)
    panels = np.arange(nt, dtype=np.int32)
    if nb == 1:
        return panels, 1, panels.copy()
    t = np.asarray(tris, dtype=np.int32)
    return panels, t.shape[1], t.reshape(-1).copy()


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def torch_callbacks(kind, k=0.0, direction=None):
    """Same data as `data_callbacks`, as torch functions on device tensors
    (the form the bem_b200 facade calls)."""
    import torch
    if kind == "laplace_point":
        def fD(x, s=1.0):
            x0 = torch.tensor([2.0, 2.0, 2.0], dtype=x.dtype, device=x.device)
            return 1.0 / torch.linalg.norm(x - x0, dim=1)

        def fN(x, n, s=1.0):
            x0 = torch.tensor([2.0, 2.0, 2.0], dtype=x.dtype, device=x.device)
            return -((x - x0) * n).sum(1) / torch.linalg.norm(x - x0, dim=1) ** 3
        return fD, fN
    if kind == "laplace_2d":
        def fD(x, s=1.0):
            return 0.5 * x[:, 0] ** 2 - 0.5 * x[:, 1] ** 2

        def fN(x, n, s=1.0):
            return x[:, 0] * n[:, 0] - x[:, 1] * n[:, 1]
        return fD, fN

    def fD(x, s=1.0):
        d = torch.as_tensor(direction, dtype=x.dtype, device=x.device)
        return torch.exp(1j * k * s * (x @ d))

    def fN(x, n, s=1.0):
        d = torch.as_tensor(direction, dtype=x.dtype, device=x.device)
        return 1j * k * s * (n @ d) * torch.exp(1j * k * s * (x @ d))
    return fD, fN
