"""The benchmark configurations as simulation_parameters + boundary data.

Each builder returns (params, fD, fN) for CoreManager.  The meshes are
generated unit icospheres (the reference's own sphere assets have the same
sizes: sphere.obj 1280 panels = subdivision 3, fined_sphere.obj 5120 =
subdivision 4); data are the configurations' analytic fields.
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import upload


def plane_wave_direction(seed: int = 0) -> np.ndarray:
    g = torch.Generator().manual_seed(seed)
    d = torch.randn(3, generator=g, dtype=torch.float64)
    return (d / d.norm()).numpy()


def laplace_point_source(x0=(2.0, 2.0, 2.0)):
    """u = 1/|x - x0| (harmonic inside the unit sphere); returns (fD, fN)."""
    def fD(x, s=1.0):
        c = upload(x0, x.device, x.dtype)
        return 1.0 / torch.linalg.norm(x - c, dim=1)

    def fN(x, n, s=1.0):
        c = upload(x0, x.device, x.dtype)
        d = x - c
        return -(d * n).sum(1) / torch.linalg.norm(d, dim=1) ** 3
    return fD, fN


def plane_wave(k: float, direction):
    """u = exp(i k sqrt_n d.x); returns (fD, fN) (fN = du/dn)."""
    dvec = np.asarray(direction, dtype=np.float64)

    def fD(x, s=1.0):
        d = upload(dvec, x.device, x.dtype)
        return torch.exp(1j * (k * s) * (x @ d))

    def fN(x, n, s=1.0):
        d = upload(dvec, x.device, x.dtype)
        return 1j * (k * s) * (n @ d) * torch.exp(1j * (k * s) * (x @ d))
    return fD, fN


class PlaneWave:
    """u = exp(i k sqrt_n d.x) with a mutable wavenumber k (for derivatives in
    k the boundary data follow the operator's k); fD and fN are the
    reference's callback signatures."""

    def __init__(self, k: float, direction):
        self.k = float(k)
        self.d = np.asarray(direction, dtype=np.float64)

    def fD(self, x, s=1.0):
        d = upload(self.d, x.device, x.dtype)
        return torch.exp(1j * (self.k * s) * (x @ d))

    def fN(self, x, n, s=1.0):
        d = upload(self.d, x.device, x.dtype)
        return 1j * (self.k * s) * (n @ d) * torch.exp(1j * (self.k * s) * (x @ d))

    def dfD_dk(self, x, s=1.0):
        """d fD / dk = i s (d.x) exp(i k s d.x)."""
        d = upload(self.d, x.device, x.dtype)
        xd = x @ d
        return 1j * s * xd * torch.exp(1j * (self.k * s) * xd)

    def dfN_dk(self, x, n, s=1.0):
        """d fN / dk = i s (n.d) exp(i k s d.x) (1 + i k s d.x)."""
        d = upload(self.d, x.device, x.dtype)
        xd = x @ d
        return 1j * s * (n @ d) * torch.exp(1j * (self.k * s) * xd) * (1.0 + 1j * (self.k * s) * xd)


def _base(**kw):
    p = dict(dim=3, object="icosphere3", GaussQR=5, n_i=1, n_o=1, k=0.0, kernel="Laplace", boundary="Dirichlet",
             scope="Interior", show="Default", Q_Neumann=0, Q_Dirichlet=1, log_to_disk=False, make_video=False,
             show_wireframe=False, vis=False)
    p.update(kw)
    return p


def laplace_dirichlet_s3(precision="fp64"):
    """Laplace 3D interior Dirichlet on icosphere s3 (1280 panels), GaussQR=5,
    u = 1/|x - x0|, x0 = (2,2,2): V t = (1/2 M + K) g."""
    fD, fN = laplace_point_source()
    return _base(object="icosphere3", precision=precision), fD, fN


def helmholtz_dirichlet_s4(precision="mixed", seed=0):
    """Helmholtz 3D interior Dirichlet, k = 3, icosphere s4 (5120 panels),
    GaussQR=5, plane wave exp(i k d.x) with a seeded random unit d."""
    fD, fN = plane_wave(3.0, plane_wave_direction(seed))
    return _base(object="icosphere4", kernel="Helmholtz", k=3.0, precision=precision), fD, fN


def transmission_sweep_s4(precision="mixed", n_k=60):
    """Wavenumber sweep of the augmented transmission operator on icosphere s4
    (5120 panels, P1 Neumann and Dirichlet: 5124 unknowns), k_i = 16 + i/30,
    with the reference sweep's parameters (demo_3d_plot_Sio.py: n_i = 3,
    n_o = 1, GaussQR = 3).  Returns (params, fD, fN, ks)."""
    fD, fN = plane_wave(16.0, plane_wave_direction(0))
    params = _base(object="icosphere4", kernel="Helmholtz_Transmission", boundary="Full", k=16.0, n_i=3.0,
                   n_o=1.0, GaussQR=3, Q_Neumann=1, Q_Dirichlet=1, precision=precision)
    ks = [16.0 + i / 30.0 for i in range(n_k)]
    return params, fD, fN, ks


def transmission_s5(precision="mixed", subdiv=5, solver="square"):
    """Helmholtz transmission (2x2 block Calderon system), icosphere s5 (20480
    panels, P0 Neumann + P1 Dirichlet: 30722 unknowns), k_out = 5,
    n_i = 2.25 (k_in = 7.5), n_o = 1, GaussQR = 5, incident plane wave with a
    seeded direction; solver "square" (LU of the square system) or "lstsq"
    (the reference's augmented least squares, by its normal equations).
    Returns (params, PlaneWave)."""
    pw = PlaneWave(5.0, plane_wave_direction(0))
    params = _base(object=f"icosphere{subdiv}", kernel="Helmholtz_Transmission", boundary="Full", k=5.0, n_i=2.25,
                   n_o=1.0, scope="Exterior", precision=precision, solver=solver)
    return params, pw


WORKLOADS = {f.__name__: f for f in (laplace_dirichlet_s3, helmholtz_dirichlet_s4, transmission_sweep_s4,
                                      transmission_s5)}
