"""Known-answer tests of the oracle's quadrature, independent of the
reference's fixtures (the GPU kernels match the oracle to 1e-12, so these
carry over):

* mass matrices of P0/P1 bases, exact for the Q^2 rule;
* the single layer of a constant on the unit sphere, 1 for Laplace and
  sin(k) e^{ik} / k (the l = 0 eigenvalue i k j_0(k) h_0(k)) for Helmholtz,
  approached at O(h^2) on icospheres (the flat panels are inscribed);
* Gauss's law for the double layer, K 1 = -1/2 per unit area with outward
  normals, which a closed polyhedron satisfies exactly up to quadrature.
"""
import numpy as np
import pytest

from bem_b200.meshes import icosphere
from oracle import oracle as O


def _p0(nt):
    idx = np.arange(nt, dtype=np.int32)
    return idx, 1, idx


def _areas(v, f):
    return 0.5 * np.linalg.norm(np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 1]]), axis=1)


def test_mass_matrices_exact():
    v, f = icosphere(1)
    nt, nv = len(f), len(v)
    a = _areas(v, f)
    panels = np.arange(nt, dtype=np.int32)
    p0 = np.arange(nt, dtype=np.int32)
    p1 = f.reshape(-1).astype(np.int32)
    want00 = np.diag(a)
    want01 = np.zeros((nt, nv))
    want11 = np.zeros((nv, nv))
    for p, tri in enumerate(f):
        for i in tri:
            want01[p, i] += a[p] / 3.0
            for j in tri:
                want11[i, j] += a[p] / 12.0 * (2.0 if i == j else 1.0)
    for nbx, tdof, nby, rdof, want in ((1, p0, 1, p0, want00), (1, p0, 3, p1, want01), (3, p1, 3, p1, want11)):
        got = np.zeros(want.shape)
        O.mass(v, f, 3, panels, nbx, tdof, nby, rdof, out=got)
        assert np.abs(got - want).max() <= 1e-14 * np.abs(want).max()


def _apply(v, f, op, helm, k, quirk, Q=4):
    nt = len(f)
    one = np.ones(nt, complex if helm else float)
    y = np.zeros(nt, one.dtype)
    O.assemble(v, f, op, int(helm), k, k * k, Q, quirk, _p0(nt), _p0(nt), x=one, y=y)
    return y / _areas(v, f)


@pytest.mark.parametrize("helm,k", [(False, 0.0), (True, 1.5)])
def test_single_layer_of_a_constant_on_the_sphere(helm, k):
    want = np.sin(k) * np.exp(1j * k) / k if helm else 1.0
    err = []
    for s in (2, 3):
        v, f = icosphere(s)
        err.append(np.abs(_apply(v, f, O.OP_V, helm, k, quirk=0) - want).max() / abs(want))
    assert err[1] < 6e-3 and err[0] / err[1] > 3.5  # O(h^2)


def test_gauss_law_for_the_double_layer():
    for s in (2, 3):
        v, f = icosphere(s)
        assert np.abs(_apply(v, f, O.OP_K, False, 0.0, quirk=0) + 0.5).max() < 1e-5


def test_reference_orientation_handling_leaves_an_O_h_error():
    """quirk = 1 reproduces the reference's Sauter-Schwab orientation handling
    (the shared vertex or edge is not moved to the map's singular point); the
    near-pair error it leaves in K 1 shrinks with the mesh but is not at
    quadrature level."""
    err = []
    for s in (2, 3):
        v, f = icosphere(s)
        err.append(np.abs(_apply(v, f, O.OP_K, False, 0.0, quirk=1) + 0.5).max())
    assert 1e-4 < err[1] < err[0] < 1e-2


def _point_source_trace_error(s, quirk):
    """Laplace interior Dirichlet on icosphere s with u = 1/|x - x0|,
    x0 = (2, 2, 2), GaussQR 4: l2 error of the P0 Neumann trace against
    du/dn at the centroids."""
    from tests._util import data_callbacks
    fD, fN = data_callbacks("laplace_point")
    v, f = icosphere(s)
    params = dict(dim=3, GaussQR=4, kernel="Laplace", boundary="Dirichlet", scope="Interior", k=0.0, Q_Neumann=0,
                  Q_Dirichlet=1)
    P = O.Problem(v, f, params, fD, fN, quirk=quirk)
    t = P.run()["raw_solved"]
    exact = fN(v[f].mean(axis=1), P.mesh.panel_normals)
    return np.linalg.norm(t - exact) / np.linalg.norm(exact)


def test_point_source_trace_converges_with_the_corrected_quadrature():
    err = [_point_source_trace_error(s, quirk=False) for s in (1, 2, 3)]
    assert err[2] < 7e-3 and err[0] / err[1] > 2.5 and err[1] / err[2] > 2.5


def test_reference_quadrature_trace_does_not_converge():
    """The reference's orientation handling (quirk = 1) leaves an O(h),
    high-frequency error in the near pairs of K g; V^{-1} amplifies it by
    O(1/h), so the trace error stays O(1) under refinement (the reference's
    own fixtures show the same: its cube and icosphere solutions are O(1) away
    from their analytic traces)."""
    err = [_point_source_trace_error(s, quirk=True) for s in (1, 2)]
    assert min(err) > 0.3


def _apply_2d(N, op, helm, k, R=0.5, Q=4):
    from bem_b200.meshes import analytical_disk
    from oracle import oracle2d as O2
    v, f = analytical_disk(R, N)
    L = np.linalg.norm(v[f[:, 1]] - v[f[:, 0]], axis=1)
    p0 = (np.arange(N, dtype=np.int32), 1, np.arange(N, dtype=np.int32))
    y = np.zeros(N, complex if helm else float)
    O2.assemble(v, f, {"V": O2.OP_V, "K": O2.OP_K}[op], helm, k, k * k, Q, p0, p0, x=np.ones(N, y.dtype), y=y)
    return y / L


def test_2d_single_layer_of_a_constant_on_a_circle():
    """On the circle of radius R the single layer of 1 is -R log R (Laplace,
    G = -log r / 2 pi) and (i pi R / 2) J_0(kR) H_0(kR) (Helmholtz,
    G = (i/4) H_0(k r))."""
    from scipy import special
    R, k = 0.5, 2.0
    lap = [np.abs(_apply_2d(N, "V", False, 0.0, R) + R * np.log(R)).max() / abs(R * np.log(R)) for N in (32, 64, 128)]
    assert max(lap) < 2e-3
    want = 0.5j * np.pi * R * special.jv(0, k * R) * special.hankel1(0, k * R)
    helm = [np.abs(_apply_2d(N, "V", True, k, R) - want).max() / abs(want) for N in (32, 64, 128)]
    assert helm[2] < 2e-4 and helm[0] / helm[1] > 3 and helm[1] / helm[2] > 3  # O(h^2)


def test_2d_gauss_law_for_the_double_layer():
    """K 1 = -1/2 on a closed polygon, to first order: the reference's scheme
    integrates vertex-sharing segment pairs with the plain Q^2 rule."""
    err = [np.abs(_apply_2d(N, "K", False, 0.0) + 0.5).max() for N in (32, 64, 128)]
    assert err[2] < 4e-4 and err[0] / err[1] > 1.8 and err[1] / err[2] > 1.8


def test_hypersingular_of_a_constant_on_the_sphere():
    """W 1 with P1 bases: the surface curls of a constant vanish, so Laplace
    W 1 = 0 exactly and Helmholtz W 1 = -k^2 int G n_x.n_y dS, which on the
    unit sphere (n_x.n_y = 1 - r^2/2, dS = 2 pi r dr) is
    -k^2 (1/2 int_0^2 e^{ikr} dr - 1/4 int_0^2 r^2 e^{ikr} dr)."""
    from scipy import integrate
    k = 1.5
    quad = lambda g: integrate.quad(lambda r: g(r) * np.cos(k * r), 0, 2)[0] + \
        1j * integrate.quad(lambda r: g(r) * np.sin(k * r), 0, 2)[0]
    want = -k * k * (0.5 * quad(lambda r: 1.0) - 0.25 * quad(lambda r: r * r))
    err = []
    for s in (2, 3):
        v, f = icosphere(s)
        nt, nv = len(f), len(v)
        va = np.bincount(f.reshape(-1), weights=np.repeat(_areas(v, f) / 3.0, 3), minlength=nv)
        p1 = (np.arange(nt, dtype=np.int32), 3, f.reshape(-1).astype(np.int32))
        lap = np.zeros(nv)
        O.assemble(v, f, O.OP_W, 0, 0.0, 0.0, 3, 0, p1, p1, x=np.ones(nv), y=lap)
        assert np.abs(lap).max() < 1e-14
        y = np.zeros(nv, complex)
        O.assemble(v, f, O.OP_W, 1, k, k * k, 3, 0, p1, p1, x=np.ones(nv, complex), y=y)
        err.append(np.abs(y / va - want).max() / abs(want))
    assert err[1] < 7e-3 and err[0] / err[1] > 3.5  # O(h^2)


def test_double_layer_and_its_adjoint_of_a_constant_on_the_sphere():
    """On the unit sphere (x - y).n_y = (y - x).n_x = -r^2/2, so K 1 and K' 1
    share the closed form -1/4 int_0^2 (1 - ikr) e^{ikr} dr (-1/2 at k = 0).
    K' takes the flat panel's normal at the test point, so unlike K it has no
    exact solid-angle identity on a polyhedron and converges to first order
    for Laplace."""
    from scipy import integrate
    k = 1.5
    quad = lambda g: integrate.quad(lambda r: (g(r) * np.exp(1j * k * r)).real, 0, 2)[0] + \
        1j * integrate.quad(lambda r: (g(r) * np.exp(1j * k * r)).imag, 0, 2)[0]
    want = -0.25 * quad(lambda r: 1 - 1j * k * r)
    err = {}
    for s in (2, 3):
        v, f = icosphere(s)
        err[("K", s)] = np.abs(_apply(v, f, O.OP_K, True, k, quirk=0) - want).max() / abs(want)
        err[("KP", s)] = np.abs(_apply(v, f, O.OP_KP, True, k, quirk=0) - want).max() / abs(want)
        err[("KPL", s)] = np.abs(_apply(v, f, O.OP_KP, False, 0.0, quirk=0) + 0.5).max() / 0.5
    assert err[("K", 3)] < 6e-3 and err[("K", 2)] / err[("K", 3)] > 3.5
    assert err[("KP", 3)] < 9e-3 and err[("KP", 2)] / err[("KP", 3)] > 2.5
    assert err[("KPL", 3)] < 8e-3 and err[("KPL", 2)] / err[("KPL", 3)] > 1.5
