"""Operator-norm API and wavenumber sweep of the transmission operator
(BEM_manager.py:874-988, demo/demo_3d_plot_Sio.py) against the oracle: the
FP64 operators assembled by the CPU restatement, scaled as the reference
does, and their singular values from numpy."""
import numpy as np
import pytest
import torch

from _util import rel_err

pytestmark = pytest.mark.gpu

KS = [1.5, 4.0]


def _params(precision):
    from bem_b200 import icosphere
    v, f = icosphere(1)
    return dict(dim=3, object="icosphere1", vertices=v, panels=f, GaussQR=3, n_i=3.0, n_o=1.0, k=0.0,
                kernel="Helmholtz_Transmission", boundary="Full", scope="Interior", show="Default", Q_Neumann=1,
                Q_Dirichlet=1, precision=precision, log_to_disk=False, make_video=False, show_wireframe=False,
                vis=False), v, f


def _manager(precision):
    from bem_b200.managers import CoreManager
    from bem_b200.workloads import plane_wave
    params, v, f = _params(precision)
    fD, fN = plane_wave(1.0, [0.0, 0.0, 1.0])
    core = CoreManager(params)
    core.initialization(fD, fN)
    return core, v, f


def _oracle_ops(v, f, k, A_type):
    from oracle import oracle as O
    params, _, _ = _params("fp64")
    params["k"] = k
    fD = lambda x, s=1.0: np.exp(1j * x[:, 2])
    fN = lambda x, n, s=1.0: 1j * n[:, 2] * np.exp(1j * x[:, 2])
    P = O.Problem(v, f, params, fD, fN)
    lo, li = P.forward(P.sqrt_no), P.forward(P.sqrt_ni)
    A = np.zeros((P.n, P.n), complex)
    P.add_identity(A, 0.5)
    P.add_M(A, lo, -1.0)
    P.add_identity(A, -0.5 if A_type == 1 else 0.5)
    P.add_M(A, li, -1.0 if A_type == 1 else 1.0)
    Pp = np.zeros_like(A)
    P.add_identity(Pp, 0.5)
    P.add_M(Pp, li, 1.0)
    return A, Pp, P.mesh


def _oracle_inv_norms(v, f, A_type):
    """Reference procedure: scaling from the k = 0 operator, then 1/sigma_min
    of the scaled operator and of the scaled augmented operator."""
    A0, _, m = _oracle_ops(v, f, 0.0, A_type)
    M = m.M_D
    if A_type == 1:
        MV = np.zeros_like(A0)
        MV[:M, :M] = A0[:M, :M]
        MV[M:, M:] = A0[M:, M:]
        MV = (MV + MV.T) / 2.0
    else:
        MV = np.zeros_like(A0)
        MV[:M, :M] = A0[:M, M:]
        MV[M:, M:] = A0[M:, :M]
    # the manager's fixed relative shift of the scaling block (BEMManager._shifted)
    L = np.linalg.cholesky(MV + 1e-10 * np.abs(MV).max() * np.eye(MV.shape[0]))
    LinvH = np.linalg.inv(L).T.conj()
    out = []
    for k in KS:
        A, Pp, _ = _oracle_ops(v, f, k, A_type)
        S = LinvH.T.conj() @ A @ LinvH
        Sa = np.concatenate([LinvH.T.conj() @ A @ LinvH, LinvH.T.conj() @ Pp @ LinvH], 0)
        out.append((1.0 / np.linalg.svd(S, compute_uv=False).min(),
                    1.0 / np.linalg.svd(Sa, compute_uv=False).min()))
    return out


@pytest.mark.parametrize("A_type", [1, 2])
def test_inverse_norms_match_oracle(A_type):
    core, v, f = _manager("fp64")
    b = core._BEM_manager
    ref = _oracle_inv_norms(v, f, A_type)
    get = b.get_mat_A1_inv_norm if A_type == 1 else b.get_mat_A2_inv_norm
    aug = b.get_augment_mat_A1_inv_norm if A_type == 1 else b.get_augment_mat_A2_inv_norm
    get(0.0)  # the reference forms the energy scaling on its first call, at k = 0
    for k, (r, ra) in zip(KS, ref):
        for method in ("svd", "iterative"):
            got = get(k, method=method)
            assert abs(got - r) <= 1e-6 * r, (k, method, got, r)
            got_a = aug(k, False, method=method)
            assert abs(got_a - ra) <= 1e-6 * ra, (k, method, got_a, ra)
    core.kill()


def test_sweep_mixed_matches_fp64():
    from bem_b200.managers.sweep import wavenumber_sweep
    out = {}
    for prec in ("fp64", "mixed"):
        core, v, f = _manager(prec)
        out[prec] = wavenumber_sweep(core._BEM_manager, KS, nrhs=4, seed=0)
        core.kill()
    for a, b_ in zip(out["fp64"]["solutions"], out["mixed"]["solutions"]):
        assert rel_err(b_.cpu().numpy(), a.cpu().numpy()) < 1e-6
    for a, b_ in zip(out["fp64"]["inv_norm"], out["mixed"]["inv_norm"]):
        assert abs(a - b_) <= 1e-5 * a


def test_sweep_solutions_match_oracle_lstsq():
    """The sweep's mixed-precision least-squares solutions against numpy's
    lstsq (the reference's torch.linalg.lstsq, BEM_manager.py:1049) of the
    oracle's stacked [A_I; P+_i] with the same right-hand sides."""
    from bem_b200.managers.sweep import wavenumber_sweep
    core, v, f = _manager("mixed")
    out = wavenumber_sweep(core._BEM_manager, KS, nrhs=2, seed=1)
    core.kill()
    for k, X, B in zip(KS, out["solutions"], out["rhs"]):
        A, Pp, _ = _oracle_ops(v, f, k, 1)
        n = A.shape[0]
        Sa = np.concatenate([A, Pp], 0)
        rhs = np.concatenate([B.cpu().numpy(), np.zeros((n, B.shape[1]))], 0)
        ref = np.linalg.lstsq(Sa, rhs, rcond=None)[0]
        assert rel_err(X.cpu().numpy(), ref) < 1e-6


def test_krylov_estimates_with_a_complete_basis():
    """The block-Krylov estimator when its bases fill the whole space
    (icosphere s1, 8-vector blocks up to n): inverse and power iteration make
    most columns numerically dependent, and the estimates must still be the
    extreme singular values of the numpy SVD of the same scaled operator."""
    from bem_b200.managers.sweep import extreme_singular_values
    core, v, f = _manager("fp64")
    b = core._BEM_manager
    b.get_mat_A1_inv_norm(0.0, method="none")
    from bem_b200.managers.sweep import transmission_operator
    At = transmission_operator(b, KS[1], 1, augmented=True)
    n = At.shape[1]
    Linv = b._L1_inv
    blocks = []
    for r0 in (0, n):
        T = torch.zeros(n, n, dtype=At.dtype, device=At.device)
        b.engine.gemm(Linv, At[r0:r0 + n].contiguous(), T, a_lower=True)
        Sb = torch.zeros_like(T)
        b.engine.gemm(T, Linv, Sb, conj_b=True, b_upper=True)
        blocks.append(Sb)
    sv = np.linalg.svd(torch.cat(blocks, 0).cpu().numpy(), compute_uv=False)
    smin, smax, its = extreme_singular_values(b.engine, blocks, tol=0.0, tol_max=0.0, maxit=n // 8)
    core.kill()
    assert abs(smin - sv[-1]) <= 1e-6 * sv[-1], (smin, sv[-1])
    assert abs(smax - sv[0]) <= 1e-9 * sv[0], (smax, sv[0])


@pytest.mark.parametrize("dtype", [torch.float64, torch.complex128])
@pytest.mark.parametrize("n", [300, 5000])
def test_basis_cgs2_matches_torch(dtype, n):
    """The fused CGS2 appends (bem_cgs2_append) against the same CGS2 steps in
    torch FP64, including nearly and exactly dependent columns; Q is
    orthonormal and W = Q R."""
    from bem_b200.engine import Engine
    from bem_b200.managers.sweep import Basis
    eng = Engine("cuda:0")
    try:
        cap = 24
        g = torch.Generator(device="cuda").manual_seed(3)
        W = torch.randn(n, 16, dtype=torch.float64, device="cuda", generator=g)
        if dtype.is_complex:
            W = torch.complex(W, torch.randn(n, 16, dtype=torch.float64, device="cuda", generator=g))
        W = torch.cat([W, W[:, :4] + 1e-13 * W[:, 4:8], W[:, 8:12] @ torch.ones(4, 4, dtype=dtype, device="cuda")],
                      1)  # 24 columns, the last 8 nearly or exactly dependent
        b = Basis(eng, n, cap, dtype, "cuda")
        assert b.append(W[:, :5]) == 5 and b.append(W[:, 5:]) == 19 and b.append(W[:, :1]) == 0
        # the same steps in torch
        Q = torch.zeros(n, cap, dtype=dtype, device="cuda")
        Rt = torch.zeros(cap, cap, dtype=dtype, device="cuda")
        for jj in range(cap):
            v = W[:, jj].clone()
            r = torch.zeros(jj, dtype=dtype, device="cuda")
            for _ in range(2):
                h = Q[:, :jj].conj().T @ v
                v = v - Q[:, :jj] @ h
                r = r + h
            rjj = torch.linalg.vector_norm(v)
            q = v / rjj.clamp_min(1e-300)
            for _ in range(2):
                q = q - Q[:, :jj] @ (Q[:, :jj].conj().T @ q)
            q = q / torch.linalg.vector_norm(q).clamp_min(1e-300)
            Q[:, jj] = q
            Rt[jj, :jj] = r
            Rt[jj, jj] = rjj
        scale = float(W.abs().max())
        assert float((b.Rt - Rt).abs().max()) < 1e-11 * scale * n ** 0.5
        # columns of the exactly dependent tail are rounding noise made orthonormal: compare the rest
        assert float((b.Q[:, :16] - Q[:, :16]).abs().max()) < 1e-10
        eye = torch.eye(cap, dtype=dtype, device="cuda")
        assert float((b.Q.conj().T @ b.Q - eye).abs().max()) < 1e-12
        R = b.Rt.T
        assert float((b.Q[:, :16] @ R[:16, :16] - W[:, :16]).abs().max()) < 1e-12 * scale * n ** 0.5
    finally:
        eng.close()
