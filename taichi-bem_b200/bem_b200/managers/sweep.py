"""Wavenumber sweeps of the transmission operator: operator-norm and
condition estimates and batched augmented least-squares solves.

The reference computes ||A^{-1}|| in an energy-scaled norm with a full SVD
of the scaled (augmented) operator for every wavenumber
(`compute_inv_norm`, `BEM_manager.py:874-920`, driven by
`demo/demo_3d_plot_Sio.py:66-104`).  Here the extreme singular values come
from block Krylov spaces of the Gram matrix G = S^H S and of its inverse,
applied with this library's LU factor and triangular solves
(`smallest_singular_value`); the Ritz values converge to the SVD's smallest
and largest singular values.
"""
from __future__ import annotations

import math
import time

import torch

from ..utils.types import AssembleType, ScopeType


def _orthonormalize(X: torch.Tensor) -> torch.Tensor:
    """Orthonormal basis of the block's columns (Householder QR of the n x p
    block; inverse iteration makes the columns nearly parallel, where
    Gram-Schmidt or Cholesky-QR lose orthogonality or break down)."""
    return torch.linalg.qr(X, mode="reduced")[0]


def _krylov_ritz(S: torch.Tensor, apply, X0: torch.Tensor, maxblocks: int, which: int, tol: float):
    """Grow a block Krylov basis Q = [X0, op X0, op^2 X0, ...] (fully
    re-orthogonalised) of the Hermitian operator `apply`, and after 2, 4, 8 ...
    blocks take the Ritz value of G = S^H S on span(Q) from the singular values
    of S Q: the smallest (which = 0) or largest (which = -1).  Stops
    when it changes by less than `tol` (relative) or at `maxblocks` blocks.
    Returns (Ritz value, blocks)."""
    blocks = [_orthonormalize(X0)]
    SQ = [S @ blocks[0]]
    prev, check = None, 2
    while True:
        if len(blocks) == min(check, maxblocks):
            # singular values of S Q (Q orthonormal): min / max of |S x| over span(Q)
            sv = torch.linalg.svdvals(torch.cat(SQ, 1))
            lam = float(sv[-1] if which == 0 else sv[0]) ** 2
            if (prev is not None and abs(lam - prev) <= tol * abs(lam)) or len(blocks) >= maxblocks:
                return lam, len(blocks)
            prev, check = lam, 2 * check
        W = apply(blocks[-1])
        Q = torch.cat(blocks, 1)
        for _ in range(2):
            W = W - Q @ (Q.conj().transpose(0, 1) @ W)
        blocks.append(_orthonormalize(W))
        SQ.append(S @ blocks[-1])


def smallest_singular_value(engine, S: torch.Tensor, block: int = 8, tol: float = 1e-10, tol_max: float = 1e-7,
                            maxit: int = 24, seed: int = 0, info: dict | None = None):
    """(sigma_min, sigma_max, Krylov blocks) of S (m x n, m >= n).

    sigma_min^2 is the smallest eigenvalue of G = S^H S.  A block Krylov
    space of G^{-1} (block size `block`; each step one multi-right-hand-side
    solve with the FP64 LU of G, bem_lu_factor / bem_lu_solve) is grown until
    the smallest Ritz value of G on it changes by less than `tol` (relative)
    between two sizes, at most `maxit` blocks.  sigma_max^2 likewise from the
    Krylov space of G itself (`tol_max`).  The Ritz values come from the
    singular values of the thin matrix S Q, with relative error eps * cond(S)
    (a Gram matrix Q^H G Q would carry eps * cond(S)^2).
    """
    n = S.shape[1]
    G = (S.conj().transpose(0, 1) @ S).contiguous()
    gen = torch.Generator(device=S.device).manual_seed(seed)
    p = min(block, n)
    X = torch.randn(n, p, dtype=torch.float64, device=S.device, generator=gen)
    if S.is_complex():
        X = torch.complex(X, torch.randn(n, p, dtype=torch.float64, device=S.device, generator=gen))
    LU = G.clone()
    piv, finfo = engine.lu_factor(LU)
    if int(finfo.item()) != 0:
        return 0.0, math.sqrt(float(torch.linalg.matrix_norm(G, 2).real)), 0

    def solve(V):
        Y = V.clone().contiguous()
        engine.lu_solve(LU, piv, Y)
        return Y

    nmax = max(1, min(maxit, n // p))
    lam_min, nb_min = _krylov_ritz(S, solve, X, nmax, 0, tol)
    lam_max, _ = _krylov_ritz(S, lambda V: G @ V, X, nmax, -1, tol_max)
    if info is not None:
        info["blocks"] = nb_min
    return math.sqrt(max(lam_min, 0.0)), math.sqrt(max(lam_max, 0.0)), nb_min


def transmission_operator(bm, k: float, A_type: int = 1, augmented: bool = True):
    """A_I = P^-_o - P^+_i (A_type 1) or A_II = P^-_o + P^+_i (A_type 2) at
    wavenumber k, assembled as get_mat_A{1,2}_inv_norm does
    (BEM_manager.py:922-950); with `augmented`, stacked on P^+_i as in
    get_augment_mat_A{1,2}_inv_norm (:952-988).  Returns a new tensor."""
    bm._mat_A.zero_()
    bm.matrix_layer_forward(k=k, sqrt_n=bm._sqrt_no, scope_type=int(ScopeType.EXTERIOR))
    bm.assemble_matA(assemble_type=int(AssembleType.ADD_P_MINUS), multiplier=1.0)
    bm.matrix_layer_forward(k=k, sqrt_n=bm._sqrt_ni, scope_type=int(ScopeType.INTERIOR))
    bm.assemble_matA(assemble_type=int(AssembleType.ADD_P_PLUS), multiplier=-1.0 if A_type == 1 else 1.0)
    A = bm._mat_A.clone()
    if not augmented:
        return A
    bm._mat_A.zero_()
    bm.assemble_matA(assemble_type=int(AssembleType.ADD_P_PLUS), multiplier=1.0)
    return torch.cat((A, bm._mat_A), 0)


def wavenumber_sweep(bm, ks, nrhs: int = 4, seed: int = 0, A_type: int = 1, scaling_k: float = 0.0,
                     norm_method: str = "iterative", norm_tol: float | None = None, norm_maxit: int | None = None):
    """For each k in `ks`: the augmented transmission operator [A(k); P^+_i(k)],
    the inverse norm and condition number of its energy-scaled form, and the
    least-squares solutions of [A; P^+_i] x = [b; 0] for `nrhs` seed-fixed
    complex Gaussian right-hand sides b.  The least-squares problems are
    solved through their normal equations with the manager's solver (mixed
    precision: FP32 tile LU + FP64 refinement; fp64: partial-pivoting LU).

    The energy scaling is formed once, at `scaling_k` (the reference forms it
    on its first call, which the reference's sweep makes at k = 0).  norm_tol
    and norm_maxit override the manager's estimator settings for the sweep."""
    n = bm.N_Neumann + bm.M_Dirichlet
    if norm_tol is not None:
        bm.norm_tol = norm_tol
    if norm_maxit is not None:
        bm.norm_maxit = norm_maxit
    bm._L1_inv_H = bm._L2_inv_H = None
    if A_type == 1:
        bm.get_mat_A1_inv_norm(scaling_k, method="none")
    else:
        bm.get_mat_A2_inv_norm(scaling_k, method="none")
    gen = torch.Generator(device=bm.device).manual_seed(seed)
    out = {"k": [], "inv_norm": [], "cond": [], "solutions": [], "ms": [], "iterations": []}
    for k in ks:
        torch.cuda.synchronize(bm.device)
        t0 = time.perf_counter()
        At = transmission_operator(bm, float(k), A_type, augmented=True)
        inv_norm, cond, its = bm.compute_inv_norm(At, A_type, method=norm_method, return_cond=True)
        b = torch.complex(torch.randn(n, nrhs, dtype=torch.float64, device=bm.device, generator=gen),
                          torch.randn(n, nrhs, dtype=torch.float64, device=bm.device, generator=gen))
        A, P = At[:n], At[n:]
        AH = A.conj().transpose(0, 1)
        Gn = (AH @ A + P.conj().transpose(0, 1) @ P).contiguous()
        rhs = (AH @ b).contiguous()
        X = bm._lu_solve_square(Gn, rhs)
        torch.cuda.synchronize(bm.device)
        out["ms"].append((time.perf_counter() - t0) * 1e3)
        out["k"].append(float(k))
        out["inv_norm"].append(inv_norm)
        out["cond"].append(cond)
        out["iterations"].append(its)
        out["solutions"].append(X)
    return out


def solution_norm_k_gradient(bm, data=None, delta: float = 1e-3, check: bool = True):
    """J(k) = ||x(k)||^2 for the manager's system A(k) x = b(k) at its
    wavenumber k (square transmission system: solver "square"), and dJ/dk by
    the adjoint method:
        A^H lam = x,     dJ/dk = 2 Re lam^H (db/dk - (dA/dk) x),
    with dA/dk x and db/dk from central differences (k +- delta) of the
    assembled operator and right-hand side, and the adjoint solve by the
    manager's solver on A^H.  `data` is the boundary-data object whose `k`
    follows the operator's (e.g. workloads.PlaneWave).  With `check`, also the
    central difference of J itself (two more solves).  Returns a dict."""
    n = bm.N_Neumann + bm.M_Dirichlet
    k0 = bm._k

    def system(k):
        bm._k = k
        if data is not None:
            data.k = k
        bm.assemble_system()
        return bm._mat_A.clone(), bm.rhs[:n].clone()

    out = {}
    torch.cuda.synchronize(bm.device)
    t0 = time.perf_counter()
    A, b = system(k0)
    x = bm._lu_solve_square(A, b)
    torch.cuda.synchronize(bm.device)
    out["solve_ms"] = (time.perf_counter() - t0) * 1e3
    out["solve_info"] = dict(bm.solve_info)
    J = float(torch.vdot(x, x).real)
    t1 = time.perf_counter()
    Ap, bp = system(k0 + delta)
    r = bp - Ap @ x
    del Ap
    Am, bm_ = system(k0 - delta)
    r = (r - (bm_ - Am @ x)) / (2.0 * delta)  # db/dk - dA/dk x
    del Am
    lam = bm._lu_solve_square(A.conj().transpose(0, 1).contiguous(), x.contiguous())
    dJ = 2.0 * float(torch.vdot(lam, r).real)
    torch.cuda.synchronize(bm.device)
    out["adjoint_ms"] = (time.perf_counter() - t1) * 1e3
    out.update(J=J, dJdk=dJ, x=x)
    if check:
        Js = []
        for k in (k0 + delta, k0 - delta):
            Ak, bk = system(k)
            xk = bm._lu_solve_square(Ak, bk)
            Js.append(float(torch.vdot(xk, xk).real))
            del Ak
        out["dJdk_central_difference"] = (Js[0] - Js[1]) / (2.0 * delta)
    bm._k = k0
    if data is not None:
        data.k = k0
    return out
