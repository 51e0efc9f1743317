"""Wavenumber sweeps of the transmission operator: operator-norm and
condition estimates and augmented least-squares solves, on this library's
kernels.

The reference computes ||A^{-1}|| in an energy-scaled norm with a full SVD
of the scaled (augmented) operator for every wavenumber
(`compute_inv_norm`, `BEM_manager.py:874-920`, driven by
`demo/demo_3d_plot_Sio.py:63-104`).  Here the extreme singular values come
from block Krylov spaces of the Gram matrix G = S^H S and of its inverse
(`extreme_singular_values`); the Ritz values converge to the SVD's smallest
and largest singular values.  Every O(n^3) and O(n^2) step runs on this
library's FP64 kernels: the scaled operator by bem_gemm (DMMA), G by
bem_gram (DMMA), its inverse by bem_chol_inverse, the bases by classical
Gram-Schmidt with one re-orthogonalisation (CGS2) on bem_gemm products.  The
host sees only the p x p triangle of the Ritz step (p <= a few hundred), whose
singular values numpy takes.
"""
from __future__ import annotations

import math
import time

import numpy as np
import torch

from ..utils.types import AssembleType, ScopeType


class Basis:
    """Orthonormal columns Q (n x j, FP64 real or complex, at most `cap`)
    grown column by column by CGS2 (bem_cgs2_append):
        h = Q^H v,  v -= Q h   (twice),   r_jj = ||v||,  q_j = v / r_jj,
    so that appended columns W satisfy W = Q R with R upper triangular, kept
    on the device as its transpose Rt (Rt[c, i] = R[i, c]).  A column
    numerically inside span(Q) (frequent in inverse and power iteration)
    leaves a tiny r_jj, which R keeps, and a residual of rounding noise with
    components along Q; the normalised q_j is therefore projected twice more
    and normalised again (these last coefficients, of the order of r_jj, do
    not enter R), which makes it orthogonal to Q whether or not the column was
    dependent.  An exactly dependent column leaves r_jj = 0.

    Each column is one cooperative launch of this library (its ten grid
    barriers replace about thirty small launches per column), queued without
    a host synchronisation; the last column of each append checks the
    device's timeout flag."""

    def __init__(self, engine, n, cap, dtype, device):
        self.engine = engine
        self.Q = torch.zeros(n, cap, dtype=dtype, device=device)
        self.Rt = torch.zeros(cap, cap, dtype=dtype, device=device)
        self.j = 0
        self.cap = cap

    @property
    def active(self) -> torch.Tensor:
        return self.Q[:, :self.j]

    def append(self, W: torch.Tensor) -> int:
        """Append the columns of W (n x p); returns the number appended (the
        basis stops at `cap`)."""
        W = W if W.stride(-1) == 1 or W.dim() == 1 else W.contiguous()
        p = W.shape[1]
        added = 0
        for c in range(p):
            if self.j >= self.cap:
                break
            last = c == p - 1 or self.j + 1 >= self.cap
            self.engine.cgs2_append(self.Q, self.j, W[:, c], self.Rt, check=last)
            self.j += 1
            added += 1
        return added

    def r_host(self):
        """R's transpose (j x j) on the host: its singular values are R's."""
        return self.Rt[:self.j, :self.j].cpu().numpy()


def _ritz(engine, S_blocks, Q: torch.Tensor, rbasis: Basis, which: int) -> float:
    """Append S q for the new columns q of Q to `rbasis` (the CGS2 basis of
    S Q with its R) and return the extreme squared singular value of S Q,
    i.e. the Ritz value of G = S^H S on span(Q): relative accuracy eps
    cond(S), where the Gram form Q^H G Q would have eps cond(S)^2."""
    n = Q.shape[0]
    SQ = torch.zeros(sum(b.shape[0] for b in S_blocks), Q.shape[1], dtype=Q.dtype, device=Q.device)
    r0 = 0
    for B in S_blocks:
        engine.gemm(B, Q, SQ[r0:r0 + B.shape[0]])
        r0 += B.shape[0]
    assert r0 == SQ.shape[0] and n == S_blocks[0].shape[1]
    rbasis.append(SQ)
    sv = np.linalg.svd(rbasis.r_host(), compute_uv=False)
    return float(sv[-1] if which == 0 else sv[0]) ** 2


def _krylov_ritz(engine, S_blocks, apply, X0, maxblocks: int, which: int, tol: float, seed: int):
    """Grow a block Krylov basis [X0, op X0, op^2 X0, ...] (CGS2) of the
    Hermitian operator `apply`; after 2, 4, 8 ... blocks take the Ritz value
    of G = S^H S on the basis: the smallest (which = 0) or largest (-1)
    squared singular value of S Q.  Stops when it changes by less than `tol`
    (relative) or at `maxblocks` blocks.  Returns (Ritz value, blocks)."""
    n, p = X0.shape
    cap = p * maxblocks
    basis = Basis(engine, n, cap, X0.dtype, X0.device)
    rbasis = Basis(engine, sum(b.shape[0] for b in S_blocks), cap, X0.dtype, X0.device)
    basis.append(X0)
    done_cols, nblocks = 0, 1
    prev, check, lam = None, 2, 0.0
    while True:
        if nblocks == min(check, maxblocks):
            lam = _ritz(engine, S_blocks, basis.Q[:, done_cols:basis.j].contiguous(), rbasis, which)
            done_cols = basis.j
            if (prev is not None and abs(lam - prev) <= tol * abs(lam)) or nblocks >= maxblocks:
                return lam, nblocks
            prev, check = lam, 2 * check
        last = basis.Q[:, basis.j - p:basis.j].contiguous()
        if basis.append(apply(last)) == 0:
            return lam, nblocks
        nblocks += 1


# relative diagonal shifts tried, in order, for the inverse iteration's Cholesky
SHIFTS = (0.0, 1e-15, 1e-13, 1e-11, 1e-9)


def extreme_singular_values(engine, S_blocks, block: int = 8, tol: float = 1e-10, tol_max: float = 1e-7,
                            maxit: int = 24, seed: int = 0, info: dict | None = None):
    """(sigma_min, sigma_max, Krylov blocks) of S = [S_0; S_1; ...] (row
    blocks, each m_i x n, sum m_i >= n).

    sigma_min^2 is the smallest eigenvalue of G = S^H S.  G is formed by the
    FP64 normal-matrix kernel (bem_gram, column scaling D: G^ = D G D) or, for
    one block, bem_gemm; the inverse of G^ (slightly shifted, see below) by
    bem_chol_inverse gives the inverse iteration's operator, applied by two
    bem_gemm products per block.  A block Krylov space of G^{-1} (block size
    `block`) is grown until the smallest Ritz
    value changes by less than `tol` (relative) between two sizes, at most
    `maxit` blocks; sigma_max^2 likewise from the Krylov space of G
    (`tol_max`)."""
    n = S_blocks[0].shape[1]
    dt, dev = S_blocks[0].dtype, S_blocks[0].device
    G = torch.zeros(n, n, dtype=dt, device=dev)
    d = torch.ones(n, dtype=torch.float64, device=dev)
    if len(S_blocks) == 2 and S_blocks[0].shape[0] == n and S_blocks[1].shape[0] == n:
        engine.gram(S_blocks[0], S_blocks[1], G, d, tensor_cores=False)
    else:
        for B in S_blocks:
            engine.gemm(B, B, G, conj_a=True)
    gen = torch.Generator(device=dev).manual_seed(seed)
    p = min(block, n)
    X = torch.randn(n, p, dtype=torch.float64, device=dev, generator=gen)
    if dt.is_complex:
        X = torch.complex(X, torch.randn(n, p, dtype=torch.float64, device=dev, generator=gen))
    dcol = d.to(dt).view(n, 1)
    nmax = max(1, min(maxit, n // p))

    def apply_g(V):
        # G V = D^{-1} G^ D^{-1} V
        Y = torch.zeros_like(V)
        engine.gemm(G, (V / dcol).contiguous(), Y)
        return Y / dcol

    lam_max, _ = _krylov_ritz(engine, S_blocks, apply_g, X, nmax, -1, tol_max, seed + 10)

    # The inverse iteration's operator: (G^ + s I)^{-1} = L^{-H} L^{-1} by the
    # FP64 Cholesky and triangular inverse (bem_chol_inverse), with the
    # smallest relative shift s of SHIFTS at which the factorisation succeeds
    # (s = 0 when G^ is numerically positive definite), starting at
    # info["shift_index"] when given (a sweep passes the previous k's).  G^ is
    # formed with rounding errors of about 1e-14 of its diagonal, and any FP64
    # factorisation of it resolves eigenvalues only down to that level (an
    # LU's backward error acts as the same perturbation); the Ritz values
    # come from S itself, so the shift steers the subspace and does not enter
    # them.
    dmax = float(torch.diagonal(G).real.max()) if dt.is_complex else float(torch.diagonal(G).max())
    Linv = None
    start = int(info.get("shift_index", 0)) if info is not None else 0
    for si in range(max(0, min(start, len(SHIFTS) - 1)), len(SHIFTS)):
        H = G.clone()
        if SHIFTS[si] > 0:
            H.diagonal().add_(SHIFTS[si] * dmax)
        Linv, cinfo = engine.chol_inverse(H)
        del H
        if int(cinfo.item()) == 0:
            if info is not None:
                info["shift_index"] = si
            break
        Linv = None
    if Linv is None:
        return 0.0, math.sqrt(max(lam_max, 0.0)), 0

    def solve(V):
        # G^{-1} V ~ D (G^ + s I)^{-1} D V = D L^{-H} (L^{-1} (D V))
        T1 = torch.zeros_like(V)
        engine.gemm(Linv, (V * dcol).contiguous(), T1, a_lower=True)
        Y = torch.zeros_like(V)
        engine.gemm(Linv, T1, Y, conj_a=True)
        return Y * dcol

    lam_min, nb_min = _krylov_ritz(engine, S_blocks, solve, X, nmax, 0, tol, seed + 20)
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
    n = bm._mat_A.shape[0]
    if not augmented:
        return bm._mat_A.clone()
    At = torch.empty(2 * n, n, dtype=bm._mat_A.dtype, device=bm._mat_A.device)
    At[:n].copy_(bm._mat_A)
    bm._mat_A.zero_()
    bm.assemble_matA(assemble_type=int(AssembleType.ADD_P_PLUS), multiplier=1.0)
    At[n:].copy_(bm._mat_A)
    return At


def transmission_operators(bm, ks, A_type: int = 1):
    """[A(k); P^+_i(k)] (2n x n, new tensors) for every k of `ks`, equal to
    transmission_operator(bm, k, A_type, augmented=True) up to the order of
    the floating-point sums, with the operators of all wavenumbers assembled
    together: per operator (V, K with its -K^T block, W) ONE bem_assemble_batch
    call over the 2 len(ks) wavenumbers k sqrt(n_o) (into A) and k sqrt(n_i)
    (into P), each separate panel pair's geometry evaluated once per launch.
    With M(m) the block operator matA_add_M(m) places (BEM_manager.py:608-628),
    linear in m:
        P = M_int(+1) + 1/2 Id,   A = M_ext(-1) + m_A M_int(+1) + (1 + m_A)/2 Id,
    m_A = -1 for A_I (A_type 1) and +1 for A_II (A_type 2), which is what the
    reference's get_augment_mat_A{1,2}_inv_norm sequence (ADD_P_MINUS(1) at
    the exterior wavenumber, ADD_P_PLUS(m_A) at the interior one, then
    ADD_P_PLUS(1) for the appended block; BEM_manager.py:922-988) builds."""
    from ..BEM_functions.layers import _D, _N
    from .. import _lib as L
    n = bm.N_Neumann + bm.M_Dirichlet
    N, M = bm.N_Neumann, bm.M_Dirichlet
    No, Do = bm._Neumann_offset_i, bm._Dirichlet_offset_i
    m_A = -1.0 if A_type == 1 else 1.0
    Qn, Qd = bm.shape_func_degree_Neumann, bm.shape_func_degree_Dirichlet
    outs = []
    for _ in ks:
        outs.append(torch.zeros(2 * n, n, dtype=torch.complex128, device=bm.device))
    A = [o[:n] for o in outs]
    P = [o[n:] for o in outs]
    # wavenumber list: (exterior of k_0, interior of k_0, exterior of k_1, ...)
    wk, wk2, tgt, sgn = [], [], [], []
    for i, k in enumerate(ks):
        for sqrt_n, X, m in ((bm._sqrt_no, A[i], -1.0), (bm._sqrt_ni, P[i], 1.0)):
            d = bm.op_desc(L.OP_V, float(k), sqrt_n)
            wk.append(d.k)
            wk2.append(d.k2)
            tgt.append(X)
            sgn.append(m)
    desc = lambda op: bm.op_desc(op, float(ks[0]), bm._sqrt_no)  # kernel, precision, quirk
    if N > 0:
        sp = bm.space("charge", Qn, "N", _N, offset=No)
        bm.engine.assemble_batch(desc(L.OP_V), sp, sp, wk, wk2, tgt, [-m for m in sgn])
    if N > 0 and M > 0:
        test = bm.space("charge", Qn, "N", _N, offset=No)
        trial = bm.space("charge", Qd, "D", _D, offset=Do)
        bm.engine.assemble_batch(desc(L.OP_K), test, trial, wk, wk2, tgt, list(sgn), outs_t=tgt,
                                 scales_t=[-m for m in sgn])
    if M > 0:
        sp = bm.space("charge", Qd, "D", _D, offset=Do)
        bm.engine.assemble_batch(desc(L.OP_W), sp, sp, wk, wk2, tgt, [-m for m in sgn])
    if bm._is_transmission:
        test = bm.space("charge", Qn, "N", _N, offset=No)
        trial = bm.space("charge", Qd, "D", _D, offset=Do)
    for i in range(len(ks)):
        A[i].add_(P[i], alpha=m_A)
        if bm._is_transmission:
            bm.engine.mass(test, trial, out=P[i], scale=0.5, out_t=P[i], scale_t=0.5)
            if m_A != -1.0:
                bm.engine.mass(test, trial, out=A[i], scale=0.5 * (1.0 + m_A), out_t=A[i], scale_t=0.5 * (1.0 + m_A))
    return outs


def wavenumber_sweep(bm, ks, nrhs: int = 4, seed: int = 0, A_type: int = 1, scaling_k: float = 0.0,
                     norm_method: str = "iterative", norm_tol: float | None = None, norm_maxit: int | None = None,
                     k_batch: int = 4):
    """For each k in `ks`: the augmented transmission operator [A(k); P^+_i(k)]
    (get_augment_mat_A{1,2}_inv_norm, BEM_manager.py:952-988), the inverse
    norm and condition number of its energy-scaled form, and the
    least-squares solutions of [A; P^+_i] x = [b; 0] for `nrhs` seed-fixed
    complex Gaussian right-hand sides b, by the manager's least-squares
    solver (normal matrix, Cholesky, flexible GMRES in FP64; tensor cores in
    mixed precision, DMMA on the plain path), one factorisation per k.

    The operators of `k_batch` consecutive wavenumbers are assembled together
    (transmission_operators: one k-batched launch per operator and pair of
    wavenumbers); k_batch <= 1 assembles each k on its own
    (transmission_operator).  The energy scaling is formed once, at
    `scaling_k` (the reference forms it on its first call, which the
    reference's sweep makes at k = 0).  norm_tol and norm_maxit override the
    manager's estimator settings for the sweep."""
    n = bm.N_Neumann + bm.M_Dirichlet
    if norm_tol is not None:
        bm.norm_tol = norm_tol
    if norm_maxit is not None:
        bm.norm_maxit = norm_maxit
    bm._L1_inv = bm._L2_inv = None
    if A_type == 1:
        bm.get_mat_A1_inv_norm(scaling_k, method="none")
    else:
        bm.get_mat_A2_inv_norm(scaling_k, method="none")
    gen = torch.Generator(device=bm.device).manual_seed(seed)
    out = {"k": [], "inv_norm": [], "cond": [], "solutions": [], "rhs": [], "ms": [], "iterations": [],
           "phase_ms": []}
    ks = [float(k) for k in ks]
    step = max(1, int(k_batch))
    for g0 in range(0, len(ks), step):
        group = ks[g0:g0 + step]
        torch.cuda.synchronize(bm.device)
        ta = time.perf_counter()
        if step > 1:
            ops = transmission_operators(bm, group, A_type)
        else:
            ops = [transmission_operator(bm, group[0], A_type, augmented=True)]
        torch.cuda.synchronize(bm.device)
        t_asm = (time.perf_counter() - ta) * 1e3 / len(group)
        for k, At in zip(group, ops):
            t1 = time.perf_counter()
            inv_norm, cond, its = bm.compute_inv_norm(At, A_type, method=norm_method, return_cond=True)
            torch.cuda.synchronize(bm.device)
            t2 = time.perf_counter()
            B = torch.zeros(2 * n, nrhs, dtype=torch.complex128, device=bm.device)
            B[:n] = torch.complex(torch.randn(n, nrhs, dtype=torch.float64, device=bm.device, generator=gen),
                                  torch.randn(n, nrhs, dtype=torch.float64, device=bm.device, generator=gen))
            X = bm.lstsq_multi(At[:n], At[n:], B)
            torch.cuda.synchronize(bm.device)
            t3 = time.perf_counter()
            out["ms"].append(t_asm + (t3 - t1) * 1e3)
            out["phase_ms"].append({"assemble": t_asm, "norm": (t2 - t1) * 1e3, "lstsq": (t3 - t2) * 1e3})
            out["k"].append(k)
            out["inv_norm"].append(inv_norm)
            out["cond"].append(cond)
            out["iterations"].append(its)
            out["solutions"].append(X)
            out["rhs"].append(B[:n])
        del ops
    return out
