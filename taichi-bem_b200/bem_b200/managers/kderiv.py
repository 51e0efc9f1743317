"""dJ/dk of the Helmholtz transmission problem through the adjoint, with the
operators' k-derivative assembled by this library's kernels.

The reference has no derivatives; the operators differentiated are its
single/double/adjoint-double/hypersingular layers (single_layer_3d.py:55-369
and the kernel functions of BEM_manager.py:476-517) in the block system
of BEM_manager.py:990-1006.  Here d/dk is taken analytically:

  * the kernels' k-derivative at fixed k2 (bem_assemble with deriv_k:
    dG/dk = i e^{ikr} / (4 pi) for V and W, k (d.n) e^{ikr} / (4 pi r) for K
    and K'), the quadrature recomputed with the assembly's rules (separate
    pairs by the tensor Gauss rule, coincident / edge / vertex pairs by the
    Sauter-Schwab rules in FP64: the derivative kernels are bounded, so the
    same points integrate them);
  * the W mass term's coefficient k2 = (k sqrt_n)^2 through dW/dk2, the
    difference of two W assemblies at k2 = 1 and k2 = 0 (W is affine in k2);
  * the chain rule of the transmission kernel's wavenumber k sqrt_n;
  * the boundary data's derivative from the data object's analytic
    dfD_dk / dfN_dk (workloads.PlaneWave).

J(k) = ||x(k)||^2.  For the square system A x = b (solver "square"):
    A^H lam = x,   dJ/dk = 2 Re lam^H (db - dA x);
for the reference's least squares min ||S x - c||, S = [A; P+_i],
c = [b; 0] (solver "lstsq"): with N = S^H S, r = c - S x and lam = N^{-1} x
(the same Cholesky and FP64 flexible GMRES as the solve),
    dJ/dk = 2 Re [ (dS lam)^H r + (S lam)^H (dc - dS x) ].
"""
from __future__ import annotations

import time

import torch

from ..utils.types import KernelType, ScopeType


def k_derivative_M(bm, k: float, sqrt_n: float, scope_type: int, out: torch.Tensor, multiplier: float = 1.0):
    """out += multiplier * dM/dk for the block operator
    M = [K, -V; -W, -K^T] that matA_add_M adds (BEM_manager.py:630-645) at
    wavenumber k scaled by sqrt_n.  The manager's layer matrices are
    overwritten (they hold derivative layers afterwards)."""
    uses_n = bm._kernel_type == int(KernelType.HELMHOLTZ_TRANSMISSION)
    dkappa = sqrt_n if uses_n else 1.0   # d(kernel wavenumber)/dk
    dk2 = 2.0 * k * sqrt_n * sqrt_n      # d(k2)/dk
    saved = bm._mat_A
    bm._mat_A = out
    try:
        bm._desc_deriv_k = True
        bm.matrix_layer_forward(k=k, sqrt_n=sqrt_n, scope_type=scope_type)
        bm._desc_deriv_k = False
        bm.matA_add_M(multiplier * dkappa)
        if bm.M_Dirichlet > 0:
            W = bm.hypersingular_layer
            bm._desc_k2 = 1.0
            W.forward(scope_type, k, sqrt_n)
            dW = W._Wmat.clone()
            bm._desc_k2 = 0.0
            W.forward(scope_type, k, sqrt_n)
            dW -= W._Wmat  # dW/dk2
            Do, M = bm._Dirichlet_offset_i, bm.M_Dirichlet
            out[Do:Do + M, Do:Do + M].add_(dW, alpha=-multiplier * dk2)  # M's DD block is -W
    finally:
        bm._desc_deriv_k = False
        bm._desc_k2 = None
        bm._mat_A = saved


def k_derivative_M_media(bm, k: float, parts):
    """For each (sqrt_n, out, multiplier) of `parts` (the exterior and the
    interior medium): out += multiplier * dM/dk as k_derivative_M adds it,
    with every operator of all media assembled together by bem_assemble_batch
    (one call per operator; the separate pairs' geometry shared by the media's
    wavenumbers): the kernels' k-derivatives of V, K (with -K^T) and W at the
    media's wavenumbers, and dW/dk2 as W(k2 = 1) - W(k2 = 0) at each medium's
    wavenumber (two batched terms of opposite sign into the same block)."""
    from .. import _lib as L
    from ..BEM_functions.layers import _D, _N
    uses_n = bm._kernel_type == int(KernelType.HELMHOLTZ_TRANSMISSION)
    N, M = bm.N_Neumann, bm.M_Dirichlet
    No, Do = bm._Neumann_offset_i, bm._Dirichlet_offset_i
    Qn, Qd = bm.shape_func_degree_Neumann, bm.shape_func_degree_Dirichlet
    kap, k2s, outs, m = [], [], [], []
    dk2 = []
    for sqrt_n, out, mult in parts:
        d = bm.op_desc(L.OP_V, k, sqrt_n)
        kap.append(d.k)
        k2s.append(d.k2)
        outs.append(out)
        m.append(mult * (sqrt_n if uses_n else 1.0))  # multiplier x d(kernel wavenumber)/dk
        dk2.append(mult * 2.0 * k * sqrt_n * sqrt_n)   # multiplier x d(k2)/dk
    bm._desc_deriv_k = True
    try:
        desc = lambda op: bm.op_desc(op, k, parts[0][0])  # kernel, precision, quirk, deriv_k
        if N > 0:
            sp = bm.space("charge", Qn, "N", _N, offset=No)
            bm.engine.assemble_batch(desc(L.OP_V), sp, sp, kap, k2s, outs, [-x for x in m])
        if N > 0 and M > 0:
            test = bm.space("charge", Qn, "N", _N, offset=No)
            trial = bm.space("charge", Qd, "D", _D, offset=Do)
            bm.engine.assemble_batch(desc(L.OP_K), test, trial, kap, k2s, outs, list(m), outs_t=outs,
                                     scales_t=[-x for x in m])
        if M > 0:
            sp = bm.space("charge", Qd, "D", _D, offset=Do)
            bm.engine.assemble_batch(desc(L.OP_W), sp, sp, kap, k2s, outs, [-x for x in m])
    finally:
        bm._desc_deriv_k = False
    if M > 0:
        sp = bm.space("charge", Qd, "D", _D, offset=Do)
        kk, kk2, oo, sc = [], [], [], []
        for w, out in enumerate(outs):
            # M's DD block is -W: out_DD += -dk2 (W(1) - W(0))
            kk += [kap[w], kap[w]]
            kk2 += [1.0, 0.0]
            oo += [out, out]
            sc += [-dk2[w], dk2[w]]
        bm.engine.assemble_batch(desc_plain(bm, L.OP_W, k, parts[0][0]), sp, sp, kk, kk2, oo, sc)


def desc_plain(bm, op, k, sqrt_n):
    """The manager's operator descriptor without the k-derivative."""
    saved = bm._desc_deriv_k
    bm._desc_deriv_k = False
    try:
        return bm.op_desc(op, k, sqrt_n)
    finally:
        bm._desc_deriv_k = saved


def _data_k_derivative(bm, data):
    """d f / dk of the transmission data vector f (rhs_constructor's
    _f_boundary) from the data object's analytic derivatives; f itself is
    restored."""
    rc = bm.rhs_constructor
    fD, fN = rc.analytical_function_Dirichlet, rc.analytical_function_Neumann
    try:
        rc.analytical_function_Dirichlet, rc.analytical_function_Neumann = data.dfD_dk, data.dfN_dk
        rc.set_boundaries(scope_type=int(ScopeType.INTERIOR), sqrt_ni=bm._sqrt_ni, sqrt_no=bm._sqrt_no)
        df = rc._f_boundary.clone()
    finally:
        rc.analytical_function_Dirichlet, rc.analytical_function_Neumann = fD, fN
        rc.set_boundaries(scope_type=int(ScopeType.INTERIOR), sqrt_ni=bm._sqrt_ni, sqrt_no=bm._sqrt_no)
    return df


def _gemv(bm, A, x, y=None, alpha=1.0, beta=0.0):
    if y is None:
        y = torch.zeros(A.shape[0], dtype=x.dtype, device=x.device)
    bm.engine.gemv(A, x.contiguous(), y, alpha=alpha, beta=beta)
    return y


def _system(bm, data, k):
    bm._k = k
    if data is not None:
        data.k = k
    bm.assemble_system()
    n = bm.N_Neumann + bm.M_Dirichlet
    A, P = bm.transmission_blocks()
    return A.clone(), P.clone(), bm.rhs[:n].clone()


def _solve(bm, A, P, b):
    n = A.shape[0]
    if bm.solver == "lstsq":
        c = torch.zeros(2 * n, dtype=b.dtype, device=b.device)
        c[:n] = b
        return bm.lstsq_multi(A, P, c.view(-1, 1), keep_factor=True)[:, 0]
    return bm._lu_solve_square(A, b)


def _J(bm, data, k):
    A, P, b = _system(bm, data, k)
    x = _solve(bm, A, P, b)
    bm._lstsq_factor = None
    return float(torch.vdot(x, x).real)


def solution_norm_k_gradient(bm, data, check: bool = True, delta: float = 1e-3):
    """J(k) = ||x(k)||^2 of the manager's transmission problem at its k and
    dJ/dk by the adjoint with the analytic operator derivative (module
    docstring).  `data` is the boundary-data object (workloads.PlaneWave)
    whose k follows the operator's.  With `check`, also the fourth-order
    central difference of J itself (four more assemblies and solves at
    k +- delta, k +- 2 delta).  Returns a dict with J, dJdk, the timings
    and the check."""
    if not bm._is_transmission or bm._n != 2:
        raise ValueError("dJ/dk is built for the Helmholtz transmission problem")
    n = bm.N_Neumann + bm.M_Dirichlet
    k0 = float(bm._k)
    out = {"solver": bm.solver}
    torch.cuda.synchronize(bm.device)
    t0 = time.perf_counter()
    A, P, b = _system(bm, data, k0)
    f = bm.rhs_constructor._f_boundary.clone()
    x = _solve(bm, A, P, b)
    torch.cuda.synchronize(bm.device)
    t1 = time.perf_counter()
    out["solve_ms"] = (t1 - t0) * 1e3
    # the adjoint solve with the solve's factor, which is then released
    if bm.solver == "lstsq":
        lam = bm.normal_solve(x)
        bm._lstsq_factor = None
    else:
        lam = bm._lu_solve_square(A.conj().transpose(0, 1).contiguous(), x.contiguous())
    torch.cuda.synchronize(bm.device)
    t1a = time.perf_counter()
    # the operators' derivatives: dP-_o = -dM_o (exterior), dP+_i = dM_i (interior)
    dPm = torch.zeros(n, n, dtype=A.dtype, device=A.device)
    dP = torch.zeros_like(dPm)
    k_derivative_M_media(bm, k0, [(bm._sqrt_no, dPm, -1.0), (bm._sqrt_ni, dP, 1.0)])
    # b = P-_o conj(f) (the reference's rhs, BEM_manager.py:647-662), P-_o = A - P
    df = _data_k_derivative(bm, data)
    fc = f.conj().resolve_conj() if bm.conj_data else f
    dfc = df.conj().resolve_conj() if bm.conj_data else df
    db = _gemv(bm, dPm, fc)
    _gemv(bm, A, dfc, db, beta=1.0)
    _gemv(bm, P, dfc, db, alpha=-1.0, beta=1.0)
    dA = dPm
    dA += dP
    torch.cuda.synchronize(bm.device)
    t2 = time.perf_counter()
    if bm.solver == "lstsq":
        r_top = _gemv(bm, A, x, b.clone(), alpha=-1.0, beta=1.0)
        r_bot = _gemv(bm, P, x, alpha=-1.0)
        e_top = _gemv(bm, dA, x, db.clone(), alpha=-1.0, beta=1.0)   # dc - dS x (top)
        e_bot = _gemv(bm, dP, x, alpha=-1.0)                         # (bottom)
        dJ = 2.0 * float((torch.vdot(_gemv(bm, dA, lam), r_top) + torch.vdot(_gemv(bm, dP, lam), r_bot)
                          + torch.vdot(_gemv(bm, A, lam), e_top) + torch.vdot(_gemv(bm, P, lam), e_bot)).real)
    else:
        e = _gemv(bm, dA, x, db.clone(), alpha=-1.0, beta=1.0)
        dJ = 2.0 * float(torch.vdot(lam, e).real)
    torch.cuda.synchronize(bm.device)
    t3 = time.perf_counter()
    out.update(J=float(torch.vdot(x, x).real), dJdk=dJ, x=x, adjoint_solve_ms=(t1a - t1) * 1e3,
               derivative_assembly_ms=(t2 - t1a) * 1e3, contraction_ms=(t3 - t2) * 1e3,
               solve_info=dict(bm.solve_info))
    del dA, dP, A, P
    if check:
        Js = {s: _J(bm, data, k0 + s * delta) for s in (-2, -1, 1, 2)}
        out["dJdk_central_difference"] = (Js[-2] - 8.0 * Js[-1] + 8.0 * Js[1] - Js[2]) / (12.0 * delta)
        # the second-order differences at delta and 2 delta: their spread shows
        # the truncation error of the fourth-order one
        out["central_difference"] = {"delta": delta, "order": 4,
                                     "order2_delta": (Js[1] - Js[-1]) / (2.0 * delta),
                                     "order2_2delta": (Js[2] - Js[-2]) / (4.0 * delta)}
    bm._k = k0
    data.k = k0
    return out
