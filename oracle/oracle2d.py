"""Oracle (TEST INFRASTRUCTURE): numpy restatement of the reference's 2D
operators on line-segment panels.

Follows, point for point:

* integrate_on_two_panels   src/BEM_functions/single_layer/single_layer_2d.py:56-215
                            (double_layer_2d.py, adj_double_layer_2d.py and
                            hypersingular_layer_2d.py:62-251 differ only in the integrand)
* G, grad_G_y (2D)          src/managers/BEM_manager.py:451-525
* shape functions, map      src/managers/BEM_manager.py:404-449
* single-panel mass         src/BEM_functions/identity_layer/identity_layer_2d.py:45-116,
                            src/BEM_functions/rhs_constructor/rhs_constructor_2d.py:185-230

Quadrature: Q x Q Gauss points, x(r) = (1 - r) x1 + r x2, weight
w_x w_y L_x L_y; for a panel with itself the Duffy triangles
(r_x, r_y) = (xsi, xsi eta) and (xsi eta, xsi), each with Jacobian xsi.  The
Hankel functions come from scipy.special (the reference calls
``scipy.special.h1vp``).  Only tests/, the smoke check and bench.py's CPU leg
use this module.
"""
from __future__ import annotations

import numpy as np
from scipy import special

INV2PI = 1.0 / (2.0 * np.pi)
OP_V, OP_K, OP_KP, OP_W = 0, 1, 2, 3


def gauss01(Q: int):
    """The Gauss-Legendre rule on [0, 1] of the 3D oracle (the reference's tables)."""
    from .oracle import gauss
    return gauss(Q)


def geometry(verts, segs):
    """Lengths and normals (e.y, -e.x)/|e| (mesh_manager.py:108-113)."""
    v = np.asarray(verts, np.float64)
    f = np.asarray(segs, np.int64)
    e = v[f[:, 1]] - v[f[:, 0]]
    L = np.linalg.norm(e, axis=1)
    n = np.stack([e[:, 1], -e[:, 0]], axis=1)
    n = n / np.linalg.norm(n, axis=1)[:, None]
    return L, n


def _hat(nb, r, b):
    if nb == 1:
        return np.ones_like(r)
    return 1.0 - r if b == 0 else r


def _block(verts, segs, op, helm, k, k2, Q, gi, gj, nbx, nby, coincide):
    """Integrals for the panel pairs (gi[m], gj[m]) -> [m, nbx, nby]."""
    v = np.asarray(verts, np.float64)
    f = np.asarray(segs, np.int64)
    L, nrm = geometry(v, f)
    gp, gw = gauss01(Q)
    x1, x2 = v[f[gi, 0]], v[f[gi, 1]]
    y1, y2 = v[f[gj, 0]], v[f[gj, 1]]
    Lx, Ly = L[gi], L[gj]
    nx, ny = nrm[gi], nrm[gj]
    nn = (nx * ny).sum(1)
    cx = [np.zeros_like(Lx)] if nbx == 1 else [-1.0 / Lx, 1.0 / Lx]
    cy = [np.zeros_like(Ly)] if nby == 1 else [-1.0 / Ly, 1.0 / Ly]
    out = np.zeros((len(gi), nbx, nby), np.complex128 if helm else np.float64)

    def add(rx, ry, w):
        px = (1.0 - rx)[:, None] * x1 + rx[:, None] * x2
        py = (1.0 - ry)[:, None] * y1 + ry[:, None] * y2
        d = px - py
        r = np.linalg.norm(d, axis=1)
        if op in (OP_V, OP_W):
            g = 0.25j * special.hankel1(0, k * r) if helm else INV2PI * np.log(1.0 / r)
        else:
            dn = (d * ny).sum(1) / r if op == OP_K else (-d * nx).sum(1) / r
            # (i/4) H0'(kr) k (-d^.n) with H0' = -H1
            g = 0.25j * special.hankel1(1, k * r) * k * dn if helm else INV2PI * dn / r
        for a in range(nbx):
            for b in range(nby):
                c = _hat(nbx, rx, a) * _hat(nby, ry, b)
                if op == OP_W:
                    c = cx[a] * cy[b] - k2 * c * nn
                out[:, a, b] += g * c * w * Lx * Ly

    one = np.ones(len(gi))
    for ix in range(Q):
        for iy in range(Q):
            w = gw[ix] * gw[iy]
            if not coincide:
                add(gp[ix] * one, gp[iy] * one, w)
            else:
                xsi, eta = gp[ix], gp[iy]
                add(xsi * one, xsi * eta * one, w * xsi)
                add(xsi * eta * one, xsi * one, w * xsi)
    return out


def assemble(verts, segs, op, helm, k, k2, Q, test, trial, out=None, out_t=None, scale=1.0, scale_t=1.0,
             x=None, y=None, conj_x=False):
    """Same contract as oracle.assemble for a segment mesh: test/trial =
    (panels, nb, dof[n*nb]); dense (out, out_t) or apply (x -> y)."""
    tp, nbx, tdof = test
    rp, nby, rdof = trial
    tp = np.asarray(tp, np.int64)
    rp = np.asarray(rp, np.int64)
    tdof = np.asarray(tdof, np.int64).reshape(len(tp), nbx)
    rdof = np.asarray(rdof, np.int64).reshape(len(rp), nby)
    if len(tp) == 0 or len(rp) == 0:
        return
    I, J = np.meshgrid(np.arange(len(tp)), np.arange(len(rp)), indexing="ij")
    I, J = I.reshape(-1), J.reshape(-1)
    gi, gj = tp[I], rp[J]
    blk = np.zeros((len(I), nbx, nby), np.complex128 if helm else np.float64)
    same = gi == gj
    if (~same).any():
        blk[~same] = _block(verts, segs, op, helm, k, k2, Q, gi[~same], gj[~same], nbx, nby, False)
    if same.any():
        blk[same] = _block(verts, segs, op, helm, k, k2, Q, gi[same], gj[same], nbx, nby, True)
    for a in range(nbx):
        for b in range(nby):
            row, col = tdof[I, a], rdof[J, b]
            ok = (row >= 0) & (col >= 0)
            val = blk[ok, a, b]
            if x is not None:
                xv = np.asarray(x)[col[ok]]
                if conj_x:
                    xv = np.conj(xv)
                np.add.at(y, row[ok], scale * val * xv)
            else:
                np.add.at(out, (row[ok], col[ok]), scale * val)
                if out_t is not None:
                    np.add.at(out_t, (col[ok], row[ok]), scale_t * val)


def mass(verts, segs, Q, panels, nbx, test_dof, nby, trial_dof, out=None, out_t=None, scale=1.0, scale_t=1.0,
         x=None, y=None, conj_x=False):
    """Single-panel mass L sum_q w_q phi_a phi_b over one panel list."""
    L, _ = geometry(verts, segs)
    gp, gw = gauss01(Q)
    p = np.asarray(panels, np.int64)
    td = np.asarray(test_dof, np.int64).reshape(len(p), nbx)
    rd = np.asarray(trial_dof, np.int64).reshape(len(p), nby)
    for a in range(nbx):
        for b in range(nby):
            m = sum(_hat(nbx, np.array(gp[q]), a) * _hat(nby, np.array(gp[q]), b) * gw[q] for q in range(Q))
            val = float(m) * L[p]
            row, col = td[:, a], rd[:, b]
            ok = (row >= 0) & (col >= 0)
            if x is not None:
                xv = np.asarray(x)[col[ok]]
                if conj_x:
                    xv = np.conj(xv)
                np.add.at(y, row[ok], scale * val[ok] * xv)
            else:
                np.add.at(out, (row[ok], col[ok]), scale * val[ok])
                if out_t is not None:
                    np.add.at(out_t, (col[ok], row[ok]), scale_t * val[ok])
