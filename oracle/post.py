"""Oracle (TEST INFRASTRUCTURE): CPU restatement of the reference's GUI
post-processing kernels, the last two steps of ``BEMManager.run``
(src/managers/BEM_manager.py:1028-1029).

* ``compute_color``       src/managers/BEM_manager.py:527-587
* ``set_mesh_instances``  src/managers/BEM_manager.py:589-606

Plain numpy, FP64 for the traces and float32 for the colour and position
buffers (the reference's fields are ``ti.f32``, BEM_manager.py:133-138; its
default float type is f32, so ``x -= 2.2`` runs in f32).  Only tests/ use this
module, as the checker; the product never imports it.  Pinned by
tests/test_oracle_golden.py against the reference's own kernels run on the
fixtures (tests/golden/gen_golden.py).
"""
from __future__ import annotations

import numpy as np

V_DIRICHLET = 1  # VertAttachType.DIRICHLET_TOBESOLVED (src/BEM_functions/utils/types.py)


def _as_vec(a):
    """[nv] real/complex or [nv, n] reference layout -> complex [nv]."""
    a = np.asarray(a)
    if a.ndim == 2:
        return a[:, 0] + 1j * a[:, 1] if a.shape[1] == 2 else a[:, 0].astype(np.complex128)
    return a.astype(np.complex128)


def _norm(z):
    # ti.Vector.norm: sqrt(x^2 + y^2), each operation rounded
    return np.sqrt(z.real * z.real + z.imag * z.imag)


def compute_color(solved, exact, vert_types, show):
    """Returns (shifted solved [nv] complex, solved colour, exact colour,
    difference colour), colours [nv, 3] float32.

    BEM_manager.py:543-553: the largest |exact| over vertices that are not
    Dirichlet-to-be-solved (max_N), and over those that are (max_D), both
    starting at -5e11; the count and the sums of solved and exact over the
    Dirichlet-to-be-solved vertices.
    :554-556: means, when the count is positive.
    :558-561: solved += mean(exact) - mean(solved) at Dirichlet-to-be-solved
    vertices, or everywhere when show is Dirichlet.
    :562-583: colour = |value| / max in the red channel when Re(value) > 0,
    else in the blue one; max_N for vertices that are not Dirichlet-to-be-
    solved when show is not Dirichlet, max_D otherwise.
    :585-587: green of the difference = |s.r - a.r - s.b + a.b| in f32.
    """
    s = _as_vec(solved).copy()
    a = _as_vec(exact)
    vt = np.asarray(vert_types).astype(np.int64)
    isd = vt == V_DIRICHLET
    na = _norm(a)
    max_n = max([-5e11] + list(na[~isd]))
    max_d = max([-5e11] + list(na[isd]))
    cnt = int(isd.sum())
    mean_s = s[isd].sum() if cnt else 0.0
    mean_a = a[isd].sum() if cnt else 0.0
    if cnt > 0:
        mean_s = mean_s / cnt
        mean_a = mean_a / cnt
    shift = isd | (show == V_DIRICHLET)
    s[shift] = s[shift] + (mean_a - mean_s)
    m = np.where(~isd & (show != V_DIRICHLET), max_n, max_d)
    ca = (na / m).astype(np.float32)
    cs = (_norm(s) / m).astype(np.float32)
    nv = len(s)
    sc = np.zeros((nv, 3), np.float32)
    ac = np.zeros((nv, 3), np.float32)
    dc = np.zeros((nv, 3), np.float32)
    pa, ps = a.real > 0, s.real > 0
    ac[pa, 0] = ca[pa]
    ac[~pa, 2] = ca[~pa]
    sc[ps, 0] = cs[ps]
    sc[~ps, 2] = cs[~ps]
    dc[:, 1] = np.abs(((sc[:, 0] - ac[:, 0]) - sc[:, 2]) + ac[:, 2])
    return s, sc, ac, dc


def set_mesh_instances(vertices):
    """(solved, exact, difference) positions [nv, 3] float32: the vertex
    (first dim coordinates, z = 0 on a 2D mesh), exact at x - 2.2, difference
    at x + 2.2 (BEM_manager.py:591-606)."""
    v = np.asarray(vertices, dtype=np.float64)
    p = np.zeros((v.shape[0], 3), np.float32)
    p[:, :v.shape[1]] = v.astype(np.float32)
    a = p.copy()
    d = p.copy()
    a[:, 0] = p[:, 0] - np.float32(2.2)
    d[:, 0] = p[:, 0] + np.float32(2.2)
    return p, a, d
