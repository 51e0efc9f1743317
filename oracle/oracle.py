"""Oracle (TEST INFRASTRUCTURE): CPU restatement of the reference BEM path.

``liboracle.so`` (bem_oracle.c / oracle_core.h) restates the reference's
quadrature kernels; this module wraps it with ctypes and restates the
reference's driver logic in numpy:

* mesh geometry             src/managers/mesh_manager.py:103-139
* BVP partition, DOF maps   src/managers/mesh_manager.py:166-389,415-445
* charge-index projections  src/managers/BEM_manager.py:224-310
* operator forward passes   single/double/hypersingular ``forward``
* RHS construction          src/BEM_functions/rhs_constructor/rhs_constructor_3d.py:50-386
* block assembly / solve    src/managers/BEM_manager.py:608-662,990-1073

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs use it, as
the checker or the timed CPU baseline; the product never imports it.
Parity of this restatement is pinned by tests/test_oracle_golden.py against
fixtures produced by running the reference's own kernels
(tests/golden/gen_golden.py).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

OP_V, OP_K, OP_KP, OP_W = 0, 1, 2, 3
# CellFluxType / VertAttachType / ScopeType (src/BEM_functions/utils/types.py:4-38)
NEUMANN, DIRICHLET, MIX, BOTH = 0, 1, 2, 3
V_NEUMANN, V_DIRICHLET, V_BOTH = 0, 1, 2
INTERIOR, EXTERIOR = 1, 2


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.oracle_gauss.argtypes = [ctypes.c_int, dp, dp]
        L.oracle_relation.argtypes = [ip, ctypes.c_int, ctypes.c_int]
        L.oracle_near_perm.argtypes = [ip, ctypes.c_int, ctypes.c_int, ctypes.c_int, ip, ip]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_assemble.argtypes = [
            ctypes.c_int, dp, ip, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ip, ctypes.c_int, ip, ctypes.c_int, ip, ctypes.c_int, ip,
            ctypes.c_int, ctypes.c_int, dp, ctypes.c_long, ctypes.c_double, dp, ctypes.c_double, dp, dp, ctypes.c_int]
        L.oracle_mass.argtypes = [
            ctypes.c_int, dp, ip, ctypes.c_int, ctypes.c_int, ip, ctypes.c_int, ip, ctypes.c_int, ip, ctypes.c_int,
            ctypes.c_int, dp, ctypes.c_long, ctypes.c_double, dp, ctypes.c_double, dp, dp, ctypes.c_int]
        _LIB = L
    return _LIB


def _dp(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def set_threads(n: int) -> int:
    return lib().oracle_set_threads(int(n))


def gauss(n: int):
    p = np.zeros(n)
    w = np.zeros(n)
    if lib().oracle_gauss(n, _dp(p), _dp(w)) != 0:
        raise ValueError(n)
    return p, w


def relation(tris, i, j) -> int:
    t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1)
    return lib().oracle_relation(_ip(t), int(i), int(j))


def _as_view(a):
    """complex128 -> float64 interleaved view (same memory)."""
    if np.iscomplexobj(a):
        return a.view(np.float64)
    return a


def assemble(verts, tris, op, helm, k, k2, Q, quirk, test, trial, out=None, out_t=None, scale=1.0, scale_t=1.0,
             x=None, y=None, conj_x=False, fp32=False):
    """test/trial = (panels[int32], nb, dof[int32, n*nb]).  Dense mode writes
    ``out`` (+ ``out_t`` transposed); apply mode (x, y given) accumulates
    y[row] += scale * val * x[col]."""
    v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1)
    t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1)
    tp, nbx, tdof = test
    rp, nby, rdof = trial
    tp = np.ascontiguousarray(tp, dtype=np.int32)
    rp = np.ascontiguousarray(rp, dtype=np.int32)
    tdof = np.ascontiguousarray(tdof, dtype=np.int32)
    rdof = np.ascontiguousarray(rdof, dtype=np.int32)
    if x is not None:
        is_c = np.iscomplexobj(y)
        xv = np.ascontiguousarray(x, dtype=np.complex128 if is_c else np.float64)
        rc = lib().oracle_assemble(int(fp32), _dp(v), _ip(t), len(t) // 3, op, int(helm), float(k), float(k2), Q,
                                   int(quirk), len(tp), _ip(tp), nbx, _ip(tdof), len(rp), _ip(rp), nby, _ip(rdof),
                                   int(is_c), 1, None, 0, float(scale), None, 0.0, _dp(_as_view(xv)),
                                   _dp(_as_view(y)), int(conj_x))
    else:
        is_c = np.iscomplexobj(out)
        assert out.flags.c_contiguous
        ld = out.shape[1]
        if out_t is not None:
            assert out_t.shape == out.shape and np.iscomplexobj(out_t) == is_c
        rc = lib().oracle_assemble(int(fp32), _dp(v), _ip(t), len(t) // 3, op, int(helm), float(k), float(k2), Q,
                                   int(quirk), len(tp), _ip(tp), nbx, _ip(tdof), len(rp), _ip(rp), nby, _ip(rdof),
                                   int(is_c), 0, _dp(_as_view(out)), ld, float(scale),
                                   _dp(_as_view(out_t)) if out_t is not None else None, float(scale_t), None, None, 0)
    if rc != 0:
        raise RuntimeError(f"oracle_assemble failed: {rc}")


def mass(verts, tris, Q, panels, nbx, test_dof, nby, trial_dof, out=None, out_t=None, scale=1.0, scale_t=1.0,
         x=None, y=None, conj_x=False):
    v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1)
    t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1)
    p = np.ascontiguousarray(panels, dtype=np.int32)
    td = np.ascontiguousarray(test_dof, dtype=np.int32)
    rd = np.ascontiguousarray(trial_dof, dtype=np.int32)
    if x is not None:
        is_c = np.iscomplexobj(y)
        xv = np.ascontiguousarray(x, dtype=np.complex128 if is_c else np.float64)
        rc = lib().oracle_mass(0, _dp(v), _ip(t), Q, len(p), _ip(p), nbx, _ip(td), nby, _ip(rd), int(is_c), 1, None,
                               0, float(scale), None, 0.0, _dp(_as_view(xv)), _dp(_as_view(y)), int(conj_x))
    else:
        is_c = np.iscomplexobj(out)
        rc = lib().oracle_mass(0, _dp(v), _ip(t), Q, len(p), _ip(p), nbx, _ip(td), nby, _ip(rd), int(is_c), 0,
                               _dp(_as_view(out)), out.shape[1], float(scale),
                               _dp(_as_view(out_t)) if out_t is not None else None, float(scale_t), None, None, 0)
    if rc != 0:
        raise RuntimeError(f"oracle_mass failed: {rc}")


# ---------------------------------------------------------------------------
# Mesh + BVP restatement (mesh_manager.py)
# ---------------------------------------------------------------------------
class Mesh:
    def __init__(self, vertices, panels, boundary="Dirichlet", Q_Neumann=0, Q_Dirichlet=1, transmission=False,
                 dim=3):
        d = self.dim = int(dim)
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float64)
        self.panels = np.ascontiguousarray(panels, dtype=np.int32).reshape(-1, d)
        self.nv = len(self.vertices)
        self.nt = len(self.panels)
        self.Q_N, self.Q_D = int(Q_Neumann), int(Q_Dirichlet)
        v, f = self.vertices, self.panels
        if d == 2:
            # segment length and normal (e.y, -e.x)/|e| (mesh_manager.py:108-113)
            e = v[f[:, 1]] - v[f[:, 0]]
            self.panel_areas = np.linalg.norm(e, axis=1)
            cr = np.stack([e[:, 1], -e[:, 0]], axis=1)
            self.panel_normals = cr / np.linalg.norm(cr, axis=1)[:, None]
        else:
            cr = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 1]])
            nrm = np.linalg.norm(cr, axis=1)
            self.panel_areas = 0.5 * nrm
            self.panel_normals = cr / nrm[:, None]
        self.vert_areas = np.zeros(self.nv)
        self.vert_normals = np.zeros((self.nv, d))
        for i in range(self.nt * d):
            self.vert_areas[f.reshape(-1)[i]] += self.panel_areas[i // d] / float(d)
            self.vert_normals[f.reshape(-1)[i]] += self.panel_normals[i // d]
        self.vert_normals /= np.linalg.norm(self.vert_normals, axis=1)[:, None]
        if boundary == "Full" or transmission:
            self._full()
        elif boundary == "Dirichlet":
            self._dirichlet()
        elif boundary == "Neumann":
            self._neumann()
        elif boundary == "Mix":
            self._mixed()
        else:
            raise RuntimeError("The Boundary Type can only be Dirichlet/Neumann/Mix")

    def _nb(self, n_p, n_v, q):
        return n_p if q == 0 else n_v

    def _full(self):
        self.N_N = self._nb(self.nt, self.nv, self.Q_N)
        self.M_D = self._nb(self.nt, self.nv, self.Q_D)
        self.panel_types = np.full(self.nt, BOTH, np.int32)
        self.vert_types = np.full(self.nv, V_BOTH, np.int32)
        self.D_index = np.arange(self.nt, dtype=np.int32)
        self.N_index = np.arange(self.nt, dtype=np.int32)
        self.map_N = np.arange(self.nv, dtype=np.int32)
        self.map_D = np.arange(self.nv, dtype=np.int32)
        self.nP_D = self.nP_N = self.nt

    def _dirichlet(self):
        self.N_N = self._nb(self.nt, self.nv, self.Q_N)
        self.M_D = 0
        self.panel_types = np.full(self.nt, NEUMANN, np.int32)
        self.vert_types = np.full(self.nv, V_NEUMANN, np.int32)
        self.D_index = np.zeros(0, np.int32)
        self.N_index = np.arange(self.nt, dtype=np.int32)
        self.map_N = np.arange(self.nv, dtype=np.int32)
        self.map_D = np.full(self.nv, -1, np.int32)
        self.nP_D, self.nP_N = 0, self.nt

    def _neumann(self):
        self.N_N = 0
        self.M_D = self._nb(self.nt, self.nv, self.Q_D)
        self.panel_types = np.full(self.nt, DIRICHLET, np.int32)
        self.vert_types = np.full(self.nv, V_DIRICHLET, np.int32)
        self.D_index = np.arange(self.nt, dtype=np.int32)
        self.N_index = np.zeros(0, np.int32)
        self.map_N = np.full(self.nv, -1, np.int32)
        self.map_D = np.arange(self.nv, dtype=np.int32)
        self.nP_D, self.nP_N = self.nt, 0

    def _mixed(self):
        f, v = self.panels, self.vertices
        pt = np.zeros(self.nt, np.int32)
        vt = np.full(self.nv, -1, np.int32)
        mapN = np.full(self.nv, -1, np.int32)
        mapD = np.full(self.nv, -1, np.int32)
        nD = nN = 0
        d = self.dim
        for i in range(self.nt):
            y = sum(v[f[i, j], 1] for j in range(d)) / float(d)
            if y > 0:
                nN += 1
                pt[i] = NEUMANN
            else:
                nD += 1
                pt[i] = DIRICHLET
        nvN = nvD = 0
        for i in range(self.nt):
            if pt[i] == NEUMANN:
                for j in range(d):
                    a = f[i, j]
                    if vt[a] == -1:
                        vt[a] = V_NEUMANN
                        mapN[a] = nvN
                        nvN += 1
        for i in range(self.nt):
            if pt[i] == DIRICHLET:
                for j in range(d):
                    a = f[i, j]
                    if vt[a] == -1:
                        vt[a] = V_DIRICHLET
                        mapD[a] = nvD
                        nvD += 1
        for i in range(self.nt):
            ds = sum(1 for j in range(d) if vt[f[i, j]] == V_DIRICHLET)
            ns = sum(1 for j in range(d) if vt[f[i, j]] == V_NEUMANN)
            t = pt[i]
            if ns == d and t == DIRICHLET:
                pt[i] = NEUMANN
                nD -= 1
                nN += 1
            elif ds == d and t == NEUMANN:
                pt[i] = DIRICHLET
                nD += 1
                nN -= 1
            elif ns != d and ds != d:
                if t == NEUMANN:
                    nN -= 1
                elif t == DIRICHLET:
                    nD -= 1
                pt[i] = MIX
        self.N_N = nN if self.Q_N == 0 else nvN
        self.M_D = nD if self.Q_D == 0 else nvD
        self.panel_types = pt
        self.vert_types = vt
        idx = np.arange(self.nt, dtype=np.int32)
        self.D_index = idx[pt != NEUMANN]
        self.N_index = idx[pt != DIRICHLET]
        self.map_N = mapN
        self.map_D = mapD
        # num_of_panels_Dirichlet/Neumann count only the pure panels while the
        # index lists also hold the MIX panels; the reference's loops run over
        # the first num_of_panels_X entries of the lists (mesh_manager.py:371-384)
        self.nP_D, self.nP_N = nD, nN

    # --- maps (mesh_manager.py:415-445, BEM_manager.py:244-310) -------------
    def local_to_panel(self, side, i):
        if side == "N":
            return int(self.N_index[i]) if self.N_N > 0 else -1
        return int(self.D_index[i]) if self.M_D > 0 else -1

    def vert_local(self, side, v):
        if side == "N":
            if self.N_N > 0 and self.Q_N == 1 and self.vert_types[v] in (V_NEUMANN, V_BOTH):
                return int(self.map_N[v])
            return -1
        if self.M_D > 0 and self.Q_D == 1 and self.vert_types[v] in (V_DIRICHLET, V_BOTH):
            return int(self.map_D[v])
        return -1

    def charge_local(self, Q, local_panel, b, ptype):
        if Q == 0:
            return local_panel if ptype != MIX else -1
        if ptype == NEUMANN:
            gp = self.local_to_panel("N", local_panel)
            gv = int(self.panels[gp, b])
            if self.vert_types[gv] != V_DIRICHLET:
                return self.vert_local("N", gv)
        elif ptype == DIRICHLET:
            gp = self.local_to_panel("D", local_panel)
            gv = int(self.panels[gp, b])
            if self.vert_types[gv] != V_NEUMANN:
                return self.vert_local("D", gv)
        return -1

    def charge_global(self, Q, local_panel, b, ptype):
        gp = -1
        if ptype == NEUMANN:
            gp = self.local_to_panel("N", local_panel)
        elif ptype == DIRICHLET:
            gp = self.local_to_panel("D", local_panel)
        if Q == 0 or gp < 0:
            return gp
        return int(self.panels[gp, b])

    def loop(self, side):
        """Global panels visited by `for local_I in range(num_of_panels_X)`."""
        return self.N_index[:self.nP_N] if side == "N" else self.D_index[:self.nP_D]

    def side(self, side, Q, as_type):
        """(panels, nb, dof) table for one side of a forward() block: the
        local panel loop of that side, with BOTH_TOBESOLVED read as
        ``as_type`` and the charge index of each basis function."""
        idx = self.loop(side)
        nb = 1 if Q == 0 else self.dim
        dof = np.full(len(idx) * nb, -1, np.int32)
        for li, gp in enumerate(idx):
            pt = self.panel_types[gp]
            if pt == BOTH:
                pt = as_type
            for b in range(nb):
                dof[li * nb + b] = self.charge_local(Q, li, b if Q == 1 else -1, pt)
        return np.asarray(idx, np.int32), nb, dof

    def side_global(self, side, Q):
        """(panels, nb, dof) where dof is the index into the boundary-data
        field (P0: global panel, P1: global vertex), used by apply_*_boundary."""
        idx = self.loop(side)
        nb = 1 if Q == 0 else self.dim
        dof = np.zeros(len(idx) * nb, np.int32)
        for li, gp in enumerate(idx):
            for b in range(nb):
                dof[li * nb + b] = gp if Q == 0 else self.panels[gp, b]
        return np.asarray(idx, np.int32), nb, dof


# ---------------------------------------------------------------------------
# Driver restatement (BEMManager.run)
# ---------------------------------------------------------------------------
class Problem:
    """FP64 restatement of BEMManager for one simulation_parameters dict.

    fD(x[m,dim], sqrt_n) and fN(x[m,dim], n[m,dim], sqrt_n) are vectorised
    numpy callables returning real (Laplace) or complex (Helmholtz) arrays.
    params["dim"] = 2 selects the segment-mesh operators (oracle2d).
    quirk=True reproduces the reference bit-for-bit in structure; quirk=False
    uses the corrected near-field orientation/basis and g instead of conj(g).
    """

    def __init__(self, vertices, panels, params, fD, fN, quirk=True):
        p = dict(params)
        self.kernel = p["kernel"]
        self.helm = "Helmholtz" in self.kernel
        self.k = float(p.get("k", 0.0)) if self.helm else 0.0
        self.transmission = ("Full" in p["boundary"]) or ("Transmission" in self.kernel)
        self.kernel_uses_sqrt_n = self.kernel == "Helmholtz_Transmission"
        self.sqrt_ni = float(np.sqrt(p.get("n_i", 1.0))) if self.kernel_uses_sqrt_n else 1.0
        self.sqrt_no = float(np.sqrt(p.get("n_o", 1.0))) if self.kernel_uses_sqrt_n else 1.0
        self.Q = int(p["GaussQR"])
        self.scope = INTERIOR if p.get("scope", "Interior") == "Interior" else EXTERIOR
        self.quirk = quirk
        self.dim = int(p.get("dim", 3))
        self.mesh = Mesh(vertices, panels, p["boundary"], p.get("Q_Neumann", 0), p.get("Q_Dirichlet", 1),
                         self.transmission, dim=self.dim)
        self.fD, self.fN = fD, fN
        m = self.mesh
        self.n = m.N_N + m.M_D
        self.D_off = 0
        self.N_off = m.M_D
        self.dtype = np.complex128 if self.helm else np.float64

    def _assemble(self, verts, panels, op, helm, k, k2, Q, quirk, test, trial, **kw):
        if self.dim == 2:
            from . import oracle2d
            oracle2d.assemble(verts, panels, op, helm, k, k2, Q, test, trial, **kw)
        else:
            assemble(verts, panels, op, helm, k, k2, Q, quirk, test, trial, **kw)

    def _mass(self, verts, panels, Q, *args, **kw):
        if self.dim == 2:
            from . import oracle2d
            oracle2d.mass(verts, panels, Q, *args, **kw)
        else:
            mass(verts, panels, Q, *args, **kw)

    # -- forward (matrix_layer_forward) ----------------------------------------
    def _kk(self, sqrt_n):
        k_kernel = self.k * (sqrt_n if self.kernel_uses_sqrt_n else 1.0)
        k2 = self.k * self.k * sqrt_n * sqrt_n
        return k_kernel, k2

    def forward(self, sqrt_n=1.0):
        m = self.mesh
        k, k2 = self._kk(sqrt_n)
        args = (m.vertices, m.panels)
        out = {}
        if m.N_N > 0:
            V = np.zeros((m.N_N, m.N_N), self.dtype)
            sN = m.side("N", m.Q_N, NEUMANN)
            self._assemble(*args, OP_V, self.helm, k, k2, self.Q, self.quirk, sN, sN, out=V)
            out["V"] = V
        if m.N_N > 0 and m.M_D > 0:
            K = np.zeros((m.N_N, m.M_D), self.dtype)
            self._assemble(*args, OP_K, self.helm, k, k2, self.Q, self.quirk, m.side("N", m.Q_N, NEUMANN),
                           m.side("D", m.Q_D, DIRICHLET), out=K)
            out["K"] = K
        if m.M_D > 0:
            W = np.zeros((m.M_D, m.M_D), self.dtype)
            sD = m.side("D", m.Q_D, DIRICHLET)
            self._assemble(*args, OP_W, self.helm, k, k2, self.Q, self.quirk, sD, sD, out=W)
            out["W"] = W
        return out

    def add_M(self, A, layers, c):
        """matA_add_M (BEM_manager.py:608-628)."""
        m = self.mesh
        No, Do = self.N_off, self.D_off
        if "V" in layers:
            A[No:No + m.N_N, No:No + m.N_N] += -c * layers["V"]
        if "K" in layers:
            A[No:No + m.N_N, Do:Do + m.M_D] += c * layers["K"]
            A[Do:Do + m.M_D, No:No + m.N_N] += -c * layers["K"].T
        if "W" in layers:
            A[Do:Do + m.M_D, Do:Do + m.M_D] += -c * layers["W"]

    def add_identity(self, A, c):
        """IdentityLayer3d.matA_add_global_Identity_matrix (identity_layer_3d.py:148-196)."""
        m = self.mesh
        nbN = 1 if m.Q_N == 0 else self.dim
        nbD = 1 if m.Q_D == 0 else self.dim
        rows = np.zeros(m.nt * nbN, np.int32)
        cols = np.zeros(m.nt * nbD, np.int32)
        panels = np.zeros(m.nt, np.int32)
        for li in range(m.nt):
            panels[li] = m.local_to_panel("D", li)
            for b in range(nbN):
                rows[li * nbN + b] = m.charge_local(m.Q_N, li, b if m.Q_N == 1 else -1, NEUMANN)
            for b in range(nbD):
                cols[li * nbD + b] = m.charge_local(m.Q_D, li, b if m.Q_D == 1 else -1, DIRICHLET)
        # rows are offset by N_off, cols by D_off: build on a view of A
        Ablk = np.zeros((self.n, self.n), self.dtype)
        rows_o = np.where(rows >= 0, rows + self.N_off, -1).astype(np.int32)
        cols_o = np.where(cols >= 0, cols + self.D_off, -1).astype(np.int32)
        self._mass(m.vertices, m.panels, self.Q, panels, nbN, rows_o, nbD, cols_o, out=Ablk, out_t=Ablk, scale=c,
                   scale_t=c)
        A += Ablk

    # -- boundary data (RHSConstructor3d.set_boundaries) -----------------------
    def set_boundaries(self):
        m = self.mesh
        v, f = m.vertices, m.panels
        self.Db = np.zeros(m.nt if m.Q_D == 0 else m.nv, self.dtype)
        self.Nb = np.zeros(m.nt if m.Q_N == 0 else m.nv, self.dtype)
        self.fb = np.zeros(self.n, self.dtype)
        cent = v[f].sum(axis=1) / float(self.dim)
        # exterior normal of the transmission data: n in 3D (get_panel_normal
        # ignores the scope, BEM_manager.py:330-335), -n in 2D
        # (rhs_constructor_2d.py:70,84)
        es = -1.0 if self.dim == 2 else 1.0
        if self.transmission:
            si, so = self.sqrt_ni, self.sqrt_no
            if m.Q_N == 0:
                for li, gp in enumerate(m.loop("N")):
                    x, nrm = cent[gp:gp + 1], m.panel_normals[gp:gp + 1]
                    self.Nb[gp] += self.fN(x, nrm, si)[0]
                    self.fb[self.N_off + li] += self.fN(x, nrm, si)[0] - self.fN(x, es * nrm, so)[0]
            else:
                for gv in range(m.nv):
                    if m.vert_types[gv] in (V_BOTH, V_NEUMANN):
                        lv = m.vert_local("N", gv)
                        x, nrm = v[gv:gv + 1], m.vert_normals[gv:gv + 1]
                        self.Nb[gv] += self.fN(x, nrm, si)[0]
                        self.fb[self.N_off + lv] += self.fN(x, nrm, si)[0] - self.fN(x, es * nrm, so)[0]
            if m.Q_D == 0:
                for li, gp in enumerate(m.loop("D")):
                    x = cent[gp:gp + 1]
                    self.Db[gp] += self.fD(x, si)[0]
                    self.fb[self.D_off + li] += self.fD(x, si)[0] - self.fD(x, so)[0]
            else:
                for gv in range(m.nv):
                    if m.vert_types[gv] in (V_BOTH, V_DIRICHLET):
                        lv = m.vert_local("D", gv)
                        x = v[gv:gv + 1]
                        self.Db[gv] += self.fD(x, si)[0]
                        self.fb[self.D_off + lv] += self.fD(x, si)[0] - self.fD(x, so)[0]
        else:
            if m.Q_N == 0:
                for gp in m.loop("D"):
                    self.Nb[gp] += self.fN(cent[gp:gp + 1], m.panel_normals[gp:gp + 1], 1.0)[0]
            else:
                for gv in range(m.nv):
                    if m.vert_types[gv] == V_DIRICHLET:
                        self.Nb[gv] += self.fN(v[gv:gv + 1], m.vert_normals[gv:gv + 1], 1.0)[0]
            if m.Q_D == 0:
                for gp in m.loop("N"):
                    self.Db[gp] += self.fD(cent[gp:gp + 1], 1.0)[0]
            else:
                for gv in range(m.nv):
                    if m.vert_types[gv] == V_NEUMANN:
                        self.Db[gv] += self.fD(v[gv:gv + 1], 1.0)[0]

    # -- RHS (RHSConstructor3d.forward) -----------------------------------------
    def rhs_forward(self):
        m = self.mesh
        conj = self.quirk and self.helm
        rhs = np.zeros(self.n, self.dtype)
        half = 0.5 if self.scope == INTERIOR else -0.5
        v, f = m.vertices, m.panels
        k, k2 = self._kk(1.0)
        # multiply_identity_to_vector (rhs_constructor_3d.py:256-359)
        if m.N_N > 0:
            panels, nbx, rdof = m.side("N", m.Q_N, NEUMANN)
            nby = 1 if m.Q_D == 0 else self.dim
            cdof = np.zeros(len(panels) * nby, np.int32)
            for li in range(len(panels)):
                pt = m.panel_types[panels[li]]
                pt = NEUMANN if pt == BOTH else pt
                for b in range(nby):
                    cdof[li * nby + b] = m.charge_global(m.Q_D, li, b if m.Q_D == 1 else -1, pt)
            rows = np.where(rdof >= 0, rdof + self.N_off, -1).astype(np.int32)
            cdof = np.where(cdof >= 0, cdof, -1).astype(np.int32)
            self._mass(v, f, self.Q, panels, nbx, rows, nby, cdof, x=self.Db, y=rhs, scale=half, conj_x=conj)
        if m.M_D > 0:
            panels, nbx, rdof = m.side("D", m.Q_D, DIRICHLET)
            nby = 1 if m.Q_N == 0 else self.dim
            cdof = np.zeros(len(panels) * nby, np.int32)
            for li in range(len(panels)):
                pt = m.panel_types[panels[li]]
                pt = DIRICHLET if pt == BOTH else pt
                for b in range(nby):
                    cdof[li * nby + b] = m.charge_global(m.Q_N, li, b if m.Q_N == 1 else -1, pt)
            rows = np.where(rdof >= 0, rdof + self.D_off, -1).astype(np.int32)
            self._mass(v, f, self.Q, panels, nbx, rows, nby, cdof, x=self.Nb, y=rhs, scale=half, conj_x=conj)
        # multiply_M_to_vector (rhs_constructor_3d.py:361-372)
        if m.N_N > 0:
            tp, nbx, tdof = m.side("N", m.Q_N, NEUMANN)
            rows = np.where(tdof >= 0, tdof + self.N_off, -1).astype(np.int32)
            self._assemble(v, f, OP_K, self.helm, k, k2, self.Q, self.quirk, (tp, nbx, rows), m.side_global("N", m.Q_D),
                           x=self.Db, y=rhs, scale=1.0, conj_x=conj)
            if m.nP_D > 0:
                self._assemble(v, f, OP_V, self.helm, k, k2, self.Q, self.quirk, (tp, nbx, rows),
                               m.side_global("D", m.Q_N), x=self.Nb, y=rhs, scale=-1.0, conj_x=conj)
        if m.M_D > 0:
            tp, nbx, tdof = m.side("D", m.Q_D, DIRICHLET)
            rows = np.where(tdof >= 0, tdof + self.D_off, -1).astype(np.int32)
            # the 2D K' product multiplies by f, not conj(f) (adj_double_layer_2d.py:344)
            self._assemble(v, f, OP_KP, self.helm, k, k2, self.Q, self.quirk, (tp, nbx, rows), m.side_global("D", m.Q_N),
                           x=self.Nb, y=rhs, scale=-1.0, conj_x=conj and self.dim == 3)
            if m.nP_N > 0:
                self._assemble(v, f, OP_W, self.helm, k, k2, self.Q, self.quirk, (tp, nbx, rows),
                               m.side_global("N", m.Q_D), x=self.Db, y=rhs, scale=-1.0, conj_x=conj)
        return rhs

    def run(self):
        """BEMManager.run (BEM_manager.py:990-1018) + solve (:1032-1073)."""
        A = np.zeros((self.n, self.n), self.dtype)
        res = {}
        if self.transmission:
            lay_o = self.forward(self.sqrt_no)
            self.add_identity(A, 0.5)
            self.add_M(A, lay_o, -1.0)
            self.set_boundaries()
            fb = np.conj(self.fb) if (self.helm and self.quirk) else self.fb
            rhs = np.concatenate([A @ fb, np.zeros(self.n, self.dtype)])
            lay_i = self.forward(self.sqrt_ni)
            self.add_identity(A, 0.5)
            self.add_M(A, lay_i, 1.0)
            P = np.zeros_like(A)
            self.add_identity(P, 0.5)
            self.add_M(P, lay_i, 1.0)
            sol = np.linalg.lstsq(np.concatenate([A, P], 0), rhs, rcond=None)[0]
            res.update(layers_o=lay_o, layers_i=lay_i, P=P)
        else:
            lay = self.forward(1.0)
            self.add_M(A, lay, -1.0)
            self.set_boundaries()
            rhs = self.rhs_forward()
            try:
                sol = np.linalg.solve(A, rhs)
            except np.linalg.LinAlgError:  # the reference's torch.linalg.solve raises here too
                sol = None
            res.update(layers=lay)
        res.update(A=A, rhs=rhs, raw_solved=sol)
        return res
