"""MeshManager: mesh ingest, geometry and the boundary-value-problem partition.

Host-side integer logic with the reference's names and behaviour
(src/managers/mesh_manager.py): BVP partition (`set_*_bvp`, :166-389), the
local<->global DOF maps (:415-445) and the charge-index projections used by
every operator (BEM_manager.py:224-310).  Its output is a set of
(panel list, dof table) pairs that the device kernels consume; geometry is
recomputed on the GPU by bem_mesh_set.
"""
from __future__ import annotations

import os
import re

import numpy as np

from ..meshes import analytical_disk, analytical_sphere, icosphere, load_obj, perturbed_sphere
from ..utils.types import CellFluxType, VertAttachType

_N = int(CellFluxType.NEUMANN_TOBESOLVED)
_D = int(CellFluxType.DIRICHLET_TOBESOLVED)
_MIX = int(CellFluxType.MIX_NONRESOLVED)
_BOTH = int(CellFluxType.BOTH_TOBESOLVED)
_VN = int(VertAttachType.NEUMANN_TOBESOLVED)
_VD = int(VertAttachType.DIRICHLET_TOBESOLVED)
_VB = int(VertAttachType.BOTH_TOBESOLVED)


class MeshManager:
    def __init__(self, core_manager):
        self._core_manager = core_manager
        self._log_manager = core_manager._log_manager
        p = core_manager._simulation_parameters
        self._params = p
        self._dim = int(p.get("dim", 3))
        if self._dim not in (2, 3):
            raise NotImplementedError("dim must be 2 or 3")
        self._boundary_type = p["boundary"]
        self._is_transmission = core_manager._is_transmission
        Q_Neumann = int(p.get("Q_Neumann", 0))
        Q_Dirichlet = int(p.get("Q_Dirichlet", 1))
        if Q_Neumann not in (0, 1) or Q_Dirichlet not in (0, 1):
            raise AssertionError("Q_Neumann and Q_Dirichlet must be 0 or 1")
        self.shape_func_degree_Neumann = Q_Neumann
        self.shape_func_degree_Dirichlet = Q_Dirichlet
        self.initialized = False

    # -- mesh sources ----------------------------------------------------------
    def _load(self):
        p = self._params
        if p.get("vertices") is not None and p.get("panels") is not None:
            return np.asarray(p["vertices"], np.float64), np.asarray(p["panels"], np.int32)
        if self._dim == 2:
            # the reference's 2D meshes are its analytical disk (mesh_manager.py:74-75)
            return self.load_analytical_disk(float(p.get("disk_r", 1.0)), int(p.get("disk_N", 256)))
        obj = str(p["object"])
        if "analytical" in obj:
            # any object name containing "analytical" selects the reference's
            # latitude-longitude sphere (mesh_manager.py:77-78)
            return self.load_analytical_sphere()
        m = re.fullmatch(r"icosphere(\d+)", obj)
        if m:
            return icosphere(int(m.group(1)))
        m = re.fullmatch(r"perturbed_sphere(\d+)", obj)
        if m:
            return perturbed_sphere(int(m.group(1)), lmax=int(p.get("sh_lmax", 6)),
                                    amplitude=float(p.get("sh_amplitude", 0.05)), seed=int(p.get("seed", 0)))
        return self.load_asset(scale=None, translate=None)

    def _object_path(self):
        obj = str(self._params["object"])
        path = obj if obj.endswith(".obj") else os.path.join(self._params.get("assets_path", "assets"), obj + ".obj")
        if not os.path.exists(path):
            raise FileNotFoundError(f"mesh '{obj}' not found ({path})")
        return path

    # the reference's mesh sources (mesh_manager.py:479-536)
    def load_asset(self, scale=None, translate=None):
        """OBJ asset: scaled by `scale` if given, moved by `translate` (default:
        minus the vertex mean), and, without `scale`, normalised to
        max |coordinate| = 1 (mesh_manager.py:479-494)."""
        v, f = load_obj(self._object_path(), normalise=False)
        if scale is not None:
            v = v * scale
        if translate is None:
            translate = -v.mean(axis=0, keepdims=True)
        v = v + translate
        if scale is None:
            v = v * (1.0 / np.abs(v).max())
        return v, f

    def load_analytical_sphere(self, r: float = 1.0, rows: int = 17, cols: int = 17):
        return analytical_sphere(r, rows, cols)

    def load_analytical_disk(self, r: float = 1.0, N: int = 256):
        return analytical_disk(r, N)

    def run_step(self):
        pass

    def initialization(self):
        v, f = self._load()
        d = self._dim
        if v.ndim != 2 or v.shape[1] != d or f.ndim != 2 or f.shape[1] != d:
            raise ValueError(f"vertices must be [nv,{d}] and panels [nt,{d}]")
        if not np.isfinite(v).all():
            raise ValueError("non-finite vertex coordinates")
        if f.min() < 0 or f.max() >= len(v):
            raise ValueError("panel vertex index out of range")
        self.vertices = np.ascontiguousarray(v, np.float64)
        self.panels = np.ascontiguousarray(f, np.int32)
        self.num_of_vertices = len(v)
        self.num_of_panels = len(f)
        # areas/normals with the reference's formulas (mesh_manager.py:108-139)
        if d == 2:
            e = v[f[:, 1]] - v[f[:, 0]]
            self.panel_areas = np.linalg.norm(e, axis=1)
            if (self.panel_areas <= 0).any():
                raise ValueError(f"degenerate panel {int(np.argmin(self.panel_areas))} (zero length)")
            cr = np.stack([e[:, 1], -e[:, 0]], axis=1)
            self.panel_normals = cr / np.linalg.norm(cr, axis=1)[:, None]
        else:
            a = v[f[:, 1]] - v[f[:, 0]]
            b = v[f[:, 2]] - v[f[:, 1]]
            cr = np.empty_like(a)  # a x b, component by component (as np.cross, without its overhead)
            cr[:, 0] = a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1]
            cr[:, 1] = a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2]
            cr[:, 2] = a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]
            nrm = np.linalg.norm(cr, axis=1)
            if (nrm <= 0).any():
                raise ValueError(f"degenerate panel {int(np.argmin(nrm))} (zero area)")
            self.panel_areas = 0.5 * nrm
            self.panel_normals = cr / nrm[:, None]
        # per-vertex sums over the incident panels (bincount adds in element
        # order, as a sequential scatter does)
        fv = f.reshape(-1)
        nv = self.num_of_vertices
        self.vert_areas = np.bincount(fv, weights=np.repeat(self.panel_areas / float(d), d), minlength=nv)
        pn = np.repeat(self.panel_normals, d, axis=0)
        vn = np.stack([np.bincount(fv, weights=pn[:, c], minlength=nv) for c in range(d)], axis=1)
        self.vert_normals = vn / np.linalg.norm(vn, axis=1)[:, None]
        if self._boundary_type == "Full" or self._is_transmission > 0:
            self.set_full_bvp()
        elif self._boundary_type == "Dirichlet":
            self.set_Dirichlet_bvp()
        elif self._boundary_type == "Neumann":
            self.set_Neumann_bvp()
        elif self._boundary_type == "Mix":
            self.set_mixed_bvp()
        else:
            raise RuntimeError("The Boundary Type can only be Dirichlet/Neumann/Mix")
        self.initialized = True

    # -- BVP partitions ----------------------------------------------------------
    def _count(self, q, n_panels, n_verts):
        return n_panels if q == 0 else n_verts

    def set_full_bvp(self):
        nt, nv = self.num_of_panels, self.num_of_vertices
        self.N_Neumann = self._count(self.shape_func_degree_Neumann, nt, nv)
        self.M_Dirichlet = self._count(self.shape_func_degree_Dirichlet, nt, nv)
        self.num_of_panels_Dirichlet = self.num_of_panels_Neumann = nt
        self.panel_types = np.full(nt, _BOTH, np.int32)
        self.vertice_types = np.full(nv, _VB, np.int32)
        self.Dirichlet_index = np.arange(nt, dtype=np.int32)
        self.Neumann_index = np.arange(nt, dtype=np.int32)
        self.map_global_Neumann_to_local = np.arange(nv, dtype=np.int32)
        self.map_global_Dirichlet_to_local = np.arange(nv, dtype=np.int32)

    def set_Dirichlet_bvp(self):
        nt, nv = self.num_of_panels, self.num_of_vertices
        self.N_Neumann = self._count(self.shape_func_degree_Neumann, nt, nv)
        self.M_Dirichlet = 0
        self.num_of_panels_Dirichlet, self.num_of_panels_Neumann = 0, nt
        self.panel_types = np.full(nt, _N, np.int32)
        self.vertice_types = np.full(nv, _VN, np.int32)
        self.Dirichlet_index = np.zeros(0, np.int32)
        self.Neumann_index = np.arange(nt, dtype=np.int32)
        self.map_global_Neumann_to_local = np.arange(nv, dtype=np.int32)
        self.map_global_Dirichlet_to_local = np.full(nv, -1, np.int32)

    def set_Neumann_bvp(self):
        nt, nv = self.num_of_panels, self.num_of_vertices
        self.N_Neumann = 0
        self.M_Dirichlet = self._count(self.shape_func_degree_Dirichlet, nt, nv)
        self.num_of_panels_Dirichlet, self.num_of_panels_Neumann = nt, 0
        self.panel_types = np.full(nt, _D, np.int32)
        self.vertice_types = np.full(nv, _VD, np.int32)
        self.Dirichlet_index = np.arange(nt, dtype=np.int32)
        self.Neumann_index = np.zeros(0, np.int32)
        self.map_global_Neumann_to_local = np.full(nv, -1, np.int32)
        self.map_global_Dirichlet_to_local = np.arange(nv, dtype=np.int32)

    def set_mixed_bvp(self):
        """Panels with centroid y > 0 carry Dirichlet data (Neumann unknown),
        the rest Neumann data; panels touching both vertex classes become
        MIX_NONRESOLVED (mesh_manager.py:266-389)."""
        f, v = self.panels, self.vertices
        nt, nv, d = self.num_of_panels, self.num_of_vertices, self._dim
        y = v[f, 1].sum(axis=1) / float(d)
        pt = np.where(y > 0, _N, _D).astype(np.int32)
        nN = int((pt == _N).sum())
        nD = nt - nN
        vt = np.full(nv, -1, np.int32)
        mapN = np.full(nv, -1, np.int32)
        mapD = np.full(nv, -1, np.int32)
        nvN = nvD = 0
        for kind, vkind, mp in ((_N, _VN, mapN), (_D, _VD, mapD)):
            cnt = 0
            for i in np.nonzero(pt == kind)[0]:
                for a in f[i]:
                    if vt[a] == -1:
                        vt[a] = vkind
                        mp[a] = cnt
                        cnt += 1
            if kind == _N:
                nvN = cnt
            else:
                nvD = cnt
        assert nvN + nvD == nv
        for i in range(nt):
            ds = int((vt[f[i]] == _VD).sum())
            ns = int((vt[f[i]] == _VN).sum())
            t = pt[i]
            if ns == d and t == _D:
                pt[i] = _N
                nD -= 1
                nN += 1
            elif ds == d and t == _N:
                pt[i] = _D
                nD += 1
                nN -= 1
            elif ns != d and ds != d:
                if t == _N:
                    nN -= 1
                elif t == _D:
                    nD -= 1
                pt[i] = _MIX
        self.N_Neumann = nN if self.shape_func_degree_Neumann == 0 else nvN
        self.M_Dirichlet = nD if self.shape_func_degree_Dirichlet == 0 else nvD
        self.num_of_panels_Dirichlet = nD
        self.num_of_panels_Neumann = nN
        self.panel_types = pt
        self.vertice_types = vt
        idx = np.arange(nt, dtype=np.int32)
        self.Dirichlet_index = idx[pt != _N]
        self.Neumann_index = idx[pt != _D]
        self.map_global_Neumann_to_local = mapN
        self.map_global_Dirichlet_to_local = mapD

    # -- accessors with the reference's names ----------------------------------
    def get_num_of_vertices(self):
        return self.num_of_vertices

    def get_num_of_panels(self):
        return self.num_of_panels

    def get_M_Dirichlet(self):
        return self.M_Dirichlet

    def get_N_Neumann(self):
        return self.N_Neumann

    def get_num_of_panels_Neumann(self):
        return self.num_of_panels_Neumann

    def get_num_of_panels_Dirichlet(self):
        return self.num_of_panels_Dirichlet

    def get_shape_func_degree_Neumann(self):
        return self.shape_func_degree_Neumann

    def get_shape_func_degree_Dirichlet(self):
        return self.shape_func_degree_Dirichlet

    def get_panel_areas(self):
        return self.panel_areas

    def get_panel_normals(self):
        return self.panel_normals

    def get_vert_areas(self):
        return self.vert_areas

    def get_vert_normals(self):
        return self.vert_normals

    def get_panel_types(self):
        return self.panel_types

    def get_vertice_types(self):
        return self.vertice_types

    # -- DOF tables --------------------------------------------------------------
    def loop_panels(self, side: str) -> np.ndarray:
        """Global panels of `for local_I in range(num_of_panels_X)` with
        map_local_X_index_to_panel_index: the first num_of_panels_X entries of
        the index list (which also holds the MIX panels in the Mix partition)."""
        if side == "N":
            return self.Neumann_index[:self.num_of_panels_Neumann] if self.N_Neumann > 0 else np.zeros(0, np.int32)
        return self.Dirichlet_index[:self.num_of_panels_Dirichlet] if self.M_Dirichlet > 0 else np.zeros(0, np.int32)

    def _vert_local(self, side, verts):
        if side == "N":
            ok = (self.N_Neumann > 0 and self.shape_func_degree_Neumann == 1)
            mp, good = self.map_global_Neumann_to_local, (_VN, _VB)
        else:
            ok = (self.M_Dirichlet > 0 and self.shape_func_degree_Dirichlet == 1)
            mp, good = self.map_global_Dirichlet_to_local, (_VD, _VB)
        if not ok:
            return np.full(verts.shape, -1, np.int32)
        vt = self.vertice_types[verts]
        return np.where(np.isin(vt, good), mp[verts], -1).astype(np.int32)

    def charge_dofs(self, Q: int, side: str, panel_type_as: int):
        """Local charge index table [len(loop), nb] of
        proj_from_local_panel_index_to_local_charge_index (BEM_manager.py:244-277)
        for the panel loop of `side` (whose index map selects the global panel),
        evaluated with BOTH_TOBESOLVED read as `panel_type_as`."""
        panels = self.loop_panels(side)
        pt = self.panel_types[panels].copy()
        pt[pt == _BOTH] = panel_type_as
        n = len(panels)
        if Q == 0:
            dof = np.where(pt != _MIX, np.arange(n), -1).astype(np.int32).reshape(n, 1)
            return panels, 1, dof
        dof = np.full((n, self._dim), -1, np.int32)
        verts = self.panels[panels]  # [n, dim]
        vt = self.vertice_types[verts]
        for kind, vside, excluded in ((_N, "N", _VD), (_D, "D", _VN)):
            rows = pt == kind
            if not rows.any():
                continue
            loc = self._vert_local(vside, verts[rows])
            dof[rows] = np.where(vt[rows] != excluded, loc, -1)
        return panels, self._dim, dof

    def data_dofs(self, Q: int, side: str):
        """Index into the boundary-data field (P0: global panel, P1: global
        vertex) for the panel loop of `side` (get_Dirichlet_boundary /
        get_Neumann_boundary, rhs_constructor_3d.py:158-182)."""
        panels = self.loop_panels(side)
        if Q == 0:
            return panels, 1, panels.reshape(-1, 1).copy()
        return panels, self._dim, self.panels[panels].copy()

    def global_charge(self, Q: int, side: str, panel_type_as: int):
        """proj_from_local_panel_index_to_global_charge_index (BEM_manager.py:279-310)
        over the panel loop of `side`, with the (substituted) panel type."""
        panels = self.loop_panels(side)
        pt = self.panel_types[panels].copy()
        pt[pt == _BOTH] = panel_type_as
        nb = 1 if Q == 0 else self._dim
        out = np.full((len(panels), nb), -1, np.int32)
        for kind, s in ((_N, "N"), (_D, "D")):
            rows = pt == kind
            if not rows.any():
                continue
            src = self.Neumann_index if s == "N" else self.Dirichlet_index
            gp = src[np.nonzero(rows)[0]]
            out[rows] = gp.reshape(-1, 1) if Q == 0 else self.panels[gp]
        return panels, nb, out

    def kill(self):
        self.initialized = False
        self.vertices = None
        self.panels = None
