"""Boundary integral operators with the reference's class and method names.

Each class is a thin host object: its `forward` assembles its block on the
GPU through the C ABI (bem_assemble) and its `apply_*_boundary` performs the
matrix-free product (bem_apply).  Blocks, panel loops and charge indices
follow the reference operator by operator:

  SingleLayer3d         src/BEM_functions/single_layer/single_layer_3d.py:371-498
  DoubleLayer3d         src/BEM_functions/double_layer/double_layer_3d.py:376-501
  AdjDoubleLayer3d      src/BEM_functions/adj_double_layer/adj_double_layer_3d.py:379-506
  HypersingularLayer3d  src/BEM_functions/hypersingular_layer/hypersingular_layer_3d.py:437-565
  IdentityLayer3d       src/BEM_functions/identity_layer/identity_layer_3d.py:148-196
  RHSConstructor3d      src/BEM_functions/rhs_constructor/rhs_constructor_3d.py:50-386

and the 2D classes (`*2d`, the reference's *_2d.py modules), which run the
same panel loops on segment panels (P1 spaces with two hats per panel):

  SingleLayer2d         single_layer/single_layer_2d.py:217-341
  DoubleLayer2d         double_layer/double_layer_2d.py:219-342
  AdjDoubleLayer2d      adj_double_layer/adj_double_layer_2d.py:220-344
  HypersingularLayer2d  hypersingular_layer/hypersingular_layer_2d.py:253-377
  IdentityLayer2d       identity_layer/identity_layer_2d.py:120-161
  RHSConstructor2d      rhs_constructor/rhs_constructor_2d.py:50-379
"""
from __future__ import annotations

import numpy as np
import torch

from .. import _lib as L
from ..engine import upload
from ..utils.types import CellFluxType, ScopeType

_N = int(CellFluxType.NEUMANN_TOBESOLVED)
_D = int(CellFluxType.DIRICHLET_TOBESOLVED)


class _Layer:
    rank = 3

    def __init__(self, BEM_manager):
        self._BEM_manager = BEM_manager
        b = BEM_manager
        self._GaussQR = b._GaussQR
        self._dim = b._dim
        self._n = b._n
        self.N_Neumann = b.N_Neumann
        self.M_Dirichlet = b.M_Dirichlet
        self._Q_Neumann = b.shape_func_degree_Neumann
        self._Q_Dirichlet = b.shape_func_degree_Dirichlet
        self.num_of_vertices = b.num_of_vertices
        self.num_of_panels = b.num_of_panels
        self.num_of_panels_Neumann = b.num_of_panels_Neumann
        self.num_of_panels_Dirichlet = b.num_of_panels_Dirichlet

    def _desc(self, op, k, sqrt_n):
        return self._BEM_manager.op_desc(op, k, sqrt_n)

    def _zeros(self, rows, cols):
        b = self._BEM_manager
        return torch.zeros(rows, cols, dtype=b.torch_dtype, device=b.device)

    def kill(self):
        self.N_Neumann = 0
        self.M_Dirichlet = 0


class SingleLayer3d(_Layer):
    def __init__(self, BEM_manager):
        super().__init__(BEM_manager)
        self._Vmat = None
        # _Vmat is a view of the manager's _mat_A (the fused Dirichlet pass)
        self._v_alias = False

    def get_V_mat(self):
        return self._Vmat

    def forward(self, scope_type: int, k: float, sqrt_n: float):
        """V on Neumann x Neumann panels (single_layer_3d.py:371-433)."""
        if self.N_Neumann <= 0:
            return
        b = self._BEM_manager
        if self._Vmat is None or self._v_alias:
            self._Vmat = self._zeros(self.N_Neumann, self.N_Neumann)
            self._v_alias = False
        else:
            self._Vmat.zero_()
        sp = b.space("charge", self._Q_Neumann, "N", _N)
        b.engine.assemble(self._desc(L.OP_V, k, sqrt_n), sp, sp, self._Vmat)

    def apply_V_dot_N_boundary(self, scope_type: int, k: float, sqrt_n: float, multiplier: float):
        """rhs[N rows] += multiplier * V f (single_layer_3d.py:435-498)."""
        b = self._BEM_manager
        if self.num_of_panels_Neumann == 0 or self.num_of_panels_Dirichlet == 0:
            return
        test = b.space("charge", self._Q_Neumann, "N", _N, offset=b._Neumann_offset_i)
        trial = b.space("data", self._Q_Neumann, "D")
        rc = b.rhs_constructor
        b.engine.apply(self._desc(L.OP_V, k, sqrt_n), test, trial, rc._Neumann_boundary, rc._rhs_vec,
                       scale=multiplier, conj_x=b.conj_data)

    def kill(self):
        super().kill()
        self._Vmat = None


class DoubleLayer3d(_Layer):
    def __init__(self, BEM_manager):
        super().__init__(BEM_manager)
        self._Kmat = None

    def get_K_mat(self):
        return self._Kmat

    def forward(self, scope_type: int, k: float, sqrt_n: float):
        """K on Neumann x Dirichlet panels (double_layer_3d.py:376-438)."""
        if not (self.N_Neumann > 0 and self.M_Dirichlet > 0):
            return
        b = self._BEM_manager
        if self._Kmat is None:
            self._Kmat = self._zeros(self.N_Neumann, self.M_Dirichlet)
        else:
            self._Kmat.zero_()
        test = b.space("charge", self._Q_Neumann, "N", _N)
        trial = b.space("charge", self._Q_Dirichlet, "D", _D)
        b.engine.assemble(self._desc(L.OP_K, k, sqrt_n), test, trial, self._Kmat)

    def apply_K_dot_D_boundary(self, scope_type: int, k: float, sqrt_n: float, multiplier: float):
        """rhs[N rows] += multiplier * K g over Neumann x Neumann panels
        (double_layer_3d.py:440-501)."""
        b = self._BEM_manager
        if self.num_of_panels_Neumann == 0:
            return
        test = b.space("charge", self._Q_Neumann, "N", _N, offset=b._Neumann_offset_i)
        trial = b.space("data", self._Q_Dirichlet, "N")
        rc = b.rhs_constructor
        b.engine.apply(self._desc(L.OP_K, k, sqrt_n), test, trial, rc._Dirichlet_boundary, rc._rhs_vec,
                       scale=multiplier, conj_x=b.conj_data)

    def kill(self):
        super().kill()
        self._Kmat = None


class AdjDoubleLayer3d(_Layer):
    """K' is only used matrix-free; its forward is a no-op in the reference
    (adj_double_layer_3d.py:383) and the block system uses -K^T instead."""
    # whether the product takes conj(f), as the other operators do with quirk
    # (adj_double_layer_3d.py:506); the 2D operator multiplies by f itself
    _conj_data = True

    def __init__(self, BEM_manager):
        super().__init__(BEM_manager)
        self._Kmat = None

    def forward(self, scope_type: int, k: float, sqrt_n: float):
        return

    def apply_K_dot_N_boundary(self, scope_type: int, k: float, sqrt_n: float, multiplier: float):
        """rhs[D rows] += multiplier * K' f over Dirichlet x Dirichlet panels
        (adj_double_layer_3d.py:444-506)."""
        b = self._BEM_manager
        if self.num_of_panels_Dirichlet == 0:
            return
        test = b.space("charge", self._Q_Dirichlet, "D", _D, offset=b._Dirichlet_offset_i)
        trial = b.space("data", self._Q_Neumann, "D")
        rc = b.rhs_constructor
        b.engine.apply(self._desc(L.OP_KP, k, sqrt_n), test, trial, rc._Neumann_boundary, rc._rhs_vec,
                       scale=multiplier, conj_x=b.conj_data and self._conj_data)


class HypersingularLayer3d(_Layer):
    def __init__(self, BEM_manager):
        super().__init__(BEM_manager)
        self._Wmat = None

    def get_W_mat(self):
        return self._Wmat

    def forward(self, scope_type: int, k: float, sqrt_n: float):
        """W on Dirichlet x Dirichlet panels (hypersingular_layer_3d.py:437-500)."""
        if self.M_Dirichlet <= 0:
            return
        b = self._BEM_manager
        if self._Wmat is None:
            self._Wmat = self._zeros(self.M_Dirichlet, self.M_Dirichlet)
        else:
            self._Wmat.zero_()
        sp = b.space("charge", self._Q_Dirichlet, "D", _D)
        b.engine.assemble(self._desc(L.OP_W, k, sqrt_n), sp, sp, self._Wmat)

    def apply_W_dot_D_boundary(self, scope_type: int, k: float, sqrt_n: float, multiplier: float):
        """rhs[D rows] += multiplier * W g over Dirichlet x Neumann panels
        (hypersingular_layer_3d.py:502-565)."""
        b = self._BEM_manager
        if self.num_of_panels_Dirichlet == 0 or self.num_of_panels_Neumann == 0:
            return
        test = b.space("charge", self._Q_Dirichlet, "D", _D, offset=b._Dirichlet_offset_i)
        trial = b.space("data", self._Q_Dirichlet, "N")
        rc = b.rhs_constructor
        b.engine.apply(self._desc(L.OP_W, k, sqrt_n), test, trial, rc._Dirichlet_boundary, rc._rhs_vec,
                       scale=multiplier, conj_x=b.conj_data)

    def kill(self):
        super().kill()
        self._Wmat = None


class IdentityLayer3d(_Layer):
    def matA_add_global_Identity_matrix(self, mutiplier: float):
        """P0 x P1 (or P1 x P1) mass added to both off-diagonal blocks of A,
        transmission only (identity_layer_3d.py:148-196)."""
        b = self._BEM_manager
        if not b._is_transmission:
            return
        test = b.space("charge", self._Q_Neumann, "N", _N, offset=b._Neumann_offset_i)
        trial = b.space("charge", self._Q_Dirichlet, "D", _D, offset=b._Dirichlet_offset_j)
        b.engine.mass(test, trial, out=b._mat_A, scale=mutiplier, out_t=b._mat_A, scale_t=mutiplier)


class RHSConstructor3d(_Layer):
    # normal of the exterior trace in the transmission data: the 3D reference
    # takes get_panel_normal(..., EXTERIOR), which returns the same normal
    # (BEM_manager.py:330-335, rhs_constructor_3d.py:69-70)
    _ext_sign = 1.0

    def __init__(self, BEM_manager):
        super().__init__(BEM_manager)
        b = BEM_manager
        self.analytical_function_Dirichlet = b.analytical_function_Dirichlet
        self.analytical_function_Neumann = b.analytical_function_Neumann
        nN = self.num_of_panels if self._Q_Neumann == 0 else self.num_of_vertices
        nD = self.num_of_panels if self._Q_Dirichlet == 0 else self.num_of_vertices
        z = lambda n: torch.zeros(n, dtype=b.torch_dtype, device=b.device)
        self._Neumann_boundary = z(nN)
        self._Dirichlet_boundary = z(nD)
        self._f_boundary = z(self.N_Neumann + self.M_Dirichlet)
        self._rhs_vec = z(self.N_Neumann + self.M_Dirichlet)

    def get_rhs_vec(self):
        return self._rhs_vec

    def get_f_boundary(self, local_index=None):
        return self._f_boundary if local_index is None else self._f_boundary[local_index]

    def _eval(self, fn, x, *args):
        b = self._BEM_manager
        xt = x if isinstance(x, torch.Tensor) else upload(x, b.device, torch.float64)
        targs = [upload(a, b.device, torch.float64) if isinstance(a, np.ndarray) else a for a in args]
        val = fn(xt, *targs)
        return torch.as_tensor(val, device=b.device).to(b.torch_dtype).reshape(-1)

    def set_boundaries(self, scope_type: int, sqrt_ni: float, sqrt_no: float):
        """Sample the boundary data (rhs_constructor_3d.py:50-152)."""
        b = self._BEM_manager
        mm = b.mesh
        v, f = mm.vertices, mm.panels
        C = b.cached
        self._Dirichlet_boundary.zero_()
        self._Neumann_boundary.zero_()
        self._f_boundary.zero_()
        cent = lambda: v[f].sum(axis=1) / float(self._dim)
        No, Do = b._Neumann_offset_j, b._Dirichlet_offset_j
        fD, fN = self.analytical_function_Dirichlet, self.analytical_function_Neumann
        if b._is_transmission:
            if self._Q_Neumann == 0:
                gp = mm.loop_panels("N")
                x, nrm = C(("bd_cent", "N"), lambda: cent()[gp]), C(("bd_pn", "N"), lambda: mm.panel_normals[gp])
                fi = self._eval(fN, x, nrm, sqrt_ni)
                fo = self._eval(fN, x, nrm if self._ext_sign > 0 else -nrm, sqrt_no)
                self._Neumann_boundary[C(("bd_gp", "N"), lambda: gp.astype(np.int64))] += fi
                self._f_boundary[No:No + len(gp)] += fi - fo
            else:
                vv = np.nonzero(np.isin(mm.vertice_types, (2, 0)))[0]
                loc = mm._vert_local("N", vv)
                x, nrm = C(("bd_v", "N"), lambda: v[vv]), C(("bd_vn", "N"), lambda: mm.vert_normals[vv])
                fi = self._eval(fN, x, nrm, sqrt_ni)
                fo = self._eval(fN, x, nrm if self._ext_sign > 0 else -nrm, sqrt_no)
                self._Neumann_boundary[C(("bd_vv", "N"), lambda: vv)] += fi
                self._f_boundary[C(("bd_loc", "N"), lambda: (No + loc).astype(np.int64))] += fi - fo
            if self._Q_Dirichlet == 0:
                gp = mm.loop_panels("D")
                x = C(("bd_cent", "D"), lambda: cent()[gp])
                fi = self._eval(fD, x, sqrt_ni)
                fo = self._eval(fD, x, sqrt_no)
                self._Dirichlet_boundary[C(("bd_gp", "D"), lambda: gp.astype(np.int64))] += fi
                self._f_boundary[Do:Do + len(gp)] += fi - fo
            else:
                vv = np.nonzero(np.isin(mm.vertice_types, (2, 1)))[0]
                loc = mm._vert_local("D", vv)
                x = C(("bd_v", "D"), lambda: v[vv])
                fi = self._eval(fD, x, sqrt_ni)
                fo = self._eval(fD, x, sqrt_no)
                self._Dirichlet_boundary[C(("bd_vv", "D"), lambda: vv)] += fi
                self._f_boundary[C(("bd_loc", "D"), lambda: (Do + loc).astype(np.int64))] += fi - fo
        else:
            if self._Q_Neumann == 0:
                gp = mm.loop_panels("D")
                if len(gp):
                    self._Neumann_boundary[C(("bd_gp", "D"), lambda: gp.astype(np.int64))] += self._eval(
                        fN, C(("bd_cent", "D"), lambda: cent()[gp]), C(("bd_pn", "D"), lambda: mm.panel_normals[gp]))
            else:
                vv = np.nonzero(mm.vertice_types == 1)[0]
                if len(vv):
                    self._Neumann_boundary[C(("bd_v1",), lambda: vv)] += self._eval(
                        fN, C(("bd_v1x",), lambda: v[vv]), C(("bd_v1n",), lambda: mm.vert_normals[vv]))
            if self._Q_Dirichlet == 0:
                gp = mm.loop_panels("N")
                if len(gp):
                    self._Dirichlet_boundary[C(("bd_gp", "N"), lambda: gp.astype(np.int64))] += self._eval(
                        fD, C(("bd_cent", "N"), lambda: cent()[gp]))
            else:
                vv = np.nonzero(mm.vertice_types == 0)[0]
                if len(vv):
                    self._Dirichlet_boundary[C(("bd_v0",), lambda: vv)] += self._eval(
                        fD, C(("bd_v0x",), lambda: v[vv]))

    def multiply_identity_to_vector(self, multiplier: float):
        """rhs += multiplier * M (g | f) (rhs_constructor_3d.py:256-359)."""
        b = self._BEM_manager
        if self.N_Neumann > 0:
            test = b.space("charge", self._Q_Neumann, "N", _N, offset=b._Neumann_offset_i)
            trial = b.space("gcharge", self._Q_Dirichlet, "N", _N)
            b.engine.mass(test, trial, x=self._Dirichlet_boundary, y=self._rhs_vec, scale=multiplier,
                          conj_x=b.conj_data)
        if self.M_Dirichlet > 0:
            test = b.space("charge", self._Q_Dirichlet, "D", _D, offset=b._Dirichlet_offset_i)
            trial = b.space("gcharge", self._Q_Neumann, "D", _D)
            b.engine.mass(test, trial, x=self._Neumann_boundary, y=self._rhs_vec, scale=multiplier,
                          conj_x=b.conj_data)

    def multiply_M_to_vector(self, scope_type: int, k: float, sqrt_n: float, multiplier: float):
        b = self._BEM_manager
        if self.N_Neumann > 0:
            b.double_layer.apply_K_dot_D_boundary(scope_type=scope_type, k=k, sqrt_n=sqrt_n, multiplier=multiplier)
            b.single_layer.apply_V_dot_N_boundary(scope_type=scope_type, k=k, sqrt_n=sqrt_n, multiplier=-multiplier)
        if self.M_Dirichlet > 0:
            b.adj_double_layer.apply_K_dot_N_boundary(scope_type=scope_type, k=k, sqrt_n=sqrt_n,
                                                      multiplier=-multiplier)
            b.hypersingular_layer.apply_W_dot_D_boundary(scope_type=scope_type, k=k, sqrt_n=sqrt_n,
                                                         multiplier=-multiplier)

    def forward(self, scope_type: int, k: float, sqrt_n: float):
        """rhs = +-1/2 M data + M(k) data (rhs_constructor_3d.py:374-386)."""
        b = self._BEM_manager
        self._rhs_vec.zero_()
        if not b._is_transmission:
            scope_type = b._scope_type
            if scope_type == int(ScopeType.INTERIOR):
                self.multiply_identity_to_vector(multiplier=0.5)
            elif scope_type == int(ScopeType.EXTERIOR):
                self.multiply_identity_to_vector(multiplier=-0.5)
            else:
                raise RuntimeError("You have to indicate a concrete scope type to construct rhs")
            self.multiply_M_to_vector(scope_type=scope_type, k=k, sqrt_n=sqrt_n, multiplier=1.0)

    def kill(self):
        super().kill()
        self._rhs_vec = None
        self._Dirichlet_boundary = None
        self._Neumann_boundary = None
        self._f_boundary = None


# ---------------------------------------------------------------------------
# 2D (segment panels).  The host logic is the 3D classes'; the library
# evaluates the 2D integrands on a mesh set with bem_mesh_set_2d.
# ---------------------------------------------------------------------------
class SingleLayer2d(SingleLayer3d):
    rank = 2


class DoubleLayer2d(DoubleLayer3d):
    rank = 2


class AdjDoubleLayer2d(AdjDoubleLayer3d):
    """K' f with f itself, not conj(f), in the Helmholtz product
    (adj_double_layer_2d.py:344)."""
    rank = 2
    _conj_data = False


class HypersingularLayer2d(HypersingularLayer3d):
    rank = 2


class IdentityLayer2d(IdentityLayer3d):
    """Transmission identity block.  identity_layer_2d.py:154-158 calls
    integrate_on_single_panel without its `rands` argument (a TypeError in
    Python, a compile error in Taichi); this class integrates with the Gauss
    point of each loop iteration, as the loop over `iii` intends."""
    rank = 2


class RHSConstructor2d(RHSConstructor3d):
    """Boundary data on segment panels.  In the transmission data the 2D
    reference takes the exterior normal as -n (rhs_constructor_2d.py:70,84;
    its lines 72 and 86 pass an undefined `normal_x`, read here as the
    interior normal as in the 3D constructor)."""
    rank = 2
    _ext_sign = -1.0
