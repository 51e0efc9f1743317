"""BEMManager: the assembly and solve driver (src/managers/BEM_manager.py).

Same method names and sequencing as the reference; every O(n^2) and heavier
step runs on the GPU through libbem_b200 (operator blocks, matrix-free
products, mass blocks, LU, triangular solves, refinement).  Block placement
follows the reference: DOF order [Dirichlet (M_D) | Neumann (N_N)]
(BEM_manager.py:104-111) and

    M = [ K  -V ]      matA_add_M(c):  A_NN += -c V,  A_ND += c K,
        [-W  -K']                      A_DN += -c K^T, A_DD += -c W.

Extra simulation_parameters keys (all optional):
  precision: "fp64" (plain path: every quadrature point and the LU in FP64)
             or "mixed" (separate pairs in FP32, near field in FP64, FP32 LU
             with FP64 iterative refinement against the FP64-stored matrix)
  quirk:     True (default) reproduces the reference's quadrature exactly;
             False uses the corrected Sauter-Schwab orientation and g (not
             conj g) in the Helmholtz right-hand side
  honour_show: whether the `show` parameter selects the splat and colouring
             (the reference's own code ignores it); default: not quirk
  solver:    "lstsq" (transmission default, the reference's least squares on
             [A; P+_i] by the column-equilibrated normal equations on this
             library's kernels) or "lu" (square A)
  refine_tol / refine_maxit: iterative-refinement controls of the mixed path
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .. import _lib as L
from ..BEM_functions.layers import (AdjDoubleLayer2d, AdjDoubleLayer3d, DoubleLayer2d, DoubleLayer3d,
                                    HypersingularLayer2d, HypersingularLayer3d, IdentityLayer2d, IdentityLayer3d,
                                    RHSConstructor2d, RHSConstructor3d, SingleLayer2d, SingleLayer3d)
from ..engine import DeviceSpace, Engine, upload
from ..utils.types import AssembleType, CellFluxType, KernelType, ScopeType, VertAttachType


class BEMManager:
    def __init__(self, core_manager):
        self._core_manager = core_manager
        self._log_manager = core_manager._log_manager
        self._is_transmission = core_manager._is_transmission
        p = core_manager._simulation_parameters
        self._simulation_parameters = p
        kern = p["kernel"]
        if kern == "Laplace":
            self._kernel_type, self._n = int(KernelType.LAPLACE), 1
        elif kern == "Helmholtz":
            self._kernel_type, self._n = int(KernelType.HELMHOLTZ), 2
        elif kern == "Helmholtz_Transmission":
            self._kernel_type, self._n = int(KernelType.HELMHOLTZ_TRANSMISSION), 2
        else:
            raise RuntimeError("Kernel Type only support Laplace and Helmholtz for now")
        show = p.get("show", "Default")
        if show not in ("Neumann", "Dirichlet", "Default"):
            raise RuntimeError("The supported type for visualization is only Neumann/Dirichlet/Default")
        self.quirk = bool(p.get("quirk", True))
        self.show = {"Neumann": int(VertAttachType.NEUMANN_TOBESOLVED),
                     "Dirichlet": int(VertAttachType.DIRICHLET_TOBESOLVED), "Default": -1}[show]
        # The reference stores the parameter in `show` and reads `_show`, which
        # stays -1 (BEM_manager.py:28,43-50): the parameter has no effect on
        # the splat and the colouring.  honour_show=False reproduces that;
        # honour_show=True applies the parameter.  By default it follows quirk
        # (reference behaviour with the reference quadrature).
        self.honour_show = bool(p.get("honour_show", not self.quirk))
        self._show = self.show if self.honour_show else -1
        if self._show == -1 and self._is_transmission:
            self._show = int(VertAttachType.NEUMANN_TOBESOLVED)
        self._k = float(p.get("k", 0.0)) if self._n == 2 else 0.0
        self._sqrt_ni = self._sqrt_no = 1.0
        if self._kernel_type == int(KernelType.HELMHOLTZ_TRANSMISSION):
            self._sqrt_ni = float(math.sqrt(p["n_i"]))
            self._sqrt_no = float(math.sqrt(p["n_o"]))
        self._dim = int(p.get("dim", 3))
        self._GaussQR = int(p["GaussQR"])
        self._scope_type = int(ScopeType.NOT_DEFINED)
        if p.get("scope") == "Interior":
            self._scope_type = int(ScopeType.INTERIOR)
        elif p.get("scope") == "Exterior":
            self._scope_type = int(ScopeType.EXTERIOR)
        self.precision = p.get("precision", "fp64")
        if self.precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        # precision of the dense solve ("fp64": partial-pivoting LU; "mixed":
        # FP32 tile LU + FP64 refinement), by default the assembly's
        self.solve_precision = p.get("solve_precision", self.precision)
        # one sweep for V and K g in the Dirichlet problem (the plain path keeps
        # one kernel per operator)
        self.fuse = bool(p.get("fuse", self.precision == "mixed"))
        self.solver = p.get("solver", "lstsq" if self._is_transmission else "lu")
        # transmission: V, K, K^T and W of both scopes from one sweep over the
        # unordered panel pairs (bem_assemble_calderon) straight into _mat_A
        # and _mat_P, instead of one kernel per operator and scope
        self.fuse_calderon = bool(p.get("fuse_calderon", True))
        # least squares of the transmission system: relative residual of the
        # scaled normal equations at which the FP64 iteration stops, the level
        # accepted once it stagnates, and its step cap
        self.lstsq_tol = float(p.get("lstsq_tol", 1e-14))
        self.lstsq_accept = float(p.get("lstsq_accept", 1e-10))
        self.lstsq_maxit = int(p.get("lstsq_maxit", 90))
        self._mat_P = None
        # relative residual at which FP64 refinement stops: 1e-9 in mixed
        # precision (its contribution to the solution error is at most
        # cond(A) * 1e-9, ~1e-7 for cond(A) ~ 1e2, the order of the FP32
        # assembly's own error and well inside the 1e-6 target), 1e-12 otherwise
        self.refine_tol = float(p.get("refine_tol", 1e-9 if self.precision == "mixed" else 1e-12))
        self.refine_maxit = int(p.get("refine_maxit", 60))
        # a refinement that stagnates at this relative residual or below is
        # accepted (the attainable FP64 level of an ill-conditioned system)
        self.refine_accept = float(p.get("refine_accept", 1e-8))
        # iterative operator-norm estimates: relative change of the smallest
        # Ritz value at which the block Krylov estimate stops, block cap
        self.norm_tol = float(p.get("norm_tol", 1e-10))
        self.norm_maxit = int(p.get("norm_maxit", 32))
        self.device = torch.device(p.get("device", "cuda"))
        self.torch_dtype = torch.complex128 if self._n == 2 else torch.float64
        self.conj_data = (self._n == 2) and self.quirk
        # operator descriptors of the k-derivative pass (managers/kderiv.py):
        # the kernel's k-derivative, and a replacement W mass coefficient k2
        self._desc_deriv_k = False
        self._desc_k2 = None
        self._lstsq_factor = None
        # the norm estimator's state carried between calls (the Cholesky shift of a sweep)
        self._norm_info = {}
        # L^{-1} of the energy scalings of A_I and A_II (compute_inv_norm)
        self._L1_inv = None
        self._L2_inv = None
        self.solve_info = {}
        self.initialized = False

    # -- set-up -------------------------------------------------------------------
    def initialization(self, analytical_function_Dirichlet, analytical_function_Neumann):
        mm = self._core_manager._mesh_manager
        if not mm.initialized:
            raise RuntimeError("The initialization of Mesh Manager should always before the BEM Manager")
        self.mesh = mm
        self.num_of_vertices = mm.get_num_of_vertices()
        self.num_of_panels = mm.get_num_of_panels()
        self.N_Neumann = mm.get_N_Neumann()
        self.M_Dirichlet = mm.get_M_Dirichlet()
        self.shape_func_degree_Neumann = mm.get_shape_func_degree_Neumann()
        self.shape_func_degree_Dirichlet = mm.get_shape_func_degree_Dirichlet()
        self.num_of_panels_Neumann = mm.get_num_of_panels_Neumann()
        self.num_of_panels_Dirichlet = mm.get_num_of_panels_Dirichlet()
        self._Dirichlet_offset_i = self._Dirichlet_offset_j = 0
        self._Neumann_offset_i = self._Neumann_offset_j = self.M_Dirichlet
        self.analytical_function_Dirichlet = analytical_function_Dirichlet
        self.analytical_function_Neumann = analytical_function_Neumann
        n = self.N_Neumann + self.M_Dirichlet
        if n <= 0:
            raise AssertionError("no unknowns")
        self.engine = Engine(self.device)
        self.engine.set_mesh(mm.vertices, mm.panels, self._GaussQR, dim=self._dim)
        self._spaces = {}
        self._dev_cache = {}
        z = lambda *s: torch.zeros(*s, dtype=self.torch_dtype, device=self.device)
        self._mat_A = z(n, n)
        self.rhs = z(2 * n if self._is_transmission else n)
        self.raw_solved = z(n)
        self.raw_analytical_solved = z(n)
        self.solved = z(self.num_of_vertices)
        self.analytical_solved = z(self.num_of_vertices)
        # colour and position buffers of the reference's window (BEM_manager.py:132-138), kept headless
        for name in ("solved_vert_color", "solved_vertices", "analytical_vert_color", "analytical_vertices",
                     "diff_vert_color", "diff_vertices"):
            setattr(self, name, torch.zeros(self.num_of_vertices, 3, dtype=torch.float32, device=self.device))
        # BIO objects of the mesh's dimension (BEM_manager.py:175-191)
        if self._dim == 2:
            self.identity_layer = IdentityLayer2d(self)
            self.single_layer = SingleLayer2d(self)
            self.double_layer = DoubleLayer2d(self)
            self.adj_double_layer = AdjDoubleLayer2d(self)
            self.hypersingular_layer = HypersingularLayer2d(self)
            self.rhs_constructor = RHSConstructor2d(self)
        else:
            self.identity_layer = IdentityLayer3d(self)
            self.single_layer = SingleLayer3d(self)
            self.double_layer = DoubleLayer3d(self)
            self.adj_double_layer = AdjDoubleLayer3d(self)
            self.hypersingular_layer = HypersingularLayer3d(self)
            self.rhs_constructor = RHSConstructor3d(self)
        self.initialized = True

    def space(self, kind: str, Q: int, side: str, as_type: int = 0, offset: int = 0) -> DeviceSpace:
        """Device (panel list, dof table) of one operator side, cached."""
        key = (kind, Q, side, as_type, offset)
        sp = self._spaces.get(key)
        if sp is None:
            mm = self.mesh
            if kind == "charge":
                panels, nb, dof = mm.charge_dofs(Q, side, as_type)
            elif kind == "data":
                panels, nb, dof = mm.data_dofs(Q, side)
            elif kind == "gcharge":
                panels, nb, dof = mm.global_charge(Q, side, as_type)
            else:
                raise ValueError(kind)
            dof = np.where(dof >= 0, dof + offset, -1)
            sp = DeviceSpace.from_numpy(panels, nb, dof, self.device)
            self._spaces[key] = sp
        return sp

    def cached(self, key, make, dtype=None) -> torch.Tensor:
        """Device copy of a mesh-derived host array, made once per mesh (the
        boundary data, post-processing and index gathers of every run reuse
        it instead of copying from pageable host memory)."""
        t = self._dev_cache.get(key)
        if t is None:
            t = upload(np.ascontiguousarray(make()), self.device)
            if dtype is not None:
                t = t.to(dtype)
            self._dev_cache[key] = t
        return t

    def op_desc(self, op: int, k: float, sqrt_n: float) -> L.OpDesc:
        helm = self._n == 2
        uses_n = self._kernel_type == int(KernelType.HELMHOLTZ_TRANSMISSION)
        k_kernel = k * sqrt_n if uses_n else k
        k2 = k * k * sqrt_n * sqrt_n
        if self._desc_k2 is not None:
            k2 = self._desc_k2
        prec = L.PREC_MIXED if self.precision == "mixed" else L.PREC_FP64
        return Engine.op_desc(op, helm, k_kernel if helm else 0.0, k2 if helm else 0.0, quirk=self.quirk,
                              precision=prec, deriv_k=self._desc_deriv_k)

    # -- accessors ------------------------------------------------------------------
    def get_GaussQR(self):
        return self._GaussQR

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

    def get_mat_A(self):
        return self._mat_A

    def get_scope_type(self):
        return self._scope_type

    def set_scope_type(self, scope_type):
        self._scope_type = scope_type

    # -- operators and block system ------------------------------------------------------
    def matrix_layer_forward(self, k: float, sqrt_n: float = 1.0, scope_type: int = int(ScopeType.NOT_DEFINED)):
        if scope_type == int(ScopeType.NOT_DEFINED):
            raise RuntimeError("Did not indicate a correct scope type!")
        self.set_scope_type(scope_type)
        self.single_layer.forward(scope_type, k, sqrt_n)
        self.double_layer.forward(scope_type, k, sqrt_n)
        self.adj_double_layer.forward(scope_type, k, sqrt_n)
        self.hypersingular_layer.forward(scope_type, k, sqrt_n)

    def rhs_layer_forward(self, scope_type, k: float, sqrt_n: float = 1.0):
        self.rhs_constructor.forward(scope_type=scope_type, k=k, sqrt_n=sqrt_n)

    def matA_add_M(self, multiplier: float):
        A = self._mat_A
        No, Do = self._Neumann_offset_i, self._Dirichlet_offset_i
        N, M = self.N_Neumann, self.M_Dirichlet
        if N > 0:
            A[No:No + N, No:No + N].add_(self.single_layer._Vmat, alpha=-multiplier)
        if N > 0 and M > 0:
            K = self.double_layer._Kmat
            A[No:No + N, Do:Do + M].add_(K, alpha=multiplier)
            A[Do:Do + M, No:No + N].add_(K.transpose(0, 1), alpha=-multiplier)
        if M > 0:
            A[Do:Do + M, Do:Do + M].add_(self.hypersingular_layer._Wmat, alpha=-multiplier)

    def assemble_matA(self, assemble_type: int, multiplier: float):
        """M = [K, -V; -W, -K'] (BEM_manager.py:630-645)."""
        if assemble_type == int(AssembleType.ADD_M):
            self.matA_add_M(multiplier)
        elif assemble_type == int(AssembleType.ADD_HALF_IDENTITY):
            self.identity_layer.matA_add_global_Identity_matrix(0.5 * multiplier)
        elif assemble_type == int(AssembleType.ADD_P_MINUS):
            self.identity_layer.matA_add_global_Identity_matrix(0.5 * multiplier)
            self.matA_add_M(-multiplier)
        elif assemble_type == int(AssembleType.ADD_P_PLUS):
            self.identity_layer.matA_add_global_Identity_matrix(0.5 * multiplier)
            self.matA_add_M(multiplier)

    def assemble_rhs(self):
        """Transmission: rhs[:n] = A conj(f) (BEM_manager.py:647-662); else a copy."""
        n = self.N_Neumann + self.M_Dirichlet
        if self._is_transmission:
            self.rhs.zero_()
            f = self.rhs_constructor._f_boundary
            f = f.conj().resolve_conj() if self.conj_data else f
            self.engine.gemv(self._mat_A, f.contiguous(), self.rhs[:n], alpha=1.0, beta=0.0)
        else:
            self.rhs.copy_(self.rhs_constructor._rhs_vec)

    # -- solve --------------------------------------------------------------------------
    def _lu_solve_fp64(self, A: torch.Tensor, b: torch.Tensor, cols) -> torch.Tensor:
        """Partial-pivoting FP64 LU and solves.  An exact zero pivot raises
        torch.linalg.LinAlgError, as the reference's torch.linalg.solve does
        on a singular matrix (BEM_manager.py:1056)."""
        LU = A.clone()
        piv, info = self.engine.lu_factor(LU)
        zero_pivot = int(info.item())  # the solves below synchronise the stream anyway
        if zero_pivot > 0:
            raise torch.linalg.LinAlgError(
                "linalg.solve: The solver failed because the input matrix is singular "
                f"(zero pivot in column {zero_pivot - 1}).")
        xs = []
        for c in cols:
            x = c.clone()
            self.engine.lu_solve(LU, piv, x)
            xs.append(x)
        self.solve_info = {"factor": "fp64", "info": info}
        return xs[0] if b.dim() == 1 else torch.stack(xs, 1)

    def _lu_solve_square(self, A: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        """x = A^{-1} b with the hand-written LU: FP64 factor (plain path) or
        FP32 factor + FP64 refinement against A (mixed path).  b is a vector
        or an n x nrhs matrix; A is factored once."""
        cols = [b.contiguous()] if b.dim() == 1 else [b[:, j].contiguous() for j in range(b.shape[1])]
        if self.solve_precision == "fp64":
            return self._lu_solve_fp64(A, b, cols)
        lo = torch.complex64 if A.is_complex() else torch.float32
        LU = A.to(lo)
        piv, dinv, info = self.engine.lu_factor_tiled(LU)
        kind = "fp32 tile-pivoted + refinement"
        state = {"LU": LU, "piv": piv, "dinv": dinv}

        class _ZeroPivot(Exception):
            pass

        def partial_pivoting():
            # tile pivoting restricts row swaps to the 64-row diagonal tiles; a
            # matrix whose large entries sit off the diagonal blocks needs
            # partial pivoting over full columns
            if state["dinv"] is not None:
                state["LU"] = A.to(lo)
                state["piv"], pinfo = self.engine.lu_factor(state["LU"])
                state["dinv"] = None
                if int(pinfo.item()) > 0:
                    # an exact zero pivot even with full-column pivoting: the FP64
                    # factorisation decides (it raises if A is singular in FP64)
                    raise _ZeroPivot()

        xs, its, rrs = [], [], []
        for c in cols:
            x = torch.zeros_like(c)
            try:
                it, rr = self.engine.refine_solve(A, state["LU"], state["piv"], c, x, tol=self.refine_tol,
                                                  maxit=self.refine_maxit, dinv=state["dinv"],
                                                  accept=self.refine_accept)
            except L.BemError as exc:
                if exc.code != -4:
                    raise
                try:
                    partial_pivoting()
                except _ZeroPivot:
                    return self._lu_solve_fp64(A, b, cols)
                x.zero_()
                try:
                    it, rr = self.engine.refine_solve(A, state["LU"], state["piv"], c, x, tol=self.refine_tol,
                                                      maxit=self.refine_maxit, accept=self.refine_accept)
                    kind = "fp32 partial pivoting + refinement"
                except L.BemError as exc2:
                    if exc2.code != -4:
                        raise
                    # plain refinement contracts too slowly (cond(A) u_fp32 near 1):
                    # GMRES in FP64 with the same factor as preconditioner
                    x.zero_()
                    it, rr = self.engine.gmres_solve(A, state["LU"], state["piv"], c, x, tol=self.refine_tol,
                                                     maxit=max(self.refine_maxit, 300), restart=60,
                                                     accept=self.refine_accept)
                    kind = "fp32 partial pivoting + GMRES-IR"
            xs.append(x)
            its.append(it)
            rrs.append(rr)
        if int(info.item()) > 0:
            # the tile factor met an exact zero pivot (read after the refinement's
            # synchronisation): refinement can still converge on a singular but
            # consistent system, where the reference's torch.linalg.solve raises,
            # so the FP64 factorisation decides
            return self._lu_solve_fp64(A, b, cols)
        self.solve_info = {"factor": kind, "info": info, "refine_iters": max(its), "relres": max(rrs)}
        return xs[0] if b.dim() == 1 else torch.stack(xs, 1)

    def _lstsq(self, A: torch.Tensor, P: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        """min ||[A; P] x - b|| (the reference's torch.linalg.lstsq on the
        stacked transmission system, BEM_manager.py:1039-1050) by the
        column-equilibrated normal equations: the normal matrix on the tensor
        cores (FP16-split products in mixed precision, FP64 products on the
        plain path), its Cholesky, and flexible GMRES in FP64 on the normal
        equations against the FP64-stored A and P."""
        return self.lstsq_multi(A, P, b.view(-1, 1))[:, 0]

    def lstsq_multi(self, A: torch.Tensor, P: torch.Tensor, B: torch.Tensor, keep_factor: bool = False) -> torch.Tensor:
        """min ||[A; P] x - b|| for each column b of B (2n x nrhs): one normal
        matrix and Cholesky, one flexible GMRES per column (see _lstsq).
        Returns X (n x nrhs); solve_info holds the last column's iterations
        and residual and the largest iteration count.  With keep_factor the
        factor stays in _lstsq_factor (normal_solve)."""
        n = A.shape[0]
        mixed = self.solve_precision == "mixed"
        # the factor is a Cholesky with an FP64 Schur complement on both
        # paths: the normal matrix of the 30722-unknown transmission problem
        # has cond ~3e6, where an FP32 factorisation no longer preconditions
        # (measured: FGMRES stalls); the mixed path forms its O(n^3) updates
        # on the tcgen05 tensor cores
        d = torch.empty(n, dtype=torch.float64, device=A.device)
        Nm = torch.empty(n, n, dtype=A.dtype, device=A.device)
        self.engine.gram(A, P, Nm, d, tensor_cores=mixed)
        piv, dinv, info = self.engine.chol_factor(Nm, tensor_cores=mixed)
        if int(info.item()) > 0:
            raise torch.linalg.LinAlgError("linalg.lstsq: the stacked system is rank deficient (its normal matrix "
                                           f"has no positive pivot in column {int(info.item()) - 1})")
        X = torch.zeros(n, B.shape[1], dtype=A.dtype, device=A.device)
        its_max = 0
        for c in range(B.shape[1]):
            x = torch.zeros(n, dtype=A.dtype, device=A.device)
            its, rr = self.engine.lstsq_refine(A, P, d, Nm, piv, dinv, B[:, c].contiguous(), x, tol=self.lstsq_tol,
                                               maxit=self.lstsq_maxit, restart=30, accept=self.lstsq_accept)
            X[:, c] = x
            its_max = max(its_max, its)
        self.solve_info = {"factor": ("fp16-split tcgen05 normal matrix, Cholesky with tcgen05 updates" if mixed
                                      else "fp64 DMMA normal matrix, Cholesky with DMMA updates")
                           + " (FP64 Schur complement), fp64 flexible GMRES",
                           "info": info, "refine_iters": its, "relres": rr, "refine_iters_max": its_max}
        self._lstsq_factor = (A, P, d, Nm, piv, dinv) if keep_factor else None
        del Nm, dinv
        return X

    def normal_solve(self, g: torch.Tensor) -> torch.Tensor:
        """(A^H A + P^H P)^{-1} g with the factor kept by the last
        lstsq_multi(keep_factor=True): the adjoint solve of the least-squares
        problem, by the same FP64 flexible GMRES (bem_normal_refine)."""
        A, P, d, Nm, piv, dinv = self._lstsq_factor
        x = torch.zeros_like(g)
        its, rr = self.engine.normal_refine(A, P, d, Nm, piv, dinv, g.contiguous(), x, tol=self.lstsq_tol,
                                            maxit=self.lstsq_maxit, restart=30, accept=self.lstsq_accept)
        self.solve_info["adjoint_iters"], self.solve_info["adjoint_relres"] = its, rr
        return x

    def transmission_blocks(self):
        """(A, P+_i) of the assembled transmission system: the fused path's
        two matrices, or A saved and P+_i assembled into _mat_A from the
        interior layers (as the reference does before its lstsq,
        BEM_manager.py:1039-1047)."""
        if self._mat_P is not None and self._calderon_fusable():
            return self._mat_A, self._mat_P
        A_top = self._mat_A.clone()
        self._mat_A.zero_()
        self.assemble_matA(assemble_type=int(AssembleType.ADD_P_PLUS), multiplier=1.0)
        return A_top, self._mat_A.clone()

    def solve(self):
        n = self.N_Neumann + self.M_Dirichlet
        if self._is_transmission:
            # the reference stacks [A; P+_i] and calls lstsq (BEM_manager.py:1039-1050)
            A_top, P = self.transmission_blocks()
            if self.solver == "lstsq":
                sol = self._lstsq(A_top.contiguous(), P.contiguous(), self.rhs.contiguous())
            else:
                sol = self._lu_solve_square(A_top.contiguous(), self.rhs[:n].contiguous())
            if A_top is not self._mat_A:
                self._mat_A.copy_(A_top)
        else:
            sol = self._lu_solve_square(self._mat_A, self.rhs)
        self.raw_solved.copy_(sol)

    # -- post-processing (headless device buffers) ------------------------------------------
    def compute_analytical_raw_solved(self):
        """Exact traces at the DOFs (BEM_manager.py:664-750)."""
        self.raw_analytical_solved.zero_()
        mm = self.mesh
        rc = self.rhs_constructor
        dev = self.device
        v, f = mm.vertices, mm.panels
        if self._is_transmission:
            Do, No = self._Dirichlet_offset_j, self._Neumann_offset_j
            nD = len(rc._Dirichlet_boundary)
            nN = len(rc._Neumann_boundary)
            self.raw_analytical_solved[Do:Do + min(nD, self.M_Dirichlet)] = rc._Dirichlet_boundary[:self.M_Dirichlet]
            self.raw_analytical_solved[No:No + min(nN, self.N_Neumann)] = rc._Neumann_boundary[:self.N_Neumann]
            return
        C = self.cached
        cent = lambda: v[f].sum(axis=1) / float(self._dim)
        if self.N_Neumann > 0:
            if self.shape_func_degree_Neumann == 0:
                gp = mm.loop_panels("N")
                val = rc._eval(self.analytical_function_Neumann, C(("ex_cent", "N"), lambda: cent()[gp]),
                               C(("ex_pn", "N"), lambda: mm.panel_normals[gp]))
                self.raw_analytical_solved[self._Neumann_offset_j:self._Neumann_offset_j + len(gp)] = val
            else:
                vv = np.nonzero(mm.vertice_types == int(VertAttachType.NEUMANN_TOBESOLVED))[0]
                loc = mm._vert_local("N", vv)
                ok = loc >= 0
                val = rc._eval(self.analytical_function_Neumann, C(("ex_v", "N"), lambda: v[vv[ok]]),
                               C(("ex_vn", "N"), lambda: mm.vert_normals[vv[ok]]))
                self.raw_analytical_solved[C(("ex_loc", "N"), lambda: loc[ok] + self._Neumann_offset_j)] = val
        if self.M_Dirichlet > 0:
            if self.shape_func_degree_Dirichlet == 0:
                gp = mm.loop_panels("D")
                val = rc._eval(self.analytical_function_Dirichlet, C(("ex_cent", "D"), lambda: cent()[gp]))
                self.raw_analytical_solved[self._Dirichlet_offset_j:self._Dirichlet_offset_j + len(gp)] = val
            else:
                vv = np.nonzero(mm.vertice_types == int(VertAttachType.DIRICHLET_TOBESOLVED))[0]
                loc = mm._vert_local("D", vv)
                ok = loc >= 0
                val = rc._eval(self.analytical_function_Dirichlet, C(("ex_v", "D"), lambda: v[vv[ok]]))
                self.raw_analytical_solved[C(("ex_loc", "D"), lambda: loc[ok] + self._Dirichlet_offset_j)] = val

    def splat_u_from_raw_solved_to_vertices(self):
        """Per-vertex values (BEM_manager.py:752-801): P0 values are
        area-weighted onto the panel's vertices, P1 values copied."""
        self.solved.zero_()
        self.analytical_solved.zero_()
        mm = self.mesh
        C = self.cached

        def splat_p0(side, offset, excluded):
            gp = mm.loop_panels(side)
            if len(gp) == 0:
                return
            ok = mm.panel_types[gp] != excluded
            gsel = gp[ok]
            # per-panel weight area/dim / vertex area, the panel's vertices and DOF rows
            w = C(("sp_w", side), lambda: (mm.panel_areas[gsel] / float(self._dim))[:, None]
                  / mm.vert_areas[mm.panels[gsel]])
            fv = C(("sp_f", side), lambda: mm.panels[gsel].reshape(-1).astype(np.int64))
            rows = C(("sp_rows", side, offset), lambda: np.arange(len(gp))[ok] + offset)
            for src, dst in ((self.raw_solved, self.solved), (self.raw_analytical_solved, self.analytical_solved)):
                vals = src[rows].unsqueeze(1) * w
                dst.index_add_(0, fv, vals.reshape(-1))

        def splat_p1(side, offset, excluded):
            vv = np.nonzero(mm.vertice_types != excluded)[0]
            loc = mm._vert_local(side, vv)
            ok = loc >= 0
            if not ok.any():
                return
            vt = C(("sp_vt", side, excluded), lambda: vv[ok])
            lt = C(("sp_lt", side, excluded, offset), lambda: loc[ok] + offset)
            self.solved[vt] += self.raw_solved[lt]
            self.analytical_solved[vt] += self.raw_analytical_solved[lt]

        if self._show != int(VertAttachType.DIRICHLET_TOBESOLVED):
            if self.shape_func_degree_Neumann == 0:
                splat_p0("N", self._Neumann_offset_j, int(CellFluxType.DIRICHLET_TOBESOLVED))
            else:
                splat_p1("N", self._Neumann_offset_j, int(VertAttachType.DIRICHLET_TOBESOLVED))
        if self._show != int(VertAttachType.NEUMANN_TOBESOLVED):
            if self.shape_func_degree_Dirichlet == 0:
                splat_p0("D", self._Dirichlet_offset_j, int(CellFluxType.NEUMANN_TOBESOLVED))
            else:
                splat_p1("D", self._Dirichlet_offset_j, int(VertAttachType.NEUMANN_TOBESOLVED))

    def compute_color(self):
        """BEMManager.compute_color (BEM_manager.py:527-587) into the headless
        colour buffers.  As in the reference, `solved` at the Dirichlet-to-be-
        solved vertices (every vertex when show is Dirichlet) is shifted onto
        the mean of the exact traces there: a Neumann problem fixes the
        Dirichlet trace only up to a constant."""
        vt = self.cached("vert_types", lambda: self.mesh.vertice_types, dtype=torch.int32)
        self.engine.compute_color(self.solved, self.analytical_solved, vt, self._show, self.solved_vert_color,
                                  self.analytical_vert_color, self.diff_vert_color)

    def set_mesh_instances(self):
        """BEMManager.set_mesh_instances (BEM_manager.py:589-606): the vertex
        positions of the solved, exact (x - 2.2) and difference (x + 2.2)
        copies of the mesh."""
        self.engine.set_mesh_instances(self.solved_vertices, self.analytical_vertices, self.diff_vertices)

    # -- driver ----------------------------------------------------------------------------
    def _fusable(self) -> bool:
        """Dirichlet problem with P0 Neumann unknowns: V and K g share every
        panel pair (Neumann x Neumann), so one sweep serves both."""
        return (self.fuse and not self._is_transmission and self.M_Dirichlet == 0 and self.N_Neumann > 0
                and self.shape_func_degree_Neumann == 0 and self.num_of_panels_Dirichlet == 0)

    def _run_dirichlet_fused(self):
        """matrix_layer_forward + assemble_matA(ADD_M, -1) + set_boundaries +
        rhs_layer_forward + assemble_rhs with V and K g assembled in one pass.
        The system matrix of this problem is V itself (P0 Neumann unknowns
        only), so the sweep writes V straight into the zeroed _mat_A and the
        single layer's _Vmat is a view of it (flagged, so that the layer's
        own forward or matrix_layer_init give it its own storage again)
        instead of a separate block zeroed, filled and copied."""
        rc = self.rhs_constructor
        rc.set_boundaries(scope_type=self._scope_type, sqrt_ni=self._sqrt_ni, sqrt_no=self._sqrt_no)
        lay = self.single_layer
        direct = self._mat_A.shape == (self.N_Neumann, self.N_Neumann) and self._Neumann_offset_i == 0 \
            and self._Neumann_offset_j == 0
        if direct:
            lay._Vmat = self._mat_A  # zeroed by assemble_system
            lay._v_alias = True
        else:
            if lay._Vmat is None or lay._v_alias:
                lay._Vmat = lay._zeros(self.N_Neumann, self.N_Neumann)
                lay._v_alias = False
            else:
                lay._Vmat.zero_()
        rc._rhs_vec.zero_()
        self.fused_assembly_call()
        half = 0.5 if self._scope_type == int(ScopeType.INTERIOR) else -0.5
        rc.multiply_identity_to_vector(multiplier=half)
        if not direct:
            self.assemble_matA(assemble_type=int(AssembleType.ADD_M), multiplier=-1.0)
        self.assemble_rhs()

    # -- operator norms (BEM_manager.py:846-988) ------------------------------------
    def matrix_layer_init(self):
        """Zero the operator blocks (BEM_manager.py:823-827)."""
        for lay in (self.single_layer, self.double_layer, self.adj_double_layer, self.hypersingular_layer):
            if getattr(lay, "_v_alias", False):
                lay._Vmat, lay._v_alias = None, False  # a view of _mat_A: give the layer its own block
            for name in ("_Vmat", "_Kmat", "_Wmat"):
                blk = getattr(lay, name, None)
                if blk is not None:
                    blk.zero_()

    def get_V_part(self, A):
        No, N = self._Neumann_offset_i, self.N_Neumann
        return A[No:No + N, self._Neumann_offset_j:self._Neumann_offset_j + N]

    def get_K_part(self, A):
        return A[self._Neumann_offset_i:self._Neumann_offset_i + self.N_Neumann,
                 self._Dirichlet_offset_j:self._Dirichlet_offset_j + self.M_Dirichlet]

    def get_adj_K_part(self, A):
        return A[self._Dirichlet_offset_i:self._Dirichlet_offset_i + self.M_Dirichlet,
                 self._Neumann_offset_j:self._Neumann_offset_j + self.N_Neumann]

    def get_W_part(self, A):
        Do, M = self._Dirichlet_offset_i, self.M_Dirichlet
        return A[Do:Do + M, self._Dirichlet_offset_j:self._Dirichlet_offset_j + M]

    # block writers, the inverse of get_*_part (BEM_manager.py:862-872)
    def set_V_part(self, old_tensor, new_tensor):
        self.get_V_part(old_tensor)[...] = new_tensor

    def set_K_part(self, old_tensor, new_tensor):
        self.get_K_part(old_tensor)[...] = new_tensor

    def set_adj_K_part(self, old_tensor, new_tensor):
        self.get_adj_K_part(old_tensor)[...] = new_tensor

    def set_W_part(self, old_tensor, new_tensor):
        self.get_W_part(old_tensor)[...] = new_tensor

    def Jacobian_solver(self) -> float:
        """One Jacobi sweep on _mat_A raw_solved = rhs, then the RMS of the new
        residual, sqrt(sum |rhs - A u|^2 / n) (BEM_manager.py:803-821; the
        reference defines it but its run never calls it).  The reference
        updates raw_solved in place inside one parallel loop, so a row may
        read neighbours of either sweep; here every row reads the previous
        sweep (plain Jacobi): u <- u + (rhs - A u) / diag(A).  The products run
        on the device through bem_gemv."""
        n = self.N_Neumann + self.M_Dirichlet
        A, u, b = self._mat_A, self.raw_solved, self.rhs[:n]
        r = b.clone()
        self.engine.gemv(A, u, r, alpha=-1.0, beta=1.0)
        u += r / torch.diagonal(A)
        r.copy_(b)
        self.engine.gemv(A, u, r, alpha=-1.0, beta=1.0)
        return float(torch.sqrt((r.abs() ** 2).sum() / n))

    # relative diagonal shift of the energy-scaling block before its Cholesky factorisation
    SCALING_SHIFT = 1e-10

    @classmethod
    def _shifted(cls, MV: torch.Tensor) -> torch.Tensor:
        """MV + shift * max|MV| * I.  The reference factors MV itself, but the
        W block of the k = 0 operator it is taken from is singular (constants
        are in the null space of the Laplace hypersingular operator), so
        whether that Cholesky succeeds depends on rounding; the fixed relative
        shift makes the scaling well defined and reproducible."""
        d = cls.SCALING_SHIFT * float(MV.abs().max())
        return MV + d * torch.eye(MV.shape[0], dtype=MV.dtype, device=MV.device)

    def compute_inv_norm(self, A: torch.Tensor, A_type: int, method: str = "svd", return_cond: bool = False):
        """||A^{-1}|| in the energy-scaled norm (BEM_manager.py:874-920).

        The scaling (L the Cholesky factor of blockdiag(W, V) of A for A_type
        1, of blockdiag(K', K) for A_type 2, shifted by `_shifted`) is formed
        on the first call and kept, as in the reference (whose sweep makes that
        call at k = 0): L^{-1} by bem_chol_inverse.  The scaled operator
        S = L^{-1} A L^{-H} (block-diagonal left factor for the augmented
        2n x n operator) is formed by bem_gemm in FP64; its smallest singular
        value sigma_min gives the result 1 / sigma_min.  method "svd" takes all
        singular values as the reference does (torch.linalg.svdvals, the
        reference's own call); "iterative" estimates the extreme ones by
        block Krylov spaces on this library's kernels
        (sweep.extreme_singular_values); "none" only forms the scaling.  With
        return_cond the result is (1 / sigma_min, sigma_max / sigma_min,
        Krylov blocks)."""
        n = self.N_Neumann + self.M_Dirichlet
        top = A[:n]
        if self._L1_inv is None and A_type == 1:
            MV = torch.zeros_like(top)
            Do, No = self._Dirichlet_offset_i, self._Neumann_offset_i
            MV[Do:Do + self.M_Dirichlet, self._Dirichlet_offset_j:self._Dirichlet_offset_j + self.M_Dirichlet] = \
                self.get_W_part(top)
            MV[No:No + self.N_Neumann, self._Neumann_offset_j:self._Neumann_offset_j + self.N_Neumann] = \
                self.get_V_part(top)
            self._L1_inv = self._scaling_inverse((MV + MV.transpose(0, 1)) / 2.0)
            self._L2_inv = None
        elif self._L2_inv is None and A_type == 2:
            MV = torch.block_diag(self.get_adj_K_part(top), self.get_K_part(top))
            self._L2_inv = self._scaling_inverse(MV)
            self._L1_inv = None
        if method == "none":
            return None
        Linv = self._L1_inv if A_type == 1 else self._L2_inv
        if A.shape[0] not in (n, 2 * n):
            raise NotImplementedError("the norm analysis takes the square operator (n x n) or the augmented one "
                                      "(2n x n)")
        blocks = []
        T = torch.zeros(n, n, dtype=A.dtype, device=A.device)
        for r0 in range(0, A.shape[0], n):
            T.zero_()
            self.engine.gemm(Linv, A[r0:r0 + n].contiguous(), T, a_lower=True)
            Sb = torch.zeros(n, n, dtype=A.dtype, device=A.device)
            self.engine.gemm(T, Linv, Sb, conj_b=True, b_upper=True)
            blocks.append(Sb)
        del T
        if method == "svd":
            sv = torch.linalg.svdvals(torch.cat(blocks, 0))
            smin, smax, its = float(sv.min()), float(sv.max()), 0
        elif method == "iterative":
            from .sweep import extreme_singular_values
            smin, smax, its = extreme_singular_values(self.engine, blocks, tol=self.norm_tol, maxit=self.norm_maxit,
                                                      info=self._norm_info)
        else:
            raise ValueError(method)
        inv = 1.0 / smin if smin > 0 else float("inf")
        if return_cond:
            return inv, smax * inv, its
        return inv

    def _scaling_inverse(self, MV: torch.Tensor) -> torch.Tensor:
        """L^{-1} for the Cholesky factor L of MV, shifted (`_shifted`; the
        lower triangle is read, as torch.linalg.cholesky reads it), on this
        library's FP64 Cholesky and triangular inverse (bem_chol_inverse)."""
        H = self._shifted(MV).contiguous()
        X, info = self.engine.chol_inverse(H)
        if int(info.item()) != 0:
            raise torch.linalg.LinAlgError("the energy-scaling block is not positive definite (Cholesky pivot "
                                           f"{int(info.item()) - 1})")
        return X

    def get_mat_A1_inv_norm(self, k: float, method: str = "svd"):
        """A_I = P^-_o - P^+_i (BEM_manager.py:922-936)."""
        from .sweep import transmission_operator
        return self.compute_inv_norm(transmission_operator(self, k, 1, augmented=False), 1, method=method)

    def get_mat_A2_inv_norm(self, k: float, method: str = "svd"):
        """A_II = P^-_o + P^+_i (BEM_manager.py:938-950)."""
        from .sweep import transmission_operator
        return self.compute_inv_norm(transmission_operator(self, k, 2, augmented=False), 2, method=method)

    def _augment(self, k, need_recompute_matrix_layers):
        A = self._mat_A.clone()
        self._mat_A.zero_()
        if need_recompute_matrix_layers:
            self.matrix_layer_forward(k=k, sqrt_n=self._sqrt_ni, scope_type=int(ScopeType.INTERIOR))
        self.assemble_matA(assemble_type=int(AssembleType.ADD_P_PLUS), multiplier=1.0)
        return torch.cat((A, self._mat_A.clone()), 0)

    def get_augment_mat_A1_inv_norm(self, k: float, need_recompute_matrix_layers: bool, method: str = "svd"):
        """[A; P^+_i] with A the current operator (BEM_manager.py:952-969)."""
        return self.compute_inv_norm(self._augment(k, need_recompute_matrix_layers), 1, method=method)

    def get_augment_mat_A2_inv_norm(self, k: float, need_recompute_matrix_layers: bool, method: str = "svd"):
        """(BEM_manager.py:971-988)."""
        return self.compute_inv_norm(self._augment(k, need_recompute_matrix_layers), 2, method=method)

    def fused_assembly_call(self):
        """The one C-ABI call of the fused Dirichlet pass: V (far pairs in
        the symmetric sweep, near pairs in FP64) accumulated into the V block
        and K g into the right-hand side (both must be zeroed by the caller)."""
        rc = self.rhs_constructor
        sp = self.space("charge", self.shape_func_degree_Neumann, "N", int(CellFluxType.NEUMANN_TOBESOLVED))
        rows = self.space("charge", self.shape_func_degree_Neumann, "N", int(CellFluxType.NEUMANN_TOBESOLVED),
                          offset=self._Neumann_offset_i)
        data = self.space("data", self.shape_func_degree_Dirichlet, "N")
        desc = self.op_desc(L.OP_V, self._k, 1.0)
        self.engine.assemble_dirichlet(desc, sp, sp, self.single_layer._Vmat, rows, data, rc._Dirichlet_boundary,
                                       rc._rhs_vec, scale=1.0, scale_k=1.0, conj_g=self.conj_data)

    def run(self):
        """BEMManager.run (BEM_manager.py:990-1030).  The exact traces do not
        depend on the solution, so they are queued before the solve, whose
        refinement is the step's one host synchronisation; the per-vertex
        splat and the colour and position buffers of the reference's window
        (headless here) follow it."""
        self.assemble_system()
        self.compute_analytical_raw_solved()
        self.solve()
        self.splat_u_from_raw_solved_to_vertices()
        self.compute_color()
        self.set_mesh_instances()

    def _calderon_fusable(self) -> bool:
        """Transmission with P0 Neumann and P1 Dirichlet unknowns on one
        panel loop: every operator block comes from the same panel pairs."""
        if not (self.fuse_calderon and self._is_transmission and self._dim == 3 and self.N_Neumann > 0
                and self.M_Dirichlet > 0 and self.shape_func_degree_Neumann == 0
                and self.shape_func_degree_Dirichlet == 1):
            return False
        key = "calderon_fusable"
        if key not in self._dev_cache:
            mm = self.mesh
            self._dev_cache[key] = bool(np.array_equal(mm.loop_panels("N"), mm.loop_panels("D")))
        return self._dev_cache[key]

    def _assemble_transmission_fused(self):
        """matrix_layer_forward + assemble_matA(ADD_P_MINUS) at sqrt_no, the
        right-hand side, then matrix_layer_forward + assemble_matA(ADD_P_PLUS)
        at sqrt_ni (BEM_manager.py:995-1006), with the operators of both
        scopes from one call: _mat_A receives P-_o = 1/2 M - M_o and _mat_P
        receives P+_i = 1/2 M + M_i; rhs[:n] = P-_o conj(f), as the reference
        forms it before the interior scope is added; then _mat_A += _mat_P."""
        n = self.N_Neumann + self.M_Dirichlet
        if self._mat_P is None:
            self._mat_P = torch.zeros(n, n, dtype=self.torch_dtype, device=self.device)
        else:
            self._mat_P.zero_()
        neu = self.space("charge", 0, "N", int(CellFluxType.NEUMANN_TOBESOLVED), offset=self._Neumann_offset_i)
        dir_ = self.space("charge", 1, "D", int(CellFluxType.DIRICHLET_TOBESOLVED), offset=self._Dirichlet_offset_i)
        desc = self.op_desc(L.OP_V, self._k, 1.0)
        ks, k2s = [], []
        for sqrt_n in (self._sqrt_no, self._sqrt_ni):
            d = self.op_desc(L.OP_V, self._k, sqrt_n)
            ks.append(d.k)
            k2s.append(d.k2)
        self.engine.assemble_calderon(desc, ks, k2s, neu, dir_, [self._mat_A, self._mat_P], [-1.0, 1.0])
        # the identity parts of ADD_P_MINUS and ADD_P_PLUS (identity_layer_3d.py:148-196)
        md = self.space("charge", 1, "D", int(CellFluxType.DIRICHLET_TOBESOLVED), offset=self._Dirichlet_offset_j)
        for X in (self._mat_A, self._mat_P):
            self.engine.mass(neu, md, out=X, scale=0.5, out_t=X, scale_t=0.5)
        self.rhs_constructor.set_boundaries(scope_type=int(ScopeType.INTERIOR), sqrt_ni=self._sqrt_ni,
                                            sqrt_no=self._sqrt_no)
        self.assemble_rhs()
        self._mat_A.add_(self._mat_P)
        self.set_scope_type(int(ScopeType.INTERIOR))

    def assemble_system(self):
        """The part of `run` before the solve (BEM_manager.py:990-1018): the
        operator into _mat_A and the right-hand side into rhs, at self._k."""
        self._mat_A.zero_()
        if self._is_transmission and self._calderon_fusable():
            self._assemble_transmission_fused()
        elif self._is_transmission:
            self.matrix_layer_forward(k=self._k, sqrt_n=self._sqrt_no, scope_type=int(ScopeType.EXTERIOR))
            self.assemble_matA(assemble_type=int(AssembleType.ADD_P_MINUS), multiplier=1.0)
            self.rhs_constructor.set_boundaries(scope_type=int(ScopeType.INTERIOR), sqrt_ni=self._sqrt_ni,
                                                sqrt_no=self._sqrt_no)
            self.assemble_rhs()
            self.matrix_layer_forward(k=self._k, sqrt_n=self._sqrt_ni, scope_type=int(ScopeType.INTERIOR))
            self.assemble_matA(assemble_type=int(AssembleType.ADD_P_PLUS), multiplier=1.0)
        elif self._fusable():
            self._run_dirichlet_fused()
        else:
            self.matrix_layer_forward(k=self._k, scope_type=self._scope_type)
            self.assemble_matA(assemble_type=int(AssembleType.ADD_M), multiplier=-1.0)
            self.rhs_constructor.set_boundaries(scope_type=self._scope_type, sqrt_ni=self._sqrt_ni,
                                                sqrt_no=self._sqrt_no)
            self.rhs_layer_forward(k=self._k, scope_type=self._scope_type)
            self.assemble_rhs()

    def autotune(self, tuner=None) -> dict:
        """Choose the launch shapes of this problem's hot calls on this GPU
        (bem_b200.tuning): the form of the fused Calderon sweep (transmission
        problems it takes; candidates 2: both wavenumbers in one scalar
        launch, 4 / 5: both packed into FP32x2 lanes (moments in registers /
        shared memory), 3: packed FP32x2 per
        wavenumber, 1: scalar per wavenumber; the packed forms in mixed
        precision only),
        timed on assemble_system, and for the least-squares solver the form
        of the tensor-core normal matrix (1: one CTA per 128 x 128 tile with
        eight epilogue warps, 3: with sixteen, 2: CTA pairs on 256 x 128
        tiles; mixed precision), the band width of the
        normal matrix's tile order (1, 12, 8, 16), timed on the normal matrix,
        and the Cholesky panel width (512, 1024, 2048), timed on its
        factorisation.  Cached choices are applied without
        timing.  Returns {key name: value}."""
        from ..tuning import Autotuner
        tuner = tuner or Autotuner(self.engine)
        n = self.N_Neumann + self.M_Dirichlet
        wl = f"{self._simulation_parameters['kernel']}/n{n}/Q{self._GaussQR}/{self.precision}-{self.solve_precision}"
        out = {}
        if self._is_transmission and self._calderon_fusable():
            groups = [2, 4, 5, 3, 1] if self.precision == "mixed" else [2, 1]
            out["calderon_group"] = tuner.tune(wl + "/calderon", L.TUNE_CALDERON_GROUP, groups,
                                               self.assemble_system)
        nbs = [512, 1024, 2048]
        mixed = self.solve_precision == "mixed"
        pairs = [1, 3, 2] if mixed else [1]
        if (self._is_transmission and self.solver == "lstsq" and tuner.cached(wl + "/chol", L.TUNE_CHOL_NB, nbs)
                and tuner.cached(wl + "/gram", L.TUNE_GRAM_BAND, [1, 12, 8, 16])
                and (not mixed or tuner.cached(wl + "/gram_pair", L.TUNE_GRAM_PAIR, pairs))):
            if mixed:
                out["gram_pair"] = tuner.cached(wl + "/gram_pair", L.TUNE_GRAM_PAIR, pairs)
            out["chol_nb"] = tuner.cached(wl + "/chol", L.TUNE_CHOL_NB, nbs)
            out["gram_band"] = tuner.cached(wl + "/gram", L.TUNE_GRAM_BAND, [1, 12, 8, 16])
        elif self._is_transmission and self.solver == "lstsq":
            self.assemble_system()
            A, P = self.transmission_blocks()
            Nm = torch.empty(n, n, dtype=A.dtype, device=A.device)
            d = torch.empty(n, dtype=torch.float64, device=A.device)
            if mixed:
                # the CTA-pair form (256 x 128 tiles, column order) against the
                # one-CTA form; the band width below only shapes the latter
                out["gram_pair"] = tuner.tune(wl + "/gram_pair", L.TUNE_GRAM_PAIR, pairs,
                                              lambda: self.engine.gram(A, P, Nm, d, tensor_cores=True))
            bands = [1] if out.get("gram_pair") == 2 else [1, 12, 8, 16]  # the pair form has one tile order
            out["gram_band"] = tuner.tune(wl + "/gram", L.TUNE_GRAM_BAND, bands,
                                          lambda: self.engine.gram(A, P, Nm, d, tensor_cores=mixed))
            W = torch.empty_like(Nm)

            def factor():
                W.copy_(Nm)
                self.engine.chol_factor(W, tensor_cores=mixed)

            out["chol_nb"] = tuner.tune(wl + "/chol", L.TUNE_CHOL_NB, nbs, factor)
            del W, Nm, A, P
        return out

    def kill(self):
        self.initialized = False
        for lay in ("single_layer", "double_layer", "adj_double_layer", "hypersingular_layer", "identity_layer",
                    "rhs_constructor"):
            obj = getattr(self, lay, None)
            if obj is not None:
                obj.kill()
        self._mat_A = None
        self._mat_P = None
        self.rhs = None
        self.raw_solved = None
        if getattr(self, "engine", None) is not None:
            self.engine.close()
            self.engine = None
