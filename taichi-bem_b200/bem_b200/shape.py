"""Shape derivatives of the Laplace interior Dirichlet problem.

Forward (the reference's Dirichlet pipeline, `BEMManager.run`,
BEM_manager.py:990-1030): for vertex positions X,
    V(X) t = (1/2 M(X) + K(X)) g(X),     g = u(X) at the vertices,
with V the P0 single layer, K the P0 x P1 double layer and M the P0 x P1 mass
matrix; t are the Neumann DOFs.  `DirichletShapeSolve` wraps this as a
`torch.autograd.Function` of X.  Its backward pass is the adjoint method:
    V^T lam = dJ/dt  (with the factor of the forward solve, `_solve_Vt`),
    dJ/dX = - d(lam^T V t)/dX + d(lam^T K g)/dX + 1/2 d(lam^T M g)/dX
            + [(1/2 M + K)^T lam]_v grad u(X_v),
where the first two terms come from the library's adjoint kernels
(bem_adjoint_vertices: every quadrature point recomputed in FP64, nothing
stored by the forward pass) and the mass term is closed-form
(M_{i,b} = J_i / 6 with J_i = 2 x area_i, exact for the quadrature used).
The reference has no derivatives; this is the shape-gradient workload.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib as L
from .engine import DeviceSpace, Engine


class DirichletShape:
    """One mesh topology (panels) and Dirichlet data u, gradient grad_u."""

    def __init__(self, panels: np.ndarray, u, grad_u, gauss_qr: int = 5, precision: str = "mixed",
                 device="cuda", quirk: bool = True, refine_tol: float = 1e-13, solver: str | None = None):
        """precision: quadrature of the forward assembly ("mixed": FP32 far
        field, "fp64"); solver: "mixed" (FP32 tile LU + FP64 refinement to
        refine_tol) or "fp64" (partial-pivoting LU), by default following
        precision."""
        self.f = np.ascontiguousarray(panels, np.int32)
        self.nt = len(self.f)
        self.u, self.grad_u = u, grad_u
        self.Q = int(gauss_qr)
        self.precision = precision
        self.solver = solver or precision
        self.quirk = quirk
        self.refine_tol = refine_tol
        self.device = torch.device(device)
        self.engine = Engine(self.device)
        ids = np.arange(self.nt, dtype=np.int32)
        self.P0 = DeviceSpace.from_numpy(ids, 1, ids, self.device)
        self.P1 = DeviceSpace.from_numpy(ids, 3, self.f.reshape(-1).copy(), self.device)
        self.tris = torch.as_tensor(self.f.astype(np.int64), device=self.device)

    def _desc(self, op, precision=None):
        prec = L.PREC_MIXED if (precision or self.precision) == "mixed" else L.PREC_FP64
        return Engine.op_desc(op, False, 0.0, 0.0, quirk=self.quirk, precision=prec)

    def set_vertices(self, X: torch.Tensor):
        v = X.detach().to("cpu", torch.float64).numpy()
        self.engine.set_mesh(np.ascontiguousarray(v), self.f, self.Q)
        self.nv = len(v)

    def forward(self, X: torch.Tensor):
        """t (Neumann DOFs) for vertex positions X [nv, 3]; keeps what the
        backward pass reuses (the factor of V, t, g)."""
        self.set_vertices(X)
        eng = self.engine
        Xd = X.detach().to(self.device, torch.float64)
        g = self.u(Xd).contiguous()
        V = torch.zeros(self.nt, self.nt, dtype=torch.float64, device=self.device)
        eng.assemble(self._desc(L.OP_V), self.P0, self.P0, V)
        b = torch.zeros(self.nt, dtype=torch.float64, device=self.device)
        eng.apply(self._desc(L.OP_K), self.P0, self.P1, g, b)
        eng.mass(self.P0, self.P1, x=g, y=b, scale=0.5)
        if self.solver == "fp64":
            LU = V.clone()
            piv, _ = eng.lu_factor(LU)
            t = b.clone()
            eng.lu_solve(LU, piv, t)
            self._factor = ("fp64", LU, piv, None)
        else:
            LU = V.to(torch.float32)
            piv, dinv, _ = eng.lu_factor_tiled(LU)
            t = torch.zeros_like(b)
            eng.refine_solve(V, LU, piv, b, t, tol=self.refine_tol, maxit=60, dinv=dinv, accept=1e-10)
            self._factor = ("mixed", LU, piv, dinv)
        self._V, self._g, self._t, self._X = V, g, t, Xd
        return t

    def _solve_Vt(self, rhs: torch.Tensor) -> torch.Tensor:
        """lam with V^T lam = rhs.  With the corrected near-field maps
        (quirk = False) V is symmetric and the forward factor solves it.  The
        reference's maps (quirk = True) integrate an edge or vertex pair (i, j)
        and (j, i) on different points, so V is symmetric only up to its near
        field: the mixed path refines against V^T in FP64 with the FP32 factor
        of V as preconditioner (V^T - V is small); the plain path factors V^T."""
        kind, LU, piv, dinv = self._factor
        rhs = rhs.contiguous()
        if not self.quirk:
            A_hi = self._V
        else:
            A_hi = self._V.transpose(0, 1).contiguous()
        if kind == "fp64":
            if self.quirk:
                LU = A_hi.clone()
                piv, _ = self.engine.lu_factor(LU)
            x = rhs.clone()
            self.engine.lu_solve(LU, piv, x)
            return x
        x = torch.zeros_like(rhs)
        self.engine.refine_solve(A_hi, LU, piv, rhs, x, tol=self.refine_tol, maxit=200, dinv=dinv, accept=1e-10)
        return x

    def backward(self, grad_t: torch.Tensor) -> torch.Tensor:
        """dJ/dX [nv, 3] for dJ/dt = grad_t (after `forward`)."""
        eng = self.engine
        lam = self._solve_Vt(grad_t.to(torch.float64).contiguous())
        grad = torch.zeros(self.nv, 3, dtype=torch.float64, device=self.device)
        # -d(lam^T V t)/dX and +d(lam^T K g)/dX from the adjoint kernels
        eng.adjoint_vertices(self._desc(L.OP_V, "fp64"), self.P0, self.P0, (-lam).contiguous(), self._t, grad)
        eng.adjoint_vertices(self._desc(L.OP_K, "fp64"), self.P0, self.P1, lam, self._g, grad)
        # 1/2 d(lam^T M g)/dX: M_{i,b} = J_i / 6, dJ_i/dP_a = n_i x (P_{a+2} - P_{a+1})
        X = self._X
        P = X[self.tris]                                    # [nt, 3 vertices, 3]
        nraw = torch.linalg.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 1])
        n = nraw / torch.linalg.norm(nraw, dim=1, keepdim=True)
        s = 0.5 * lam * self._g[self.tris].sum(1) / 6.0     # [nt]
        for a in range(3):
            e = P[:, (a + 2) % 3] - P[:, (a + 1) % 3]
            grad.index_add_(0, self.tris[:, a], s[:, None] * torch.linalg.cross(n, e))
        # data term: [(1/2 M + K)^T lam]_v grad u(X_v)
        w = torch.zeros(self.nv, dtype=torch.float64, device=self.device)
        Kt = torch.zeros(self.nt, self.nv, dtype=torch.float64, device=self.device)
        eng.assemble(self._desc(L.OP_K, "fp64"), self.P0, self.P1, Kt)
        w += Kt.transpose(0, 1) @ lam
        area6 = (torch.linalg.norm(nraw, dim=1) / 6.0) * lam  # (1/2 M)^T lam: 1/2 * J_i / 6 per panel vertex
        for a in range(3):
            w.index_add_(0, self.tris[:, a], 0.5 * area6)
        grad += w[:, None] * self.grad_u(X)
        return grad


class DirichletShapeSolve(torch.autograd.Function):
    """t = solve(X) for a `DirichletShape` problem, differentiable in X."""

    @staticmethod
    def forward(ctx, X, problem: DirichletShape):
        ctx.problem = problem
        return problem.forward(X)

    @staticmethod
    def backward(ctx, grad_t):
        return ctx.problem.backward(grad_t).to(grad_t.device), None


def point_source(x0=(2.0, 2.0, 2.0)):
    """u = 1/|x - x0| and its gradient (torch callables on [m, 3])."""
    def u(x):
        c = torch.as_tensor(x0, dtype=x.dtype, device=x.device)
        return 1.0 / torch.linalg.norm(x - c, dim=1)

    def grad_u(x):
        c = torch.as_tensor(x0, dtype=x.dtype, device=x.device)
        d = x - c
        return -d / torch.linalg.norm(d, dim=1, keepdim=True) ** 3
    return u, grad_u
