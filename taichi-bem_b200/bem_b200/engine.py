"""Device engine: one libbem_b200 context, a mesh on the GPU, and typed calls.

All tensors passed in are CUDA tensors; every call is issued on the current
torch CUDA stream.  Nothing here computes on the CPU: the engine raises when
the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L


def _stream_ptr():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def upload(a, device, dtype=None) -> torch.Tensor:
    """A host array (numpy or list) as a tensor on `device`.  For a CUDA
    device the values are staged in pinned memory and copied on the current
    stream without blocking the host: kernels already queued keep the GPU busy
    while the host prepares the next launch (a pageable copy would wait for
    them to finish).  torch's caching host allocator keeps the staging block
    until the copy has run."""
    t = torch.as_tensor(np.ascontiguousarray(a) if isinstance(a, np.ndarray) else a, dtype=dtype)
    device = torch.device(device)
    if device.type != "cuda":
        return t.to(device)
    return t.pin_memory().to(device, non_blocking=True)


def _dtype_code(t: torch.Tensor) -> int:
    return {torch.float64: L.F64, torch.complex128: L.C128, torch.float32: L.F32,
            torch.complex64: L.C64}[t.dtype]


@dataclass
class DeviceSpace:
    """One side of an operator block: global panel ids and a dof table
    [n_panels, nb] (-1 = skipped), both int32 on the device.  ``max_panel``
    and ``max_dof`` are checked against the mesh and the output extents
    before every launch (an out-of-range index is rejected on the host)."""
    panels: torch.Tensor
    nb: int
    dof: torch.Tensor
    max_panel: int = -1
    max_dof: int = -1

    @staticmethod
    def from_numpy(panels, nb, dof, device):
        pn = np.ascontiguousarray(panels, dtype=np.int32).reshape(-1)
        dn = np.ascontiguousarray(dof, dtype=np.int32).reshape(-1)
        if dn.size != pn.size * nb:
            raise ValueError("dof table must have n_panels * nb entries")
        if pn.size and pn.min() < 0:
            raise ValueError("negative panel index")
        if pn.size != np.unique(pn).size:
            raise ValueError("a panel may appear only once per space")
        p = upload(pn, device)
        d = upload(dn, device)
        return DeviceSpace(p, int(nb), d, int(pn.max()) if pn.size else -1, int(dn.max()) if dn.size else -1)

    def shifted(self, offset: int):
        """Same space with every valid dof moved by `offset` (block placement)."""
        d = torch.where(self.dof >= 0, self.dof + int(offset), self.dof)
        return DeviceSpace(self.panels, self.nb, d, self.max_panel, self.max_dof + int(offset) if self.max_dof >= 0
                           else -1)

    def c(self):
        return L.Space(int(self.panels.numel()), self.panels.data_ptr() if self.panels.numel() else None, self.nb,
                       self.dof.data_ptr() if self.dof.numel() else None)

    @property
    def n_panels(self):
        return int(self.panels.numel())


class Engine:
    """Owns one bem_ctx.  ``set_mesh`` uploads a mesh and builds the device
    geometry and the near-pair list; ``assemble``/``apply``/``mass`` evaluate
    operator blocks; ``lu_factor``/``lu_solve``/``refine_solve`` solve."""

    def __init__(self, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("bem_b200 needs a CUDA device (no CPU fallback)")
        self.device = torch.device(device if device is not None else "cuda")
        self.lib = L.load()
        with torch.cuda.device(self.device):
            h = ctypes.c_void_p()
            rc = self.lib.bem_ctx_create(ctypes.byref(h))
            if rc != 0:
                raise L.BemError(rc, "bem_ctx_create failed")
        self.ctx = h
        self.nt = self.nv = 0
        self.Q = 0
        self.dim = 3

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.bem_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise L.BemError(rc, self.lib.bem_last_error(self.ctx).decode())

    @property
    def launches(self) -> int:
        return int(self.lib.bem_launch_count(self.ctx))

    # -- mesh ---------------------------------------------------------------
    def set_mesh(self, vertices, panels, gauss_qr: int, dim: int = 3):
        """Upload a triangle mesh (dim 3: vertices [nv,3], panels [nt,3]) or a
        segment mesh (dim 2: vertices [nv,2], panels [nt,2])."""
        if dim not in (2, 3):
            raise ValueError("dim must be 2 or 3")
        v = np.ascontiguousarray(np.asarray(vertices, dtype=np.float64).reshape(-1, dim))
        f = np.ascontiguousarray(np.asarray(panels, dtype=np.int32).reshape(-1, dim))
        fn = self.lib.bem_mesh_set if dim == 3 else self.lib.bem_mesh_set_2d
        with torch.cuda.device(self.device):
            self._check(fn(self.ctx, v.ctypes.data, f.ctypes.data, len(v), len(f), int(gauss_qr)))
        self.nv, self.nt, self.Q, self.dim = len(v), len(f), int(gauss_qr), dim
        self.vertices_host, self.panels_host = v, f

    @property
    def near_pairs(self) -> int:
        return int(self.lib.bem_near_pair_count(self.ctx))

    def near_pair_list(self) -> np.ndarray:
        """The device-built near-pair list as int32 [n, 4]: (test panel,
        trial panel, relation, packed parameter orders) (bem_near_pair_list)."""
        out = np.zeros((self.near_pairs, 4), np.int32)
        if out.size:
            self._check(self.lib.bem_near_pair_list(self.ctx, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def geometry(self):
        areas = torch.empty(self.nt, dtype=torch.float64, device=self.device)
        normals = torch.empty(self.nt, self.dim, dtype=torch.float64, device=self.device)
        self._check(self.lib.bem_mesh_geometry(self.ctx, _ptr(areas), _ptr(normals), _stream_ptr()))
        return areas, normals

    # -- operators ------------------------------------------------------------
    @staticmethod
    def op_desc(op, helmholtz, k=0.0, k2=0.0, quirk=True, precision=L.PREC_FP64, deriv_k=False):
        """deriv_k: the operator of the kernel's k-derivative at fixed k2
        (Helmholtz; bem_assemble and bem_apply)."""
        return L.OpDesc(int(op), L.KERNEL_HELMHOLTZ if helmholtz else L.KERNEL_LAPLACE, float(k), float(k2),
                        1 if quirk else 0, int(precision), 1 if deriv_k else 0)

    def _check_spaces(self, test, trial, nrow, ncol):
        for sp in (test, trial):
            if sp.max_panel >= self.nt:
                raise ValueError(f"panel index {sp.max_panel} out of range for a mesh of {self.nt} panels")
        if test.max_dof >= nrow or trial.max_dof >= ncol:
            raise ValueError(f"dof out of range: rows {test.max_dof} >= {nrow} or cols {trial.max_dof} >= {ncol}")

    def assemble(self, desc: L.OpDesc, test: DeviceSpace, trial: DeviceSpace, out: torch.Tensor, scale=1.0,
                 out_t: torch.Tensor | None = None, scale_t=0.0):
        """out[row, col] += scale * A(row, col) (and out_t[col, row] += scale_t * A)."""
        assert out.is_cuda and out.dim() == 2 and out.stride(1) == 1
        self._check_spaces(test, trial, out.shape[0], out.shape[1])
        if out_t is not None:
            assert out_t.dtype == out.dtype and out_t.stride(0) == out.stride(0)
            self._check_spaces(trial, test, out_t.shape[0], out_t.shape[1])
        ts, rs = test.c(), trial.c()
        self._check(self.lib.bem_assemble(self.ctx, ctypes.byref(desc), ctypes.byref(ts), ctypes.byref(rs),
                                          _dtype_code(out), _ptr(out), out.stride(0), float(scale), _ptr(out_t),
                                          float(scale_t), _stream_ptr()))

    def apply(self, desc: L.OpDesc, test: DeviceSpace, trial: DeviceSpace, x: torch.Tensor, y: torch.Tensor,
              scale=1.0, conj_x=False):
        """y[row] += scale * sum_col A(row, col) x[col] (x conjugated if conj_x)."""
        assert x.dtype == y.dtype and x.is_contiguous() and y.is_contiguous()
        self._check_spaces(test, trial, y.numel(), x.numel())
        ts, rs = test.c(), trial.c()
        self._check(self.lib.bem_apply(self.ctx, ctypes.byref(desc), ctypes.byref(ts), ctypes.byref(rs),
                                       _dtype_code(y), _ptr(x), _ptr(y), float(scale), int(bool(conj_x)),
                                       _stream_ptr()))

    def assemble_dirichlet(self, desc: L.OpDesc, test: DeviceSpace, trial: DeviceSpace, out: torch.Tensor,
                           rows: DeviceSpace, data: DeviceSpace, g: torch.Tensor, y: torch.Tensor, scale=1.0,
                           scale_k=1.0, conj_g=False):
        """One pass: out += scale * V (test x trial) and y += scale_k * K g."""
        assert out.is_cuda and out.dim() == 2 and out.stride(1) == 1 and g.is_contiguous() and y.is_contiguous()
        self._check_spaces(test, trial, out.shape[0], out.shape[1])
        self._check_spaces(rows, data, y.numel(), g.numel())
        ts, rs, ws, ds = test.c(), trial.c(), rows.c(), data.c()
        self._check(self.lib.bem_assemble_dirichlet(self.ctx, ctypes.byref(desc), ctypes.byref(ts), ctypes.byref(rs),
                                                    _ptr(out), out.stride(0), float(scale), ctypes.byref(ws),
                                                    ctypes.byref(ds), _ptr(g), _ptr(y), float(scale_k),
                                                    int(bool(conj_g)), _stream_ptr()))

    def assemble_calderon(self, desc: L.OpDesc, ks, k2s, neu: DeviceSpace, dir_: DeviceSpace, outs, coefs):
        """outs[w] += coefs[w] * [K -V; -W -K'](ks[w]) with the reference's
        block placement (bem_assemble_calderon): one sweep over the unordered
        separate panel pairs serves V, K, K^T and W of every wavenumber."""
        nk = len(ks)
        assert 1 <= nk <= 2 and len(k2s) == nk == len(outs) == len(coefs)
        o0 = outs[0]
        for o in outs:
            assert o.is_cuda and o.dim() == 2 and o.stride(1) == 1 and o.dtype == o0.dtype
            assert o.stride(0) == o0.stride(0) and o.shape == o0.shape
        self._check_spaces(neu, neu, o0.shape[0], o0.shape[1])
        self._check_spaces(dir_, dir_, o0.shape[0], o0.shape[1])
        kk = (ctypes.c_double * nk)(*[float(v) for v in ks])
        k2 = (ctypes.c_double * nk)(*[float(v) for v in k2s])
        cf = (ctypes.c_double * nk)(*[float(v) for v in coefs])
        po = (ctypes.c_void_p * nk)(*[o.data_ptr() for o in outs])
        ns, ds = neu.c(), dir_.c()
        self._check(self.lib.bem_assemble_calderon(self.ctx, ctypes.byref(desc), nk, kk, k2, ctypes.byref(ns),
                                                   ctypes.byref(ds), po, cf, o0.stride(0), _stream_ptr()))

    def assemble_batch(self, desc: L.OpDesc, test: DeviceSpace, trial: DeviceSpace, ks, k2s, outs, scales,
                       outs_t=None, scales_t=None):
        """outs[w][row, col] += scales[w] * A(ks[w])(row, col) (and, where
        outs_t[w] is given, outs_t[w][col, row] += scales_t[w] * A(ks[w])) for
        the Helmholtz operator desc.op at every wavenumber of ks, W's mass
        coefficient k2s[w] (bem_assemble_batch: each separate pair's geometry
        evaluated once for 2 or 4 wavenumbers)."""
        nk = len(ks)
        assert 1 <= nk <= L.MAX_KBATCH and len(k2s) == nk == len(outs) == len(scales)
        o0 = outs[0]
        for o in outs:
            assert o.is_cuda and o.dim() == 2 and o.stride(1) == 1 and o.dtype == o0.dtype == torch.complex128
            assert o.stride(0) == o0.stride(0)
            self._check_spaces(test, trial, o.shape[0], o.shape[1])
        dbl = ctypes.c_double * nk
        po = (ctypes.c_void_p * nk)(*[o.data_ptr() for o in outs])
        pt, st = None, None
        if outs_t is not None:
            assert len(outs_t) == nk and scales_t is not None and len(scales_t) == nk
            for o in outs_t:
                if o is not None:
                    assert o.dtype == o0.dtype and o.stride(0) == o0.stride(0) and o.stride(1) == 1
                    self._check_spaces(trial, test, o.shape[0], o.shape[1])
            pt = (ctypes.c_void_p * nk)(*[None if o is None else o.data_ptr() for o in outs_t])
            st = dbl(*[float(v) for v in scales_t])
        ts, rs = test.c(), trial.c()
        self._check(self.lib.bem_assemble_batch(self.ctx, ctypes.byref(desc), ctypes.byref(ts), ctypes.byref(rs), nk,
                                                dbl(*[float(v) for v in ks]), dbl(*[float(v) for v in k2s]), po,
                                                o0.stride(0), dbl(*[float(v) for v in scales]), pt, st,
                                                _stream_ptr()))

    def gram(self, A: torch.Tensor, P: torch.Tensor, out: torch.Tensor, colscale: torch.Tensor, tensor_cores=True):
        """out = D (A^H A + P^H P) D (full Hermitian, complex64/128 or
        float32/64), colscale = D (bem_gram): FP16-split tcgen05 products with
        FP64 sums (tensor_cores) or FP64 DMMA products."""
        n = A.shape[0]
        for M in (A, P):
            assert M.is_cuda and M.shape == (n, n) and M.stride(1) == 1 and M.stride(0) == A.stride(0)
            assert M.dtype == A.dtype
        assert out.shape == (n, n) and out.stride(1) == 1 and colscale.dtype == torch.float64
        assert colscale.numel() == n and colscale.is_contiguous()
        method = L.PREC_MIXED if tensor_cores else L.PREC_FP64
        self._check(self.lib.bem_gram(self.ctx, _dtype_code(A), _ptr(A), _ptr(P), n, A.stride(0), _ptr(colscale),
                                      method, _dtype_code(out), _ptr(out), out.stride(0), _stream_ptr()))
        return out, colscale

    def chol_factor(self, A: torch.Tensor, tensor_cores=True):
        """In-place Cholesky of the Hermitian positive definite A (complex128
        or float64, lower triangle read), left in the tile-LU form; returns
        (piv, dinv, info) like lu_factor_tiled (bem_chol_factor)."""
        n = A.shape[0]
        assert A.is_cuda and A.shape == (n, n) and A.stride(1) == 1 and A.dtype in (torch.complex128, torch.float64)
        piv = torch.empty(n, dtype=torch.int32, device=A.device)
        info = torch.zeros(1, dtype=torch.int32, device=A.device)
        dinv = torch.empty(int(self.lib.bem_lu_dinv_elems(n)), dtype=torch.complex128, device=A.device)
        method = L.PREC_MIXED if tensor_cores else L.PREC_FP64
        self._check(self.lib.bem_chol_factor(self.ctx, _dtype_code(A), _ptr(A), n, A.stride(0), method, _ptr(piv),
                                             _ptr(dinv), _ptr(info), _stream_ptr()))
        return piv, dinv, info

    def normal_refine(self, A, P, colscale, LU, piv, dinv, g, x, tol=1e-14, maxit=60, restart=30, accept=1e-10):
        """(A^H A + P^H P) x = g (g: n) by the flexible GMRES of lstsq_refine
        (bem_normal_refine); x holds the initial guess.  Returns
        (iterations, relative residual)."""
        n = A.shape[0]
        assert g.numel() == n and g.is_contiguous() and x.is_contiguous() and x.numel() == n
        it = ctypes.c_int(0)
        rr = ctypes.c_double(0.0)
        self._check(self.lib.bem_normal_refine(self.ctx, _dtype_code(A), _ptr(A), _ptr(P), n, A.stride(0),
                                               _ptr(colscale), _dtype_code(LU), _ptr(LU), LU.stride(0), _ptr(piv),
                                               _ptr(dinv), _ptr(g), _ptr(x), float(tol), int(maxit), int(restart),
                                               float(accept), ctypes.byref(it), ctypes.byref(rr), _stream_ptr()))
        return it.value, rr.value

    def gemm(self, A, B, C, alpha=1.0, conj_a=False, conj_b=False, a_lower=False, b_upper=False):
        """C += alpha op(A) op(B) in FP64 on the FP64 tensor cores (bem_gemm);
        op(X) = X^H where conj_x; a_lower / b_upper declare op(A) lower / op(B)
        upper triangular (the other side of the diagonal is not read).  A, B,
        C: complex128 or float64 (all the same), row-major with unit column
        stride."""
        dt = C.dtype
        assert dt in (torch.complex128, torch.float64) and A.dtype == dt and B.dtype == dt
        assert A.is_cuda and B.is_cuda and C.is_cuda and A.stride(1) == 1 and B.stride(1) == 1 and C.stride(1) == 1
        m, n = C.shape
        k = A.shape[0] if conj_a else A.shape[1]
        assert (A.shape[1] if conj_a else A.shape[0]) == m
        assert (B.shape[1] if conj_b else B.shape[0]) == k and (B.shape[0] if conj_b else B.shape[1]) == n
        tri = (1 if a_lower else 0) | (2 if b_upper else 0)
        self._check(self.lib.bem_gemm(self.ctx, _dtype_code(C), int(bool(conj_a)), int(bool(conj_b)), tri, m, n, k,
                                      float(alpha), _ptr(A), A.stride(0), _ptr(B), B.stride(0), _ptr(C), C.stride(0),
                                      _stream_ptr()))
        return C

    def cgs2_append(self, Q: torch.Tensor, j: int, v: torch.Tensor, Rt: torch.Tensor, check: bool = False):
        """Q[:, j] and Rt[j, :j + 1] of one CGS2 step against the first j
        orthonormal columns of Q (bem_cgs2_append); v (a column, any element
        stride) is not modified.  With check the call synchronises and
        reports a device timeout."""
        dt = Q.dtype
        assert dt in (torch.complex128, torch.float64) and v.dtype == dt and Rt.dtype == dt
        assert Q.is_cuda and Q.stride(1) == 1 and Rt.stride(1) == 1 and v.dim() in (1, 2)
        n = Q.shape[0]
        assert v.shape[0] == n and (v.dim() == 1 or v.shape[1] == 1) and 0 <= j < min(Q.shape[1], Rt.shape[0])
        self._check(self.lib.bem_cgs2_append(self.ctx, _dtype_code(Q), _ptr(Q), n, Q.stride(0), int(j), _ptr(v),
                                             v.stride(0), _ptr(Rt), Rt.stride(0), int(bool(check)), _stream_ptr()))

    def chol_inverse(self, A: torch.Tensor, X: torch.Tensor | None = None):
        """L^{-1} for A = L L^H (bem_chol_inverse): A (complex128 or float64,
        lower triangle read) is overwritten by L in its lower triangle.
        Returns (X, info)."""
        n = A.shape[0]
        assert A.is_cuda and A.shape == (n, n) and A.stride(1) == 1 and A.dtype in (torch.complex128, torch.float64)
        if X is None:
            X = torch.empty_like(A)
        assert X.shape == (n, n) and X.stride(1) == 1 and X.dtype == A.dtype
        info = torch.zeros(1, dtype=torch.int32, device=A.device)
        self._check(self.lib.bem_chol_inverse(self.ctx, _dtype_code(A), _ptr(A), n, A.stride(0), _ptr(X), X.stride(0),
                                              _ptr(info), _stream_ptr()))
        return X, info

    def lstsq_refine(self, A, P, colscale, LU, piv, dinv, b, x, tol=1e-14, maxit=60, restart=30, accept=1e-10):
        """Flexible GMRES in FP64 on the scaled normal equations of
        min ||[A; P] x - b|| (bem_lstsq_refine); x holds the initial guess.
        Returns (iterations, relative normal-equation residual)."""
        n = A.shape[0]
        assert b.numel() == 2 * n and b.is_contiguous() and x.is_contiguous() and x.numel() == n
        it = ctypes.c_int(0)
        rr = ctypes.c_double(0.0)
        self._check(self.lib.bem_lstsq_refine(self.ctx, _dtype_code(A), _ptr(A), _ptr(P), n, A.stride(0),
                                              _ptr(colscale), _dtype_code(LU), _ptr(LU), LU.stride(0), _ptr(piv),
                                              _ptr(dinv), _ptr(b), _ptr(x), float(tol), int(maxit), int(restart),
                                              float(accept), ctypes.byref(it), ctypes.byref(rr), _stream_ptr()))
        return it.value, rr.value

    def set_tuning(self, key: int, value: int):
        """A launch-shape choice of this context (bem_ctx_set_tuning)."""
        self._check(self.lib.bem_ctx_set_tuning(self.ctx, int(key), int(value)))

    def adjoint_vertices(self, desc: L.OpDesc, test: DeviceSpace, trial: DeviceSpace, lam: torch.Tensor,
                         u: torch.Tensor, grad: torch.Tensor):
        """grad [nv, 3] += d/dX sum lam[r] A(r, c) u[c] (Laplace V or K, FP64)."""
        assert lam.dtype == torch.float64 and u.dtype == torch.float64 and grad.dtype == torch.float64
        assert lam.is_contiguous() and u.is_contiguous() and grad.is_contiguous() and grad.numel() == 3 * self.nv
        self._check_spaces(test, trial, lam.numel(), u.numel())
        ts, rs = test.c(), trial.c()
        self._check(self.lib.bem_adjoint_vertices(self.ctx, ctypes.byref(desc), ctypes.byref(ts), ctypes.byref(rs),
                                                  _ptr(lam), _ptr(u), _ptr(grad), _stream_ptr()))
        return grad

    def mass(self, test: DeviceSpace, trial: DeviceSpace, out=None, scale=1.0, out_t=None, scale_t=0.0, x=None,
             y=None, conj_x=False):
        ts, rs = test.c(), trial.c()
        if x is not None:
            self._check_spaces(test, trial, y.numel(), x.numel())
            self._check(self.lib.bem_mass(self.ctx, ctypes.byref(ts), ctypes.byref(rs), _dtype_code(y), None, 0,
                                          float(scale), None, 0.0, _ptr(x), _ptr(y), int(bool(conj_x)),
                                          _stream_ptr()))
        else:
            self._check_spaces(test, trial, out.shape[0], out.shape[1])
            if out_t is not None:
                self._check_spaces(trial, test, out_t.shape[0], out_t.shape[1])
            self._check(self.lib.bem_mass(self.ctx, ctypes.byref(ts), ctypes.byref(rs), _dtype_code(out), _ptr(out),
                                          out.stride(0), float(scale), _ptr(out_t), float(scale_t), None, None, 0,
                                          _stream_ptr()))

    # -- post-processing ---------------------------------------------------------------
    def _vertex_buffers(self, *bufs):
        for b in bufs:
            if not (b.is_cuda and b.dtype == torch.float32 and b.is_contiguous() and b.shape == (self.nv, 3)):
                raise ValueError("colour/position buffers must be contiguous float32 [nv, 3] on the device")

    def compute_color(self, solved, exact, vert_types, show, solved_color, exact_color, diff_color):
        """BEMManager.compute_color (BEM_manager.py:527-587): shifts `solved`
        in place and writes the three colour buffers [nv, 3] float32."""
        for t in (solved, exact):
            if not (t.is_cuda and t.is_contiguous() and t.dtype in (torch.float64, torch.complex128)
                    and t.numel() == self.nv):
                raise ValueError("solved/exact must be contiguous float64 or complex128 [nv] on the device")
        if solved.dtype != exact.dtype:
            raise ValueError("solved and exact must have the same dtype")
        if not (vert_types.is_cuda and vert_types.dtype == torch.int32 and vert_types.numel() == self.nv):
            raise ValueError("vert_types must be int32 [nv] on the device")
        self._vertex_buffers(solved_color, exact_color, diff_color)
        n = 2 if solved.is_complex() else 1
        self._check(self.lib.bem_compute_color(self.ctx, n, _ptr(solved), _ptr(exact), _ptr(vert_types), int(show),
                                               _ptr(solved_color), _ptr(exact_color), _ptr(diff_color),
                                               _stream_ptr()))

    def set_mesh_instances(self, solved_vertices, exact_vertices, diff_vertices):
        """BEMManager.set_mesh_instances (BEM_manager.py:589-606)."""
        self._vertex_buffers(solved_vertices, exact_vertices, diff_vertices)
        self._check(self.lib.bem_set_mesh_instances(self.ctx, _ptr(solved_vertices), _ptr(exact_vertices),
                                                    _ptr(diff_vertices), _stream_ptr()))

    # -- dense solve ---------------------------------------------------------------
    def lu_factor(self, A: torch.Tensor):
        """In-place LU with partial pivoting; returns (piv, info) device int32."""
        n = A.shape[0]
        assert A.is_cuda and A.shape[0] == A.shape[1] and A.stride(1) == 1
        piv = torch.empty(n, dtype=torch.int32, device=A.device)
        info = torch.zeros(1, dtype=torch.int32, device=A.device)
        self._check(self.lib.bem_lu_factor(self.ctx, _dtype_code(A), _ptr(A), n, A.stride(0), _ptr(piv), _ptr(info),
                                           _stream_ptr()))
        return piv, info

    def lu_solve(self, LU: torch.Tensor, piv: torch.Tensor, b: torch.Tensor):
        """b (n or n x nrhs, FP64 real/complex) overwritten by the solution."""
        n = LU.shape[0]
        b2 = b.view(n, -1)
        assert b2.is_contiguous()
        self._check(self.lib.bem_lu_solve(self.ctx, _dtype_code(LU), _ptr(LU), n, LU.stride(0), _ptr(piv), _ptr(b2),
                                          b2.shape[1], b2.shape[1], _stream_ptr()))
        return b

    def gemv(self, A, x, y, alpha=1.0, beta=0.0):
        m, n = A.shape
        self._check(self.lib.bem_gemv(self.ctx, _dtype_code(A), _ptr(A), m, n, A.stride(0), _ptr(x), _ptr(y),
                                      float(alpha), float(beta), _stream_ptr()))
        return y

    def lu_factor_tiled(self, A: torch.Tensor):
        """In-place tile-pivoted LU; returns (piv, dinv, info)."""
        n = A.shape[0]
        assert A.is_cuda and A.shape[0] == A.shape[1] and A.stride(1) == 1
        piv = torch.empty(n, dtype=torch.int32, device=A.device)
        info = torch.zeros(1, dtype=torch.int32, device=A.device)
        cdt = A.dtype if A.is_complex() else (torch.complex64 if A.dtype == torch.float32 else torch.complex128)
        dinv = torch.empty(int(self.lib.bem_lu_dinv_elems(n)), dtype=cdt, device=A.device)
        self._check(self.lib.bem_lu_factor_tiled(self.ctx, _dtype_code(A), _ptr(A), n, A.stride(0), _ptr(piv),
                                                 _ptr(dinv), _ptr(info), _stream_ptr()))
        return piv, dinv, info

    def lu_solve_tiled(self, LU, piv, dinv, b):
        n = LU.shape[0]
        assert b.is_contiguous() and b.numel() == n
        self._check(self.lib.bem_lu_solve_tiled(self.ctx, _dtype_code(LU), _ptr(LU), n, LU.stride(0), _ptr(piv),
                                                _ptr(dinv), _ptr(b), _stream_ptr()))
        return b

    def gmres_solve(self, A_hi, LU_lo, piv, b, x, tol=1e-12, maxit=300, restart=60, dinv=None, accept=1e-8):
        """Restarted GMRES in FP64 preconditioned by the low-precision factors
        (bem_gmres_ir); x holds the initial guess.  Returns (iterations,
        relative residual); raises BemError(BEM_ERR_NOCONVERGE) when neither
        tol nor, after stagnation, `accept` is reached."""
        it = ctypes.c_int(0)
        rr = ctypes.c_double(0.0)
        n = A_hi.shape[0]
        assert b.is_contiguous() and x.is_contiguous() and b.dtype == A_hi.dtype == x.dtype
        self._check(self.lib.bem_gmres_ir(self.ctx, _dtype_code(A_hi), _ptr(A_hi), _ptr(LU_lo), _ptr(piv),
                                          _ptr(dinv), n, A_hi.stride(0), _ptr(b), _ptr(x), float(tol), int(maxit),
                                          int(restart), float(accept), ctypes.byref(it), ctypes.byref(rr),
                                          _stream_ptr()))
        return it.value, rr.value

    def refine_solve(self, A_hi, LU_lo, piv, b, x, tol=1e-12, maxit=50, dinv=None, accept=None):
        """FP64 iterative refinement (bem_refine_solve); returns (iterations,
        relative residual).  When the residual stagnates above `tol` -- the
        FP64 residual of an ill-conditioned system cannot fall below about
        eps * cond(A) -- a final residual <= `accept` is returned instead of
        raising BEM_ERR_NOCONVERGE."""
        it = ctypes.c_int(0)
        rr = ctypes.c_double(0.0)
        n = A_hi.shape[0]
        rc = self.lib.bem_refine_solve(self.ctx, _dtype_code(A_hi), _ptr(A_hi), _ptr(LU_lo), _ptr(piv), _ptr(dinv),
                                       n, A_hi.stride(0), _ptr(b), _ptr(x), float(tol), int(maxit), ctypes.byref(it),
                                       ctypes.byref(rr), _stream_ptr())
        if rc == -4 and accept is not None and rr.value <= accept:
            return it.value, rr.value
        self._check(rc)
        return it.value, rr.value


def measure_peaks(engine: Engine):
    """(FP32 TFLOP/s, FP64 TFLOP/s, MUFU Gop/s) measured on this device."""
    out = (ctypes.c_double * 3)()
    engine._check(engine.lib.bem_measure_peaks(engine.ctx, out, _stream_ptr()))
    return float(out[0]), float(out[1]), float(out[2])
