"""ctypes binding of libbem_b200.so (declarations in include/bem_b200.h).

The library is built in-tree by ``taichi-bem_b200/Makefile`` (or
``bem_b200.build.build()``).  There is no fallback: if the shared library is
missing or CUDA is unavailable, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbem_b200.so")

BEM_OK = 0
ERRORS = {
    -1: "BEM_ERR_INVALID",
    -2: "BEM_ERR_CUDA",
    -3: "BEM_ERR_NOMESH",
    -4: "BEM_ERR_NOCONVERGE",
    -5: "BEM_ERR_SINGULAR",
    -6: "BEM_ERR_TIMEOUT",
    -7: "BEM_ERR_MESH",
}

OP_V, OP_K, OP_KP, OP_W = 0, 1, 2, 3
KERNEL_LAPLACE, KERNEL_HELMHOLTZ = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
F64, C128, F32, C64 = 0, 1, 2, 3

# Every symbol include/bem_b200.h declares (checked by tests/test_abi.py).
EXPORTS = [
    "bem_ctx_create", "bem_ctx_destroy", "bem_last_error", "bem_launch_count", "bem_mesh_set",
    "bem_near_pair_count", "bem_mesh_geometry", "bem_assemble", "bem_apply", "bem_mass", "bem_lu_factor",
    "bem_lu_solve", "bem_gemv", "bem_refine_solve", "bem_measure_peaks", "bem_lu_dinv_elems",
    "bem_lu_factor_tiled", "bem_lu_solve_tiled", "bem_assemble_dirichlet", "bem_lu_solve_tiled_static",
    "bem_adjoint_vertices", "bem_mesh_set_2d", "bem_gmres_ir", "bem_compute_color", "bem_set_mesh_instances",
    "bem_lu_factor_status", "bem_binary_version", "bem_ctx_set_tuning", "bem_assemble_calderon", "bem_gram",
    "bem_lstsq_refine", "bem_chol_factor", "bem_gemm", "bem_chol_inverse", "bem_normal_refine", "bem_near_pair_list",
    "bem_assemble_batch", "bem_cgs2_append",
]
STATIC_SOLVE_MAX_N = 32768  # BEM_STATIC_SOLVE_MAX_N
TUNE_CALDERON_GROUP = 0  # BEM_TUNE_CALDERON_GROUP
TUNE_GRAM_KSEG = 1  # BEM_TUNE_GRAM_KSEG
TUNE_CHOL_NB = 2  # BEM_TUNE_CHOL_NB
TUNE_GRAM_BAND = 3  # BEM_TUNE_GRAM_BAND
TUNE_KBATCH_GROUP = 4  # BEM_TUNE_KBATCH_GROUP
TUNE_GRAM_PAIR = 5  # BEM_TUNE_GRAM_PAIR
TUNE_LU_UPDATE = 6  # BEM_TUNE_LU_UPDATE
MAX_KBATCH = 64  # BEM_MAX_KBATCH


class BemError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class OpDesc(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int), ("kernel", ctypes.c_int), ("k", ctypes.c_double), ("k2", ctypes.c_double),
                ("quirk", ctypes.c_int), ("precision", ctypes.c_int), ("deriv_k", ctypes.c_int)]


class Space(ctypes.Structure):
    _fields_ = [("n_panels", ctypes.c_int), ("panels", ctypes.c_void_p), ("nb", ctypes.c_int),
                ("dof", ctypes.c_void_p)]


_lib = None


def load():
    """Load and type the shared library (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libbem_b200.so is not built ({LIB_PATH}); run `make -C taichi-bem_b200`")
    L = ctypes.CDLL(LIB_PATH)
    vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
    L.bem_ctx_create.argtypes = [ctypes.POINTER(vp)]
    L.bem_ctx_destroy.argtypes = [vp]
    L.bem_last_error.argtypes = [vp]
    L.bem_last_error.restype = ctypes.c_char_p
    L.bem_launch_count.argtypes = [vp]
    L.bem_launch_count.restype = i64
    L.bem_mesh_set.argtypes = [vp, vp, vp, i32, i32, i32]
    L.bem_mesh_set_2d.argtypes = [vp, vp, vp, i32, i32, i32]
    L.bem_near_pair_count.argtypes = [vp]
    L.bem_near_pair_count.restype = i64
    L.bem_mesh_geometry.argtypes = [vp, vp, vp, vp]
    L.bem_assemble.argtypes = [vp, ctypes.POINTER(OpDesc), ctypes.POINTER(Space), ctypes.POINTER(Space), i32, vp,
                               i64, dbl, vp, dbl, vp]
    L.bem_apply.argtypes = [vp, ctypes.POINTER(OpDesc), ctypes.POINTER(Space), ctypes.POINTER(Space), i32, vp, vp,
                            dbl, i32, vp]
    L.bem_mass.argtypes = [vp, ctypes.POINTER(Space), ctypes.POINTER(Space), i32, vp, i64, dbl, vp, dbl, vp, vp,
                           i32, vp]
    L.bem_lu_factor.argtypes = [vp, i32, vp, i64, i64, vp, vp, vp]
    L.bem_lu_solve.argtypes = [vp, i32, vp, i64, i64, vp, vp, i64, i64, vp]
    L.bem_gemv.argtypes = [vp, i32, vp, i64, i64, i64, vp, vp, dbl, dbl, vp]
    L.bem_refine_solve.argtypes = [vp, i32, vp, vp, vp, vp, i64, i64, vp, vp, dbl, i32,
                                   ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), vp]
    L.bem_gmres_ir.argtypes = [vp, i32, vp, vp, vp, vp, i64, i64, vp, vp, dbl, i32, i32, dbl,
                               ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), vp]
    L.bem_assemble_dirichlet.argtypes = [vp, ctypes.POINTER(OpDesc), ctypes.POINTER(Space), ctypes.POINTER(Space),
                                         vp, i64, dbl, ctypes.POINTER(Space), ctypes.POINTER(Space), vp, vp, dbl,
                                         i32, vp]
    L.bem_lu_solve_tiled_static.argtypes = [i32, vp, i64, i64, vp, vp, vp, vp]
    L.bem_lu_dinv_elems.argtypes = [i64]
    L.bem_lu_dinv_elems.restype = i64
    L.bem_lu_factor_tiled.argtypes = [vp, i32, vp, i64, i64, vp, vp, vp, vp]
    L.bem_lu_solve_tiled.argtypes = [vp, i32, vp, i64, i64, vp, vp, vp, vp]
    L.bem_lu_factor_status.argtypes = [vp, vp]
    L.bem_binary_version.argtypes = [ctypes.POINTER(ctypes.c_int)]
    L.bem_ctx_set_tuning.argtypes = [vp, i32, i32]
    L.bem_chol_factor.argtypes = [vp, i32, vp, i64, i64, i32, vp, vp, vp, vp]
    L.bem_near_pair_list.argtypes = [vp, vp]
    L.bem_gemm.argtypes = [vp, i32, i32, i32, i32, i64, i64, i64, dbl, vp, i64, vp, i64, vp, i64, vp]
    L.bem_chol_inverse.argtypes = [vp, i32, vp, i64, i64, vp, i64, vp, vp]
    L.bem_gram.argtypes = [vp, i32, vp, vp, i64, i64, vp, i32, i32, vp, i64, vp]
    L.bem_lstsq_refine.argtypes = [vp, i32, vp, vp, i64, i64, vp, i32, vp, i64, vp, vp, vp, vp, dbl, i32, i32, dbl,
                                   ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), vp]
    L.bem_normal_refine.argtypes = list(L.bem_lstsq_refine.argtypes)
    L.bem_assemble_calderon.argtypes = [vp, ctypes.POINTER(OpDesc), i32, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_double), ctypes.POINTER(Space), ctypes.POINTER(Space),
                                        ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_double), i64, vp]
    pd, pp = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_void_p)
    L.bem_assemble_batch.argtypes = [vp, ctypes.POINTER(OpDesc), ctypes.POINTER(Space), ctypes.POINTER(Space), i32,
                                     pd, pd, pp, i64, pd, pp, pd, vp]
    L.bem_cgs2_append.argtypes = [vp, i32, vp, i64, i64, i32, vp, i64, vp, i64, i32, vp]
    L.bem_measure_peaks.argtypes = [vp, ctypes.POINTER(ctypes.c_double), vp]
    L.bem_compute_color.argtypes = [vp, i32, vp, vp, vp, i32, vp, vp, vp, vp]
    L.bem_set_mesh_instances.argtypes = [vp, vp, vp, vp, vp]
    L.bem_adjoint_vertices.argtypes = [vp, ctypes.POINTER(OpDesc), ctypes.POINTER(Space), ctypes.POINTER(Space), vp,
                                       vp, vp, vp]
    for name in EXPORTS:
        if name not in ("bem_last_error", "bem_launch_count", "bem_near_pair_count", "bem_lu_dinv_elems"):
            getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L
