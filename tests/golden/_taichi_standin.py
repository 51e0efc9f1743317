"""Minimal sequential stand-in for the subset of the Taichi API that the
reference BEM code (GeCao/taichi-BEM, ``src/``) uses on its 3D path.

Taichi is not installable in this container, so ``gen_golden.py`` registers
this module as ``taichi`` (and a tiny OBJ reader as ``pywavefront``) before
importing the reference's own ``src.managers`` / ``src.BEM_functions``
modules.  The reference kernels then run *as written*, line for line, as plain
Python: ``@ti.kernel`` and ``@ti.func`` are identity decorators, loops run
sequentially (Taichi's parallel ``+=`` on fields is an atomic add, so the
sequential sum differs only in floating-point summation order), and every
value is a Python float (FP64).  The resulting matrices are the reference's
algorithm evaluated in FP64, which is what the FP64 oracle and the FP64 GPU
path must reproduce.

This is test infrastructure for generating golden fixtures only; nothing in
the product imports it.
"""
from __future__ import annotations

import ast
import inspect
import math
import sys
import textwrap
import types

import numpy as np

# ----------------------------------------------------------------------------
# dtypes / decorators
# ----------------------------------------------------------------------------
f32 = "f32"
f64 = "f64"
i32 = "i32"


def data_oriented(cls):
    return cls


def kernel(fn):
    """Identity, except for kernels that reduce into a kernel-scope local with
    ``ti.atomic_max(local, value)``: Taichi updates that local in place, which a
    Python call cannot do, so those statements are rewritten as
    ``local = max(local, value)`` (the sequential form of the same reduction)."""
    try:
        src = textwrap.dedent(inspect.getsource(fn))
    except (OSError, TypeError):
        return fn
    if "atomic_max" not in src:
        return fn
    tree = ast.parse(src)
    fdef = tree.body[0]
    fdef.decorator_list = []

    class _Rewrite(ast.NodeTransformer):
        def visit_Expr(self, node):
            c = node.value
            if (isinstance(c, ast.Call) and isinstance(c.func, ast.Attribute) and c.func.attr == "atomic_max"
                    and isinstance(c.args[0], ast.Name)):
                name = c.args[0].id
                new = ast.Assign(targets=[ast.Name(name, ast.Store())],
                                 value=ast.Call(ast.Name("max", ast.Load()), [ast.Name(name, ast.Load()), c.args[1]], []))
                return ast.copy_location(new, node)
            return node

    tree = ast.fix_missing_locations(_Rewrite().visit(tree))
    ast.increment_lineno(tree, fn.__code__.co_firstlineno - 1)
    ns = {}
    exec(compile(tree, inspect.getsourcefile(fn), "exec"), fn.__globals__, ns)
    return ns[fdef.name]


def func(fn):
    return fn


def static(x, *args):
    return x


def static_assert(cond, msg=None):
    assert cond, msg


def init(*args, **kwargs):
    return None


def atomic_max(a, b):  # on a local, rewritten by ``kernel``; on anything else, the new maximum
    return max(a, b)


def abs(x):  # noqa: A001 - mirrors ti.abs
    return x.__abs__()


# ----------------------------------------------------------------------------
# small vectors / matrices
# ----------------------------------------------------------------------------
_NAMES = {"x": 0, "y": 1, "z": 2, "w": 3}


class Vector:
    """Fixed-size value vector with Taichi's element-wise arithmetic."""

    __slots__ = ("v",)

    def __init__(self, data, dt=None):
        object.__setattr__(self, "v", [float(a) if dt != i32 else int(a) for a in data]
                           if not isinstance(data, Vector) else list(data.v))

    # -- element access -----------------------------------------------------
    def __getattr__(self, name):
        if name in _NAMES:
            return self.v[_NAMES[name]]
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in _NAMES:
            self.v[_NAMES[name]] = value
        else:
            object.__setattr__(self, name, value)

    def __getitem__(self, i):
        return self.v[i]

    def __setitem__(self, i, value):
        self.v[i] = value

    def __len__(self):
        return len(self.v)

    def __iter__(self):
        return iter(self.v)

    # -- arithmetic -----------------------------------------------------------
    def _binop(self, other, op):
        if isinstance(other, Vector):
            return Vector([op(a, b) for a, b in zip(self.v, other.v)])
        return Vector([op(a, other) for a in self.v])

    def __add__(self, o):
        return self._binop(o, lambda a, b: a + b)

    def __radd__(self, o):
        return self._binop(o, lambda a, b: b + a)

    def __sub__(self, o):
        return self._binop(o, lambda a, b: a - b)

    def __rsub__(self, o):
        return self._binop(o, lambda a, b: b - a)

    def __mul__(self, o):
        return self._binop(o, lambda a, b: a * b)

    def __rmul__(self, o):
        return self._binop(o, lambda a, b: b * a)

    def __truediv__(self, o):
        return self._binop(o, lambda a, b: a / b)

    def __neg__(self):
        return Vector([-a for a in self.v])

    def __abs__(self):
        return Vector([a if a >= 0 else -a for a in self.v])

    def dot(self, o):
        return sum(a * b for a, b in zip(self.v, o.v))

    def norm(self):
        return math.sqrt(sum(a * a for a in self.v))

    def normalized(self):
        n = self.norm()
        return Vector([a / n for a in self.v])

    def __repr__(self):
        return f"Vector({self.v})"

    @staticmethod
    def field(n, dtype=None, shape=()):
        return Field(shape, n=n)

    # Taichi allows ti.Vector.norm(v) / ti.Vector.normalized(v) as functions
    # (the instance methods above serve both forms).


class Matrix:
    __slots__ = ("m",)

    def __init__(self, rows):
        self.m = [list(map(float, r)) for r in rows]

    def __matmul__(self, vec):
        return Vector([sum(a * b for a, b in zip(row, vec.v)) for row in self.m])

    @staticmethod
    def field(n, m, dtype=None, shape=()):
        return Field(shape, n=n, m=m)


class _Types:
    @staticmethod
    def vector(n, dtype):
        return ("vector", n, dtype)

    @staticmethod
    def matrix(n, m, dtype):
        return ("matrix", n, m, dtype)


types_ = _Types()


# ----------------------------------------------------------------------------
# fields
# ----------------------------------------------------------------------------
class Field:
    """Dense field of scalars, Vectors (n) or Matrices (n x m)."""

    def __init__(self, shape, n=None, m=None, dtype=None):
        if isinstance(shape, int):
            shape = (shape,)
        self.shape = tuple(shape)
        self.n = n
        self.m = m
        self.dtype = dtype
        size = int(np.prod(self.shape)) if len(self.shape) else 1
        self._data = [self._zero() for _ in range(size)]

    def _zero(self):
        if self.n is None:
            return 0 if self.dtype == i32 else 0.0
        if self.m is None:
            return Vector([0.0] * self.n)
        return Matrix([[0.0] * self.m for _ in range(self.n)])

    def _flat(self, idx):
        if not isinstance(idx, tuple):
            idx = (idx,)
        if len(self.shape) == 0:
            return 0
        f = 0
        for d, i in zip(self.shape, idx):
            i = int(i)
            if i < 0 or i >= d:
                raise IndexError(f"field index {idx} out of range for shape {self.shape}")
            f = f * d + i
        return f

    def __getitem__(self, idx):
        # The reference reads index -1 of a boundary field for skipped
        # (MIX_NONRESOLVED) panels and never uses the value; Taichi does not
        # bounds-check there, so an out-of-range read yields a zero here.
        try:
            return self._data[self._flat(idx)]
        except IndexError:
            return self._zero()

    def __setitem__(self, idx, value):
        if self.n is not None and self.m is None:
            value = Vector(value)
        self._data[self._flat(idx)] = value

    def __iter__(self):
        if len(self.shape) == 1:
            return iter(range(self.shape[0]))
        return iter(np.ndindex(*self.shape))

    def fill(self, value):
        for i in range(len(self._data)):
            if self.n is None:
                self._data[i] = value if isinstance(value, int) and self.dtype == i32 else float(value)
            elif self.m is None:
                self._data[i] = Vector([float(value)] * self.n)
            else:
                self._data[i] = Matrix([[float(value)] * self.m for _ in range(self.n)])

    def from_numpy(self, arr):
        arr = np.asarray(arr)
        flat = arr.reshape((-1,) + arr.shape[len(self.shape):]) if len(self.shape) else arr.reshape((1,) + arr.shape)
        for i in range(len(self._data)):
            if self.n is None:
                v = flat[i].item()
                self._data[i] = int(v) if arr.dtype.kind in "iu" else float(v)
            elif self.m is None:
                self._data[i] = Vector(flat[i].tolist())
            else:
                self._data[i] = Matrix(flat[i].tolist())

    def to_numpy(self):
        if self.n is None:
            return np.array(self._data, dtype=np.float64).reshape(self.shape)
        if self.m is None:
            return np.array([d.v for d in self._data], dtype=np.float64).reshape(self.shape + (self.n,))
        return np.array([d.m for d in self._data], dtype=np.float64).reshape(self.shape + (self.n, self.m))

    def to_torch(self, device=None):
        import torch
        return torch.from_numpy(self.to_numpy())

    def from_torch(self, t):
        self.from_numpy(t.detach().cpu().numpy())


def field(dtype=None, shape=()):
    return Field(shape, dtype=dtype)


# ----------------------------------------------------------------------------
# ti.math
# ----------------------------------------------------------------------------
def _cmul(a, b):
    return Vector([a[0] * b[0] - a[1] * b[1], a[0] * b[1] + a[1] * b[0]])


def _cconj(a):
    return Vector([a[0], -a[1]])


def _cexp(a):
    e = math.exp(a[0])
    return Vector([e * math.cos(a[1]), e * math.sin(a[1])])


def _cross(a, b):
    return Vector([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])


def _dot(a, b):
    return a.dot(b)


math_ = types.SimpleNamespace(
    pi=math.pi,
    log=math.log,
    exp=math.exp,
    sqrt=math.sqrt,
    cos=math.cos,
    sin=math.sin,
    cmul=_cmul,
    cconj=_cconj,
    cexp=_cexp,
    cross=_cross,
    dot=_dot,
    _complex=types.SimpleNamespace(cmul=_cmul),
)


def install():
    """Register this module as ``taichi`` and a tiny OBJ reader as ``pywavefront``."""
    mod = sys.modules[__name__]
    ti = types.ModuleType("taichi")
    for name in ("f32", "f64", "i32", "data_oriented", "kernel", "func", "static", "static_assert",
                 "init", "atomic_max", "abs", "Vector", "Matrix", "field"):
        setattr(ti, name, getattr(mod, name))
    ti.types = types_
    ti.math = math_
    ti.ui = types.SimpleNamespace()
    ti.tools = types.SimpleNamespace(VideoManager=lambda *a, **k: None)
    ti.gpu = "gpu"
    ti.cpu = "cpu"
    sys.modules["taichi"] = ti

    pw = types.ModuleType("pywavefront")

    class _Mesh:
        def __init__(self, faces):
            self.faces = faces

    class Wavefront:
        """Reads ``v`` and ``f`` records; polygons are fan-triangulated."""

        def __init__(self, path, collect_faces=True, **kwargs):
            self.vertices = []
            faces = []
            with open(path) as fh:
                for line in fh:
                    parts = line.split()
                    if not parts:
                        continue
                    if parts[0] == "v":
                        self.vertices.append(tuple(float(p) for p in parts[1:4]))
                    elif parts[0] == "f":
                        idx = [int(p.split("/")[0]) - 1 for p in parts[1:]]
                        for t in range(1, len(idx) - 1):
                            faces.append([idx[0], idx[t], idx[t + 1]])
            self.meshes = {None: _Mesh(faces)}

    pw.Wavefront = Wavefront
    sys.modules["pywavefront"] = pw
    return ti
