"""Generate golden fixtures by running the reference's own BEM code.

The reference (GeCao/taichi-BEM) is pure Python + Taichi.  Taichi and
pywavefront are not installed here, so ``_taichi_standin.install()`` registers
a sequential FP64 stand-in for the Taichi API subset the reference uses; the
reference's ``src/managers`` and ``src/BEM_functions`` modules are then
imported unmodified from the reference checkout and driven through the same
method sequence as ``BEMManager.run`` (``src/managers/BEM_manager.py:990-1029``),
including the two GUI kernels at its end (``compute_color``, which shifts
``solved``, and ``set_mesh_instances``); ``solved`` is stored both before
(``solved``) and after (``colour_solved``) the shift.

Usage (in a container that has the reference checkout):

    python tests/golden/gen_golden.py --ref <path of the reference checkout> [--only NAME] [--colour-only] [--meshes]

Writes ``tests/golden/<case>.npz``.  Every array needed to re-run a case
(vertices after the reference's own normalisation, panels, BVP maps, Gauss
order, wavenumber) is stored in the fixture, so the tests never read the
reference checkout.
"""
from __future__ import annotations

import argparse
import math
import os
import shutil
import sys
import tempfile
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _taichi_standin  # noqa: E402


# ---------------------------------------------------------------------------
# meshes
# ---------------------------------------------------------------------------
def icosphere(subdiv: int):
    """Unit icosphere: icosahedron, each level splits a triangle in four."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
         (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    v = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
         (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                p = v[a] + v[b]
                v.append(p / np.linalg.norm(p))
                cache[key] = len(v) - 1
            return cache[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    return np.array(v), np.array(f, dtype=np.int64)


def write_obj(path, verts, faces):
    with open(path, "w") as fh:
        for p in verts:
            fh.write("v %.17g %.17g %.17g\n" % tuple(p))
        for a, b, c in faces:
            fh.write("f %d %d %d\n" % (a + 1, b + 1, c + 1))


# ---------------------------------------------------------------------------
# boundary data written as Taichi-style functions on stand-in vectors
# ---------------------------------------------------------------------------
def make_data(kind, k, direction):
    ti = sys.modules["taichi"]
    if kind == "laplace_point":
        x0 = (2.0, 2.0, 2.0)

        def fD(x, sqrt_n=1.0):
            d = [x[0] - x0[0], x[1] - x0[1], x[2] - x0[2]]
            r = math.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2)
            return ti.Vector([1.0 / r])

        def fN(x, n, sqrt_n=1.0):
            d = [x[0] - x0[0], x[1] - x0[1], x[2] - x0[2]]
            r = math.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2)
            return ti.Vector([-(d[0] * n[0] + d[1] * n[1] + d[2] * n[2]) / r ** 3])
        return fD, fN
    if kind == "plane_wave":
        dx = direction
        dim = len(dx)

        def fD(x, sqrt_n=1.0):
            ph = k * sqrt_n * sum(dx[c] * x[c] for c in range(dim))
            return ti.Vector([math.cos(ph), math.sin(ph)])

        def fN(x, n, sqrt_n=1.0):
            kk = k * sqrt_n
            ph = kk * sum(dx[c] * x[c] for c in range(dim))
            dn = sum(dx[c] * n[c] for c in range(dim))
            return ti.Vector([-kk * dn * math.sin(ph), kk * dn * math.cos(ph)])
        return fD, fN
    if kind == "laplace_2d":
        # the 2D data of demo/demo_Laplace.py:65-72: u = (x^2 - y^2) / 2
        def fD(x, sqrt_n=1.0):
            return ti.Vector([0.5 * x[0] * x[0] - 0.5 * x[1] * x[1]])

        def fN(x, n, sqrt_n=1.0):
            return ti.Vector([x[0] * n[0] - x[1] * n[1]])
        return fD, fN
    raise ValueError(kind)


class _Log:
    initialized = True

    def InfoLog(self, s=""):
        pass

    WarnLog = InfoLog
    ErrorLog = InfoLog


class _Core:
    """The attributes of ``CoreManager`` (src/managers/core_manager.py:11-43)
    that MeshManager/BEMManager read, without the GUI and file side effects."""

    def __init__(self, root, params):
        self.root_path = root
        self._simulation_parameters = dict(params)
        if "Helmholtz" not in params["kernel"]:
            self._simulation_parameters["k"] = 0
        self._is_transmission = 1 if ("Full" in params["boundary"] or "Transmission" in params["kernel"]) else 0
        self._np_dtype = np.float64
        self._ti_dtype = "f64"
        self._log_manager = _Log()


CASES = {
    # name: (mesh, params overrides, data kind)
    "cube_lap_dir_q5": ("cube", dict(kernel="Laplace", boundary="Dirichlet", scope="Interior", GaussQR=5), "laplace_point"),
    "cube_lap_neu_q5": ("cube", dict(kernel="Laplace", boundary="Neumann", scope="Interior", GaussQR=5), "laplace_point"),
    "cube_helm_mix_ext_q4": ("cube", dict(kernel="Helmholtz", boundary="Mix", scope="Exterior", GaussQR=4, k=1.5), "plane_wave"),
    "cube_trans_q3": ("cube", dict(kernel="Helmholtz_Transmission", boundary="Full", scope="Interior", GaussQR=3, k=2.0,
                                   n_i=2.25, n_o=1.0), "plane_wave"),
    "ico1_lap_full_q3": ("ico1", dict(kernel="Laplace", boundary="Full", scope="Interior", GaussQR=3), "laplace_point"),
    "ico1_helm_dir_p1_q3": ("ico1", dict(kernel="Helmholtz", boundary="Dirichlet", scope="Interior", GaussQR=3, k=3.0,
                                         Q_Neumann=1), "plane_wave"),
    # 2D: MeshManager.load_analytical_disk (mesh_manager.py:520-536) with N segments
    "disk32_lap_dir_q4": ("disk32", dict(dim=2, kernel="Laplace", boundary="Dirichlet", scope="Interior", GaussQR=4),
                          "laplace_2d"),
    "disk32_lap_neu_q4": ("disk32", dict(dim=2, kernel="Laplace", boundary="Neumann", scope="Interior", GaussQR=4),
                          "laplace_2d"),
    "disk24_helm_mix_ext_q3": ("disk24", dict(dim=2, kernel="Helmholtz", boundary="Mix", scope="Exterior", GaussQR=3,
                                              k=2.0), "plane_wave"),
    "disk24_helm_dir_p1_q3": ("disk24", dict(dim=2, kernel="Helmholtz", boundary="Dirichlet", scope="Interior",
                                             GaussQR=3, k=3.0, Q_Neumann=1), "plane_wave"),
    "disk256_lap_dir_q3": ("disk256", dict(dim=2, kernel="Laplace", boundary="Dirichlet", scope="Interior",
                                           GaussQR=3), "laplace_2d"),
    # the colouring's show = "Dirichlet" branch (every vertex shifted)
    "disk32_lap_mix_showD_q3": ("disk32", dict(dim=2, kernel="Laplace", boundary="Mix", scope="Interior",
                                               GaussQR=3, show="Dirichlet"), "laplace_2d"),
}


def _setup(ref, name, tmp, patched):
    """The reference's MeshManager and BEMManager for one case, initialised
    (mesh loaded, fields allocated, boundary callbacks set) but not run."""
    mesh, over, data_kind = CASES[name]
    os.makedirs(os.path.join(tmp, "assets"))
    if mesh == "cube":
        shutil.copy(os.path.join(ref, "assets", "cube.obj"), os.path.join(tmp, "assets", "cube.obj"))
    elif mesh.startswith("disk"):
        pass
    else:
        v, f = icosphere(int(mesh[3:]))
        write_obj(os.path.join(tmp, "assets", mesh + ".obj"), v, f)
    params = dict(dim=3, object=mesh, GaussQR=5, n_i=1, n_o=1, k=0.0, kernel="Laplace", boundary="Dirichlet",
                  scope="Interior", show="Default", Q_Neumann=0, Q_Dirichlet=1, log_to_disk=False,
                  make_video=False, show_wireframe=False, vis=False)
    params.update(over)
    from src.managers.mesh_manager import MeshManager
    from src.managers.BEM_manager import BEMManager

    dim = int(params["dim"])
    if mesh.startswith("disk"):
        # the reference's own disk generator with N segments instead of its default 256
        n_seg = int(mesh[4:])
        disk = MeshManager.load_analytical_disk
        patched.append((MeshManager, "load_analytical_disk", disk))
        MeshManager.load_analytical_disk = lambda self, r=1.0, N=n_seg: disk(self, r, N)
    core = _Core(tmp, params)
    core._mesh_manager = MeshManager(core)
    core._BEM_manager = BEMManager(core)
    core._mesh_manager.initialization()
    rng = np.random.default_rng(0)
    d = rng.standard_normal(dim)
    d = d / np.linalg.norm(d)
    fD, fN = make_data(data_kind, float(params.get("k", 0.0)), d)
    bem = core._BEM_manager
    bem.initialization(fD, fN)
    return bem, core._mesh_manager, params, d, data_kind


def _colour(bem, out):
    """The GUI preparation that ends BEMManager.run (BEM_manager.py:1028-1029):
    compute_color shifts ``solved`` and fills the colour fields,
    set_mesh_instances fills the three position fields."""
    bem.compute_color()
    bem.set_mesh_instances()
    out["colour_solved"] = bem.solved.to_numpy()
    for key in ("solved_vert_color", "analytical_vert_color", "diff_vert_color", "solved_vertices",
                "analytical_vertices", "diff_vertices"):
        out[key] = getattr(bem, key).to_numpy()


def colour_case(ref, name):
    """Adds the colouring outputs to an existing fixture: the case's managers
    are set up again, ``solved`` / ``analytical_solved`` are loaded from the
    fixture, and the reference's two GUI kernels are run on them."""
    path = os.path.join(HERE, name + ".npz")
    out = dict(np.load(path))
    tmp = tempfile.mkdtemp(prefix="bemgold_")
    patched = []
    try:
        bem, mm, params, d, data_kind = _setup(ref, name, tmp, patched)
        bem.solved.from_numpy(out["solved"])
        bem.analytical_solved.from_numpy(out["analytical_solved"])
        _colour(bem, out)
        np.savez_compressed(path, **out)
        print(f"{name}: colouring added", flush=True)
    finally:
        for owner, attr, val in patched:
            setattr(owner, attr, val)
        shutil.rmtree(tmp, ignore_errors=True)


def run_case(ref, name):
    tmp = tempfile.mkdtemp(prefix="bemgold_")
    patched = []
    try:
        from src.BEM_functions.utils import AssembleType, ScopeType

        bem, mm, params, d, data_kind = _setup(ref, name, tmp, patched)
        dim = int(params["dim"])

        out = {}
        snaps = []
        orig_forward = bem.matrix_layer_forward

        def forward(k, sqrt_n=1.0, scope_type=0):
            orig_forward(k=k, sqrt_n=sqrt_n, scope_type=scope_type)
            snap = {}
            if bem.N_Neumann > 0:
                snap["V"] = bem.single_layer._Vmat.to_numpy()
            if bem.N_Neumann > 0 and bem.M_Dirichlet > 0:
                snap["K"] = bem.double_layer._Kmat.to_numpy()
            if bem.M_Dirichlet > 0:
                snap["W"] = bem.hypersingular_layer._Wmat.to_numpy()
            snaps.append((int(scope_type), float(sqrt_n), snap))
        bem.matrix_layer_forward = forward

        t0 = time.time()
        # Same sequence as BEMManager.run (src/managers/BEM_manager.py:990-1029).
        bem._mat_A.fill(0)
        if bem._is_transmission > 0:
            bem.matrix_layer_forward(k=bem._k, sqrt_n=bem._sqrt_no, scope_type=int(ScopeType.EXTERIOR))
            bem.assemble_matA(assemble_type=int(AssembleType.ADD_P_MINUS), multiplier=1.0)
            bem.rhs_constructor.set_boundaries(scope_type=int(ScopeType.INTERIOR), sqrt_ni=bem._sqrt_ni, sqrt_no=bem._sqrt_no)
            bem.assemble_rhs()
            bem.matrix_layer_forward(k=bem._k, sqrt_n=bem._sqrt_ni, scope_type=int(ScopeType.INTERIOR))
            bem.assemble_matA(assemble_type=int(AssembleType.ADD_P_PLUS), multiplier=1.0)
        else:
            bem.matrix_layer_forward(k=bem._k, scope_type=bem._scope_type)
            bem.assemble_matA(assemble_type=int(AssembleType.ADD_M), multiplier=-1.0)
            bem.rhs_constructor.set_boundaries(scope_type=bem._scope_type, sqrt_ni=bem._sqrt_ni, sqrt_no=bem._sqrt_no)
            bem.rhs_layer_forward(k=bem._k, scope_type=bem._scope_type)
            bem.assemble_rhs()
        out["A"] = bem._mat_A.to_numpy()
        out["rhs"] = bem.rhs.to_numpy()
        out["rhs_vec"] = bem.rhs_constructor._rhs_vec.to_numpy()
        out["f_boundary"] = bem.rhs_constructor._f_boundary.to_numpy()
        out["Dirichlet_boundary"] = bem.rhs_constructor._Dirichlet_boundary.to_numpy()
        out["Neumann_boundary"] = bem.rhs_constructor._Neumann_boundary.to_numpy()
        try:
            bem.solve()
            out["raw_solved"] = bem.raw_solved.to_numpy()
        except Exception as exc:  # the reference's own solve failed (e.g. singular A)
            out["solve_error"] = np.array(repr(exc))
        bem.compute_analytical_raw_solved()
        out["raw_analytical_solved"] = bem.raw_analytical_solved.to_numpy()
        bem.splat_u_from_raw_solved_to_vertices()
        out["solved"] = bem.solved.to_numpy()
        out["analytical_solved"] = bem.analytical_solved.to_numpy()
        _colour(bem, out)
        elapsed = time.time() - t0

        for idx, (scope, sqrt_n, snap) in enumerate(snaps):
            for key, val in snap.items():
                out[f"{key}_{idx}"] = val
            out[f"scope_{idx}"] = np.int64(scope)
            out[f"sqrt_n_{idx}"] = np.float64(sqrt_n)
        out["n_forward"] = np.int64(len(snaps))

        out["vertices"] = mm.vertices.to_numpy()
        out["panels"] = np.array(mm.panels.to_numpy(), dtype=np.int64).reshape(-1, dim)
        out["panel_types"] = np.array(mm.panel_types.to_numpy(), dtype=np.int64)
        out["vertice_types"] = np.array(mm.vertice_types.to_numpy(), dtype=np.int64)
        out["panel_areas"] = mm.panel_areas.to_numpy()
        out["panel_normals"] = mm.panel_normals.to_numpy()
        out["vert_areas"] = mm.vert_areas.to_numpy()
        out["vert_normals"] = mm.vert_normals.to_numpy()
        out["N_Neumann"] = np.int64(bem.N_Neumann)
        out["M_Dirichlet"] = np.int64(bem.M_Dirichlet)
        out["GaussQR"] = np.int64(params["GaussQR"])
        out["k"] = np.float64(bem._k)
        out["sqrt_ni"] = np.float64(bem._sqrt_ni)
        out["sqrt_no"] = np.float64(bem._sqrt_no)
        out["direction"] = d
        out["params"] = np.array(repr(params))
        out["data_kind"] = np.array(data_kind)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(f"{name}: done in {elapsed:.1f}s", flush=True)
    finally:
        for owner, attr, val in patched:
            setattr(owner, attr, val)
        shutil.rmtree(tmp, ignore_errors=True)


def mesh_fixture(ref):
    """The reference's own analytic mesh generators
    (MeshManager.load_analytical_sphere / load_analytical_disk,
    src/managers/mesh_manager.py:496-536), called on an object that carries
    only the dtype they read, into tests/golden/meshes_analytical.npz."""
    from src.managers.mesh_manager import MeshManager

    holder = types.SimpleNamespace(_np_dtype=np.float64)
    out = {}
    for tag, kw in (("sphere_default", {}), ("sphere_r07_5x6", dict(r=0.7, rows=5, cols=6))):
        v, f = MeshManager.load_analytical_sphere(holder, **kw)
        out[f"{tag}_vertices"], out[f"{tag}_panels"] = v, f
    for tag, kw in (("disk_default", {}), ("disk_r05_37", dict(r=0.5, N=37))):
        v, f = MeshManager.load_analytical_disk(holder, **kw)
        out[f"{tag}_vertices"], out[f"{tag}_panels"] = v, f
    np.savez_compressed(os.path.join(HERE, "meshes_analytical.npz"), **out)
    print("meshes_analytical: done", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="path of the reference checkout (its src/ is imported)")
    ap.add_argument("--only", default=None)
    ap.add_argument("--meshes", action="store_true",
                    help="only write the analytic-mesh fixture from the reference's generators")
    ap.add_argument("--colour-only", action="store_true",
                    help="add the GUI colouring outputs to the existing fixtures without re-running the cases")
    args = ap.parse_args()
    _taichi_standin.install()
    sys.path.insert(0, args.ref)
    if args.meshes:
        mesh_fixture(args.ref)
        return
    names = [args.only] if args.only else list(CASES)
    for name in names:
        if args.colour_only:
            colour_case(args.ref, name)
        else:
            run_case(args.ref, name)


if __name__ == "__main__":
    main()
