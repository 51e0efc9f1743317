"""Pin the CPU oracle to the reference: every golden fixture was produced by
running the reference's own kernels (tests/golden/gen_golden.py)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests._util import FIXTURES, data_callbacks, load_fixture, rel_err, to_complex

TOL = 1e-12  # FP64 restatement vs the reference's algorithm in FP64


def _problem(d, quirk=True):
    params = eval(str(d["params"]))
    fD, fN = data_callbacks(str(d["data_kind"]), float(params.get("k", 0.0)), d["direction"])
    return O.Problem(d["vertices"], d["panels"], params, fD, fN, quirk=quirk)


def test_gauss_tables_match_legendre():
    for n in list(range(1, 9)) + [12]:
        p, w = O.gauss(n)
        x, wl = np.polynomial.legendre.leggauss(n)
        assert np.allclose(p, (x + 1) / 2, atol=1e-15, rtol=0)
        assert np.allclose(w, wl / 2, atol=1e-15, rtol=0)


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_reference(name):
    d = load_fixture(name)
    P = _problem(d)
    assert (P.mesh.panel_types == d["panel_types"]).all()
    assert (P.mesh.vert_types == d["vertice_types"]).all()
    assert P.mesh.N_N == int(d["N_Neumann"]) and P.mesh.M_D == int(d["M_Dirichlet"])
    assert np.allclose(P.mesh.panel_areas, d["panel_areas"], rtol=1e-14)
    assert np.allclose(P.mesh.panel_normals, d["panel_normals"], atol=1e-14)
    r = P.run()
    nf = int(d["n_forward"])
    for i in range(nf):
        lay = r["layers"] if "layers" in r else (r["layers_o"] if i == 0 else r["layers_i"])
        for key in ("V", "K", "W"):
            if f"{key}_{i}" in d:
                assert rel_err(lay[key], to_complex(d[f"{key}_{i}"])) < TOL, (key, i)
    assert rel_err(r["A"], to_complex(d["A"])) < TOL
    assert rel_err(r["rhs"], to_complex(d["rhs"])) < TOL
    if "solve_error" in d:
        assert r["raw_solved"] is None or np.linalg.cond(r["A"]) > 1e12
    elif np.linalg.cond(r["A"]) < 1e8:
        assert rel_err(r["raw_solved"], to_complex(d["raw_solved"])) < 1e-10


def test_relation_rule_cube():
    d = load_fixture("cube_lap_dir_q5")
    tris = d["panels"]
    for i in range(len(tris)):
        for j in range(len(tris)):
            shared = len(set(tris[i]) & set(tris[j]))
            want = 1 if i == j else {0: 0, 1: 2, 2: 3, 3: 3}[shared]
            assert O.relation(tris, i, j) == want


# cases used only here: the colouring with show = "Dirichlet"
POST_ONLY = ["disk32_lap_mix_showD_q3"]


@pytest.mark.parametrize("name", FIXTURES + POST_ONLY)
def test_post_oracle_matches_reference(name):
    """oracle/post.py against the reference's compute_color and
    set_mesh_instances run on the fixture's own per-vertex traces.  The
    reference stores the `show` parameter in `show` but reads `_show`, which
    stays -1 except for transmission (BEM_manager.py:28,43-53)."""
    from oracle import post as OP
    d = load_fixture(name)
    params = eval(str(d["params"]))
    transmission = "Full" in params["boundary"] or "Transmission" in params["kernel"]
    show = 0 if transmission else -1
    s, sc, ac, dc = OP.compute_color(d["solved"], d["analytical_solved"], d["vertice_types"], show)
    want = to_complex(d["colour_solved"])
    assert np.abs(s - want).max() <= 1e-15 * max(np.abs(to_complex(d["solved"])).max(), 1.0)
    # the reference's colour/position fields hold FP64 here; the oracle rounds to float32 as ti.f32 does
    for got, key in ((sc, "solved_vert_color"), (ac, "analytical_vert_color"), (dc, "diff_vert_color")):
        assert np.abs(got - d[key]).max() <= 2e-7, key
    for got, key in zip(OP.set_mesh_instances(d["vertices"]), ("solved_vertices", "analytical_vertices",
                                                              "diff_vertices")):
        assert np.abs(got - d[key]).max() <= 4e-7, key


def test_analytic_meshes_match_reference_generators():
    """bem_b200.meshes against the reference's own load_analytical_sphere /
    load_analytical_disk output (tests/golden/meshes_analytical.npz): the
    same vertices, bit for bit, and the same panels in the same order (the
    P0 unknowns are numbered by panel)."""
    from bem_b200.meshes import analytical_disk, analytical_sphere
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "meshes_analytical.npz"))
    cases = {"sphere_default": analytical_sphere(), "sphere_r07_5x6": analytical_sphere(0.7, 5, 6),
             "disk_default": analytical_disk(), "disk_r05_37": analytical_disk(0.5, 37)}
    for tag, (v, f) in cases.items():
        assert np.array_equal(v, d[f"{tag}_vertices"]), tag
        assert np.array_equal(f, d[f"{tag}_panels"]), tag
