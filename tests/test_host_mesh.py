"""MeshManager's mesh sources on the host (no GPU): the reference's object
names and normalisation (src/managers/mesh_manager.py:67-139,479-536)."""
import numpy as np
import pytest

from bem_b200.meshes import analytical_disk, analytical_sphere


def _mesh_manager(**params):
    from bem_b200.managers import CoreManager
    p = dict(dim=3, object="sphere", GaussQR=3, kernel="Laplace", boundary="Dirichlet", scope="Interior")
    p.update(params)
    core = CoreManager(p)  # no device work before initialization()
    mm = core._mesh_manager
    mm.initialization()
    return mm


@pytest.mark.parametrize("name", ["analytical_sphere", "my_analytical"])
def test_analytical_object_names_load_the_reference_sphere(name):
    mm = _mesh_manager(object=name)
    v, f = analytical_sphere()
    assert np.array_equal(mm.vertices, v) and np.array_equal(mm.panels, f)
    assert (mm.num_of_vertices, mm.num_of_panels) == (2 + 16 * 17, 2 * 17 + 2 * 15 * 17)
    # consistently oriented: the reference's generator turns every panel inward
    cent = v[f].mean(axis=1)
    assert ((cent * mm.panel_normals).sum(1) < 0).all()
    assert 0.97 * 4 * np.pi < mm.panel_areas.sum() < 4 * np.pi  # an inscribed polyhedron


def test_asset_is_centred_and_normalised(tmp_path):
    v = np.array([[0, 0, 0], [2, 0, 0], [0, 4, 0], [0, 0, 6]], dtype=np.float64) + 10.0
    f = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]])
    path = tmp_path / "tet.obj"
    path.write_text("".join("v %.17g %.17g %.17g\n" % tuple(p) for p in v) + "".join("f %d %d %d\n" % tuple(t + 1) for t in f))
    mm = _mesh_manager(object=str(path))
    want = (v - v.mean(axis=0)) / np.abs(v - v.mean(axis=0)).max()
    assert np.array_equal(mm.vertices, want)
    a, _ = mm.load_asset(scale=2.0, translate=np.zeros((1, 3)))  # explicit scale: no normalisation
    assert np.array_equal(a, v * 2.0)


def test_2d_default_is_the_reference_disk():
    mm = _mesh_manager(dim=2, object="disk")
    v, f = analytical_disk()
    assert np.array_equal(mm.vertices, v) and np.array_equal(mm.panels, f)


def test_missing_asset_raises():
    with pytest.raises(FileNotFoundError):
        _mesh_manager(object="no_such_mesh_here")


@pytest.mark.parametrize("mesh", ["icosphere2", "analytical_sphere", "disk"])
@pytest.mark.parametrize("boundary", ["Dirichlet", "Neumann", "Mix", "Full"])
@pytest.mark.parametrize("qn,qd", [(0, 1), (1, 1), (0, 0), (1, 0)])
def test_partitions_match_the_oracle(mesh, boundary, qn, qd):
    """The BVP partition, the DOF counts and the local<->global maps
    (mesh_manager.py:166-389,415-445) and the per-vertex geometry, against the
    oracle's restatement (pinned to the reference's fixtures)."""
    from oracle import oracle as O
    dim = 2 if mesh == "disk" else 3
    mm = _mesh_manager(object=mesh, dim=dim, boundary=boundary, Q_Neumann=qn, Q_Dirichlet=qd)
    om = O.Mesh(mm.vertices, mm.panels, boundary=boundary, Q_Neumann=qn, Q_Dirichlet=qd, dim=dim)
    assert (mm.N_Neumann, mm.M_Dirichlet) == (om.N_N, om.M_D)
    assert (mm.num_of_panels_Neumann, mm.num_of_panels_Dirichlet) == (om.nP_N, om.nP_D)
    for ours, theirs in ((mm.panel_types, om.panel_types), (mm.vertice_types, om.vert_types),
                         (mm.Dirichlet_index, om.D_index), (mm.Neumann_index, om.N_index),
                         (mm.map_global_Neumann_to_local, om.map_N), (mm.map_global_Dirichlet_to_local, om.map_D)):
        assert np.array_equal(np.asarray(ours), np.asarray(theirs))
    assert np.allclose(mm.vert_areas, om.vert_areas, rtol=1e-14, atol=0)
    assert np.allclose(mm.vert_normals, om.vert_normals, rtol=0, atol=1e-14)


@pytest.mark.parametrize("bad,exc", [
    (dict(kernel="Stokes"), RuntimeError),             # BEM_manager.py:40-50
    (dict(show="Both"), RuntimeError),
    (dict(precision="fp16"), ValueError),
    (dict(dim=4), NotImplementedError),
    (dict(Q_Neumann=2), AssertionError),
])
def test_bad_configuration_is_rejected_on_the_host(bad, exc):
    from bem_b200.managers import CoreManager
    p = dict(dim=3, object="icosphere1", GaussQR=3, kernel="Laplace", boundary="Dirichlet", scope="Interior")
    p.update(bad)
    with pytest.raises(exc):
        CoreManager(p)


def test_bad_boundary_type_is_rejected():
    with pytest.raises(RuntimeError, match="Boundary Type"):
        _mesh_manager(object="icosphere1", boundary="Robin")


@pytest.mark.parametrize("case", ["nan_vertex", "index_out_of_range", "zero_area", "wrong_width"])
def test_bad_mesh_is_rejected_on_the_host(case):
    v, f = analytical_sphere(1.0, 4, 5)
    v, f = v.copy(), f.copy()
    if case == "nan_vertex":
        v[3, 1] = np.nan
    elif case == "index_out_of_range":
        f[7, 2] = len(v)
    elif case == "zero_area":
        f[2] = [f[2, 0], f[2, 0], f[2, 1]]
    else:
        f = f[:, :2]
    with pytest.raises(ValueError):
        _mesh_manager(vertices=v, panels=f)


def test_obj_reader_forms(tmp_path):
    """`a/b/c` vertex references, negative (relative) indices and polygons,
    fan-triangulated from their first vertex."""
    from bem_b200.meshes import load_obj
    text = ("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvn 0 0 1\nvt 0 0\n"
            "f 1/1/1 2/1/1 3/1/1\n"      # slash forms
            "f -4 -2 -1\n"               # relative: vertices 1, 3, 4
            "f 1 2 3 4\n")               # quad -> (1,2,3), (1,3,4)
    path = tmp_path / "forms.obj"
    path.write_text(text)
    v, f = load_obj(str(path), normalise=False)
    assert v.shape == (4, 3)
    assert f.tolist() == [[0, 1, 2], [0, 2, 3], [0, 1, 2], [0, 2, 3]]


@pytest.mark.parametrize("show,quirk,transmission,want", [
    ("Dirichlet", True, False, -1),   # the reference reads _show, never set from the parameter
    ("Neumann", True, False, -1),
    ("Default", True, True, 0),       # transmission: Neumann (BEM_manager.py:52-53)
    ("Dirichlet", False, False, 1),   # corrected mode honours the parameter
    ("Neumann", False, False, 0),
    ("Dirichlet", False, True, 1),
])
def test_show_parameter_follows_the_reference(show, quirk, transmission, want):
    from bem_b200.managers import CoreManager
    p = dict(dim=3, object="icosphere1", GaussQR=3, scope="Interior", show=show, quirk=quirk,
             kernel="Helmholtz_Transmission" if transmission else "Laplace",
             boundary="Full" if transmission else "Dirichlet", k=1.0, n_i=1.0, n_o=1.0)
    b = CoreManager(p)._BEM_manager
    assert b._show == want
    assert b.show == {"Neumann": 0, "Dirichlet": 1, "Default": -1}[show]
