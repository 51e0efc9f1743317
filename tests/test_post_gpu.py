"""Headless post-processing (bem_compute_color, bem_set_mesh_instances): the
colour and position buffers that end BEMManager.run (BEM_manager.py:527-606),
against the oracle (oracle/post.py, pinned to the reference's own kernels by
tests/test_oracle_golden.py) and the golden fixtures.

Tolerances: the shifted traces are FP64 (1e-12 of the largest trace the shift
is computed from; the mean's summation order differs); colours and positions
are float32 buffers (2e-6 absolute on values of order one).
"""
import numpy as np
import pytest
import torch

from oracle import post as OP
from tests._util import FIXTURES, load_fixture, to_complex, torch_callbacks

pytestmark = pytest.mark.gpu

TOL_F32 = 2e-6


@pytest.fixture(scope="module")
def engine():
    from bem_b200.engine import Engine
    e = Engine()
    yield e
    e.close()


def _buffers(nv):
    return [torch.zeros(nv, 3, dtype=torch.float32, device="cuda") for _ in range(3)]


def _run_colour(engine, solved, exact, vt, show):
    """compute_color through the C ABI; returns (shifted solved, colours)."""
    s = torch.as_tensor(solved, device="cuda").clone()
    a = torch.as_tensor(exact, device="cuda")
    t = torch.as_tensor(vt.astype(np.int32), device="cuda")
    bufs = _buffers(len(vt))
    engine.compute_color(s, a, t, show, *bufs)
    torch.cuda.synchronize()
    return s.cpu().numpy(), [b.cpu().numpy() for b in bufs]


def _check_colour(pre, exact, vt, show, got_s, got_c):
    want_s, *want_c = OP.compute_color(pre, exact, vt, show)
    scale = max(np.abs(pre).max(), np.abs(want_s).max(), 1e-300)
    assert np.abs(got_s - want_s).max() <= 1e-12 * scale
    # The shift carries the rounding of traces of size `scale`; a colour is a
    # trace divided by a class maximum of |exact|.
    na = np.abs(np.asarray(exact))
    isd = np.asarray(vt) == OP.V_DIRICHLET
    m = min([na[c].max() for c in (isd, ~isd) if c.any()] + [np.inf])
    tol = TOL_F32 + 1e-12 * scale / max(m, 1e-300)
    assert np.abs(got_c[1] - want_c[1]).max() <= TOL_F32  # exact-trace colour
    assert np.abs(got_c[0] - want_c[0]).max() <= tol
    assert np.abs(got_c[2] - want_c[2]).max() <= tol


@pytest.mark.parametrize("complex_", [False, True])
@pytest.mark.parametrize("show", [-1, 0, 1])
@pytest.mark.parametrize("types", ["mixed", "all_neumann", "all_dirichlet", "both"])
def test_compute_color_matches_oracle(engine, complex_, show, types):
    """Every branch: vertex classes (with and without Dirichlet-to-be-solved
    vertices, so the mean and both maxima take their initial values too),
    each show mode, real and complex traces, nv > the block size."""
    from bem_b200.meshes import analytical_disk
    v, f = analytical_disk(1.0, 2500)
    engine.set_mesh(v, f, 2, dim=2)
    nv = len(v)
    rng = np.random.default_rng(11)
    vt = {"mixed": rng.integers(0, 3, nv), "all_neumann": np.zeros(nv, np.int64),
          "all_dirichlet": np.ones(nv, np.int64), "both": np.full(nv, 2)}[types]
    if complex_:
        exact = rng.standard_normal(nv) + 1j * rng.standard_normal(nv)
        pre = exact + 0.3 + 0.1 * (rng.standard_normal(nv) + 1j * rng.standard_normal(nv))
    else:
        exact = rng.standard_normal(nv)
        pre = exact - 0.7 + 0.05 * rng.standard_normal(nv)
    got_s, got_c = _run_colour(engine, pre, exact, vt, show)
    _check_colour(pre, exact, vt, show, got_s, got_c)


def test_compute_color_small_mesh(engine):
    """nv below one warp: most of the block's threads hold no vertex."""
    v = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    f = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], np.int32)
    engine.set_mesh(v, f, 2)
    exact = np.array([1.0, -2.0, 0.5, 3.0])
    pre = np.array([0.2, -1.0, 0.9, 2.5])
    vt = np.array([1, 0, 1, 2])
    for show in (-1, 0, 1):
        got_s, got_c = _run_colour(engine, pre, exact, vt, show)
        _check_colour(pre, exact, vt, show, got_s, got_c)


@pytest.mark.parametrize("dim", [2, 3])
def test_set_mesh_instances_matches_oracle(engine, dim):
    from bem_b200.meshes import analytical_disk, icosphere
    v, f = analytical_disk(0.5, 300) if dim == 2 else icosphere(3)
    engine.set_mesh(v, f, 2, dim=dim)
    bufs = _buffers(len(v))
    engine.set_mesh_instances(*bufs)
    torch.cuda.synchronize()
    for g, w in zip(bufs, OP.set_mesh_instances(v)):
        assert np.array_equal(g.cpu().numpy(), w)


def test_compute_color_rejects_bad_buffers(engine):
    from bem_b200.meshes import icosphere
    v, f = icosphere(1)
    engine.set_mesh(v, f, 2)
    nv = len(v)
    s = torch.zeros(nv, dtype=torch.float64, device="cuda")
    t = torch.zeros(nv, dtype=torch.int32, device="cuda")
    with pytest.raises(ValueError):
        engine.compute_color(s, s, t, -1, *_buffers(nv - 1))
    with pytest.raises(ValueError):
        engine.compute_color(s, s.to(torch.complex128), t, -1, *_buffers(nv))
    with pytest.raises(ValueError):
        engine.compute_color(s, s, t.to(torch.int64), -1, *_buffers(nv))


@pytest.mark.parametrize("name", FIXTURES)
def test_driver_colour_buffers(name):
    """BEMManager.run's post-processing on the golden cases: the shifted
    traces and colours against the oracle applied to this build's own splat,
    and against the reference's buffers where the system is well conditioned
    (the singular interior Neumann problem leaves its constant to rounding)."""
    from bem_b200.managers import CoreManager
    d = load_fixture(name)
    if "solve_error" in d:
        pytest.skip("exactly singular: the reference's run() raises in its solve, before the colouring")
    params = eval(str(d["params"]))
    params.update(vertices=d["vertices"], panels=d["panels"])
    fD, fN = torch_callbacks(str(d["data_kind"]), float(params.get("k", 0.0)), d["direction"])
    core = CoreManager(params)
    core.initialization(fD, fN)
    b = core._BEM_manager
    b.assemble_system()
    b.compute_analytical_raw_solved()
    b.solve()
    b.splat_u_from_raw_solved_to_vertices()
    pre = b.solved.cpu().numpy().copy()
    exact = b.analytical_solved.cpu().numpy()
    b.compute_color()
    b.set_mesh_instances()
    got_s = b.solved.cpu().numpy()
    got_c = [getattr(b, k).cpu().numpy() for k in ("solved_vert_color", "analytical_vert_color", "diff_vert_color")]
    vt = d["vertice_types"]
    _check_colour(pre, exact, vt, b._show, got_s, got_c)
    # exact-trace colours and positions do not depend on the solve
    assert np.abs(got_c[1] - d["analytical_vert_color"]).max() <= TOL_F32
    for key in ("solved_vertices", "analytical_vertices", "diff_vertices"):
        assert np.abs(getattr(b, key).cpu().numpy() - d[key]).max() <= TOL_F32
    A = to_complex(d["A"])
    if "solve_error" not in d and np.linalg.cond(A.reshape(A.shape[0], -1)) < 1e8:
        want = to_complex(d["colour_solved"])
        assert np.abs(got_s - want).max() <= 1e-9 * max(np.abs(want).max(), 1e-300)
        assert np.abs(got_c[0] - d["solved_vert_color"]).max() <= 1e-6
        assert np.abs(got_c[2] - d["diff_vert_color"]).max() <= 1e-6
    core.kill()
