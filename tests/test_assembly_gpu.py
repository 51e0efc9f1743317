"""GPU assembly (libbem_b200 through the C ABI) against the FP64 CPU oracle.

Tolerances: FP64 path 1e-12 of the block's max entry (different summation
order only); mixed path (separate pairs in FP32) 2e-6.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests._util import full_spaces, load_fixture, rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 2e-6


@pytest.fixture(scope="module")
def engine():
    from bem_b200.engine import Engine
    e = Engine()
    yield e
    e.close()


def _meshes():
    from bem_b200 import icosphere
    d = load_fixture("cube_lap_dir_q5")
    v2, f2 = icosphere(2)
    return {"cube": (d["vertices"], d["panels"]), "ico2": (v2, f2)}


MESHES = _meshes()


def _space(engine, v, f, nb):
    from bem_b200.engine import DeviceSpace
    p, nb, dof = full_spaces(len(v), f, nb)
    return (p, nb, dof), DeviceSpace.from_numpy(p, nb, dof, engine.device)


def _oracle_block(v, f, op, helm, k, k2, Q, quirk, ts, rs, nrow, ncol):
    out = np.zeros((nrow, ncol), np.complex128 if helm else np.float64)
    O.assemble(v, f, op, helm, k, k2, Q, quirk, ts, rs, out=out)
    return out


CASES = [
    # (mesh, op, helm, nbx, nby, Q, quirk)
    ("cube", O.OP_V, False, 1, 1, 5, True),
    ("cube", O.OP_K, True, 1, 3, 4, True),
    ("cube", O.OP_KP, True, 3, 1, 4, False),
    ("cube", O.OP_W, True, 3, 3, 3, True),
    ("ico2", O.OP_V, False, 1, 1, 5, True),
    ("ico2", O.OP_V, True, 1, 1, 4, False),
    ("ico2", O.OP_V, True, 3, 3, 3, True),
    ("ico2", O.OP_V, True, 3, 3, 3, False),
    ("ico2", O.OP_K, False, 1, 3, 4, True),
    ("ico2", O.OP_K, True, 1, 3, 3, False),
    ("ico2", O.OP_KP, False, 3, 1, 3, True),
    ("ico2", O.OP_W, False, 3, 3, 3, True),
    ("ico2", O.OP_W, True, 3, 3, 3, False),
    ("ico2", O.OP_W, True, 1, 1, 3, True),
]


@pytest.mark.parametrize("mesh,op,helm,nbx,nby,Q,quirk", CASES)
def test_dense_block_fp64(engine, mesh, op, helm, nbx, nby, Q, quirk):
    v, f = MESHES[mesh]
    engine.set_mesh(v, f, Q)
    k = 2.5 if helm else 0.0
    k2 = k * k
    ts, tsd = _space(engine, v, f, nbx)
    rs, rsd = _space(engine, v, f, nby)
    nrow = len(f) if nbx == 1 else len(v)
    ncol = len(f) if nby == 1 else len(v)
    ref = _oracle_block(v, f, op, helm, k, k2, Q, quirk, ts, rs, nrow, ncol)
    out = torch.zeros(nrow, ncol, dtype=torch.complex128 if helm else torch.float64, device="cuda")
    desc = engine.op_desc(op, helm, k, k2, quirk=quirk)
    engine.assemble(desc, tsd, rsd, out)
    got = out.cpu().numpy()
    assert rel_err(got, ref) < FP64_TOL


@pytest.mark.parametrize("helm", [False, True])
def test_dense_block_mixed(engine, helm):
    from bem_b200 import _lib as L
    v, f = MESHES["ico2"]
    engine.set_mesh(v, f, 4)
    k = 3.0 if helm else 0.0
    ts, tsd = _space(engine, v, f, 1)
    ref = _oracle_block(v, f, O.OP_V, helm, k, k * k, 4, True, ts, ts, len(f), len(f))
    out = torch.zeros(len(f), len(f), dtype=torch.complex128 if helm else torch.float64, device="cuda")
    engine.assemble(engine.op_desc(O.OP_V, helm, k, k * k, precision=L.PREC_MIXED), tsd, tsd, out)
    assert rel_err(out.cpu().numpy(), ref) < MIXED_TOL


def test_transposed_output_and_scale(engine):
    v, f = MESHES["cube"]
    engine.set_mesh(v, f, 3)
    ts, tsd = _space(engine, v, f, 1)
    rs, rsd = _space(engine, v, f, 3)
    n = len(f) + len(v)
    A = torch.zeros(n, n, dtype=torch.complex128, device="cuda")
    # K block at rows [nv, n), cols [0, nv); -K^T at rows [0, nv), cols [nv, n)
    tsd_off = tsd.shifted(len(v))
    desc = engine.op_desc(O.OP_K, True, 1.5, 2.25)
    engine.assemble(desc, tsd_off, rsd, A, scale=2.0, out_t=A, scale_t=-3.0)
    ref = np.zeros((len(f), len(v)), np.complex128)
    O.assemble(v, f, O.OP_K, True, 1.5, 2.25, 3, True, ts, rs, out=ref)
    got = A.cpu().numpy()
    assert rel_err(got[len(v):, :len(v)], 2.0 * ref) < FP64_TOL
    assert rel_err(got[:len(v), len(v):], -3.0 * ref.T) < FP64_TOL


@pytest.mark.parametrize("op,nbx,nby,conj", [(O.OP_K, 1, 3, True), (O.OP_V, 1, 1, False), (O.OP_KP, 3, 1, True),
                                             (O.OP_W, 3, 3, False)])
def test_apply_matches_oracle(engine, op, nbx, nby, conj):
    v, f = MESHES["ico2"]
    engine.set_mesh(v, f, 3)
    ts, tsd = _space(engine, v, f, nbx)
    rs, rsd = _space(engine, v, f, nby)
    nrow = len(f) if nbx == 1 else len(v)
    ncol = len(f) if nby == 1 else len(v)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(ncol) + 1j * rng.standard_normal(ncol)
    y = np.zeros(nrow, np.complex128)
    O.assemble(v, f, op, True, 2.0, 4.0, 3, True, ts, rs, x=x, y=y, scale=-0.5, conj_x=conj)
    xd = torch.as_tensor(x, device="cuda")
    yd = torch.zeros(nrow, dtype=torch.complex128, device="cuda")
    engine.apply(engine.op_desc(op, True, 2.0, 4.0), tsd, rsd, xd, yd, scale=-0.5, conj_x=conj)
    assert rel_err(yd.cpu().numpy(), y) < FP64_TOL


def test_mass_block(engine):
    v, f = MESHES["ico2"]
    engine.set_mesh(v, f, 5)
    ts, tsd = _space(engine, v, f, 1)
    rs, rsd = _space(engine, v, f, 3)
    ref = np.zeros((len(f), len(v)))
    O.mass(v, f, 5, ts[0], 1, ts[2], 3, rs[2], out=ref)
    out = torch.zeros(len(f), len(v), dtype=torch.float64, device="cuda")
    engine.mass(tsd, rsd, out=out)
    assert rel_err(out.cpu().numpy(), ref) < FP64_TOL
    # P0 x P1 mass of a panel is area/3 per vertex
    areas, _ = engine.geometry()
    assert np.allclose(out.sum(1).cpu().numpy(), areas.cpu().numpy(), rtol=1e-13)


def test_near_pair_count_icosphere(engine):
    from bem_b200 import icosphere
    v, f = icosphere(3)
    engine.set_mesh(v, f, 3)
    # each panel: itself + 3 edge neighbours + 9 (or 8 at the 12 valence-5 vertices) vertex neighbours
    n = engine.near_pairs
    assert 12 * len(f) < n <= 13 * len(f)


def _near_list_reference(f):
    """The ordered pairs sharing a vertex index, by relation, in (i, j)
    order: a numpy restatement of get_panels_relation
    (mesh_manager.py:538-573) over the vertex-sharing candidates."""
    from oracle import oracle as O
    f = np.asarray(f)
    nt = len(f)
    by_v = {}
    for p in range(nt):
        for c in f[p]:
            by_v.setdefault(int(c), []).append(p)
    rows = []
    for i in range(nt):
        for j in sorted({j for c in f[i] for j in by_v[int(c)]}):
            rel = O.relation(f, i, j)
            if rel != 0:
                rows.append((i, j, rel))
    return np.array(rows, np.int32).reshape(-1, 3)


@pytest.mark.parametrize("mesh", ["cube", "ico2", "analytical_sphere", "perturbed3"])
def test_near_pair_list_matches_reference(engine, mesh):
    """The device-built near-pair list: every vertex-sharing ordered pair with
    the oracle's relation, in (test, trial) order; parameter orders in range."""
    from bem_b200.meshes import analytical_sphere, perturbed_sphere
    if mesh in MESHES:
        v, f = MESHES[mesh]
    elif mesh == "analytical_sphere":
        v, f = analytical_sphere()
    else:
        v, f = perturbed_sphere(3, lmax=6, amplitude=0.05, seed=0)
    engine.set_mesh(v, f, 3)
    got = engine.near_pair_list()
    ref = _near_list_reference(f)
    assert got.shape[0] == ref.shape[0]
    assert np.array_equal(got[:, :3], ref)
    # packed orders: two 6-bit permutations of (0, 1, 2)
    for sh in (0, 6):
        perm = [(got[:, 3] >> (sh + 2 * s)) & 3 for s in range(3)]
        assert np.all(np.sort(np.stack(perm, 1), 1) == np.array([0, 1, 2]))


def test_bad_mesh_rejected(engine):
    from bem_b200._lib import BemError
    v = np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0]], dtype=np.float64)  # collinear -> zero area
    with pytest.raises(BemError):
        engine.set_mesh(v, np.array([[0, 1, 2]]), 3)
    with pytest.raises(BemError):
        engine.set_mesh(v, np.array([[0, 1, 5]]), 3)


@pytest.mark.parametrize("sym", [True, False])
@pytest.mark.parametrize("helm", [False, True])
@pytest.mark.parametrize("fp32", [False, True])
def test_fused_dirichlet_pass(engine, helm, fp32, sym):
    """V and K g in one sweep == V assembly + K g apply (oracle)."""
    from bem_b200 import _lib as L
    v, f = MESHES["ico2"]
    Q = 4
    engine.set_mesh(v, f, Q)
    k = 2.0 if helm else 0.0
    ts, tsd = _space(engine, v, f, 1)
    ds, dsd = _space(engine, v, f, 3)
    nt, nv = len(f), len(v)
    rng = np.random.default_rng(3)
    g = rng.standard_normal(nv) + (1j * rng.standard_normal(nv) if helm else 0)
    Vref = _oracle_block(v, f, O.OP_V, helm, k, k * k, Q, True, ts, ts, nt, nt)
    yref = np.zeros(nt, np.complex128 if helm else np.float64)
    O.assemble(v, f, O.OP_K, helm, k, k * k, Q, True, ts, ds, x=g, y=yref, scale=0.75, conj_x=helm)
    dt = torch.complex128 if helm else torch.float64
    V = torch.zeros(nt, nt, dtype=dt, device="cuda")
    y = torch.zeros(nt, dtype=dt, device="cuda")
    gd = torch.as_tensor(g, device="cuda")
    desc = engine.op_desc(O.OP_V, helm, k, k * k, precision=L.PREC_MIXED if fp32 else L.PREC_FP64)
    # sym: identical test/trial spaces select the symmetric i<j sweep; a copy
    # of the trial space (other device pointers) selects the general sweep
    trial = tsd if sym else _space(engine, v, f, 1)[1]
    engine.assemble_dirichlet(desc, tsd, trial, V, tsd, dsd, gd, y, scale=1.0, scale_k=0.75, conj_g=helm)
    tol = MIXED_TOL if fp32 else FP64_TOL
    assert rel_err(V.cpu().numpy(), Vref) < tol
    assert rel_err(y.cpu().numpy(), yref) < tol
