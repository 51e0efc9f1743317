"""The drop-in driver (CoreManager / BEMManager on libbem_b200) against the
reference's own outputs (golden fixtures) and the CPU oracle."""
import numpy as np
import pytest
import torch

from tests._util import FIXTURES, load_fixture, rel_err, to_complex, torch_callbacks

pytestmark = pytest.mark.gpu


def _run(d, **extra):
    from bem_b200.managers import CoreManager
    params = eval(str(d["params"]))
    params.update(vertices=d["vertices"], panels=d["panels"])
    params.update(extra)
    fD, fN = torch_callbacks(str(d["data_kind"]), float(params.get("k", 0.0)), d["direction"])
    core = CoreManager(params)
    core.initialization(fD, fN)
    b = core._BEM_manager
    return core, b


@pytest.mark.parametrize("fuse", [False, True])
@pytest.mark.parametrize("name", FIXTURES)
def test_driver_matches_reference_fp64(name, fuse):
    d = load_fixture(name)
    core, b = _run(d, fuse=fuse, fuse_calderon=fuse)
    b._mat_A.zero_()
    if "solve_error" in d:
        # the reference's torch.linalg.solve raised on this exactly singular system
        with pytest.raises(torch.linalg.LinAlgError, match="singular"):
            core._BEM_manager.run()
    else:
        core._BEM_manager.run()
    A = b._mat_A.cpu().numpy()
    assert rel_err(A, to_complex(d["A"])) < 1e-12
    assert rel_err(b.rhs.cpu().numpy(), to_complex(d["rhs"])) < 1e-12
    if "raw_solved" in d and "solve_error" not in d:
        cond = np.linalg.cond(to_complex(d["A"]).reshape(A.shape)) if A.shape[0] < 2000 else 0
        if cond < 1e8:
            assert rel_err(b.raw_solved.cpu().numpy(), to_complex(d["raw_solved"])) < 1e-9
            assert rel_err(b.raw_analytical_solved.cpu().numpy(), to_complex(d["raw_analytical_solved"])) < 1e-12
            # run() ends with compute_color, which shifts the Dirichlet-to-be-solved traces
            assert rel_err(b.solved.cpu().numpy(), to_complex(d["colour_solved"])) < 1e-9
    core.kill()


@pytest.mark.parametrize("name", ["cube_lap_dir_q5", "cube_trans_q3", "ico1_helm_dir_p1_q3"])
def test_driver_mixed_precision(name):
    d = load_fixture(name)
    core, b = _run(d, precision="mixed")
    core.run()
    ref = to_complex(d["raw_solved"])
    # FP32 far field: ~1e-7 relative entry error; refinement converges on the
    # FP64-stored matrix; the bound is the stated mixed-precision tolerance
    assert rel_err(b.raw_solved.cpu().numpy(), ref) < 1e-6
    assert b.solve_info["relres"] <= 1e-12
    core.kill()


@pytest.mark.parametrize("kernel,boundary", [("Laplace", "Dirichlet"), ("Helmholtz", "Neumann")])
def test_driver_on_reference_analytic_sphere(kernel, boundary):
    """The reference's latitude-longitude sphere (object "analytical_sphere":
    poles shared by 17 panels, inward-oriented panels) through the driver,
    against the oracle on the same mesh."""
    from bem_b200.managers import CoreManager
    from bem_b200.meshes import analytical_sphere
    from oracle import oracle as O
    from tests._util import data_callbacks
    k = 1.3 if kernel == "Helmholtz" else 0.0
    params = dict(dim=3, object="analytical_sphere", GaussQR=3, kernel=kernel, boundary=boundary, scope="Interior",
                  k=k, Q_Neumann=0, Q_Dirichlet=1)
    kind = "plane_wave" if kernel == "Helmholtz" else "laplace_point"
    d = np.array([0.6, 0.0, 0.8])
    v, f = analytical_sphere()
    P = O.Problem(v, f, params, *data_callbacks(kind, k, d))
    r = P.run()
    core = CoreManager(params)
    core.initialization(*torch_callbacks(kind, k, d))
    b = core._BEM_manager
    assert np.array_equal(core._mesh_manager.vertices, v)
    b.assemble_system()
    assert rel_err(b._mat_A.cpu().numpy(), r["A"]) < 1e-12
    assert rel_err(b.rhs.cpu().numpy(), r["rhs"]) < 1e-12
    core.kill()


@pytest.mark.parametrize("name", ["cube_helm_mix_ext_q4", "disk24_helm_mix_ext_q3"])
def test_mixed_path_raises_on_singular_system(name):
    """On the exactly singular fixtures the mixed path ends in the FP64
    factorisation, which raises the reference's error type."""
    d = load_fixture(name)
    assert "solve_error" in d
    core, b = _run(d, precision="mixed")
    with pytest.raises(torch.linalg.LinAlgError, match="singular"):
        b.run()
    core.kill()
