"""Host-side checks of the engine that run before any launch (no GPU needed):
operator-space validation, block placement and host-to-device staging."""
import numpy as np
import pytest
import torch

from bem_b200.engine import DeviceSpace, upload


def test_space_records_extents_for_the_launch_checks():
    sp = DeviceSpace.from_numpy([4, 0, 7], 3, [[0, 1, 2], [3, -1, 4], [5, 6, -1]], "cpu")
    assert sp.n_panels == 3 and sp.nb == 3
    assert (sp.max_panel, sp.max_dof) == (7, 6)
    assert sp.panels.dtype == torch.int32 and sp.dof.dtype == torch.int32
    sh = sp.shifted(10)
    assert sh.dof.tolist() == [10, 11, 12, 13, -1, 14, 15, 16, -1]  # skipped dofs stay skipped
    assert sh.max_dof == 16 and sh.max_panel == 7


def test_empty_space():
    sp = DeviceSpace.from_numpy(np.zeros(0, np.int32), 1, np.zeros(0, np.int32), "cpu")
    assert sp.n_panels == 0 and sp.max_panel == -1 and sp.max_dof == -1
    assert sp.shifted(5).max_dof == -1


@pytest.mark.parametrize("panels,nb,dof,msg", [
    ([0, 1], 3, [0, 1, 2], "n_panels"),        # dof table of the wrong size
    ([-1, 2], 1, [0, 1], "negative"),          # negative panel index
    ([3, 3], 1, [0, 1], "only once"),          # a panel twice on one side
])
def test_space_rejects_bad_tables(panels, nb, dof, msg):
    with pytest.raises(ValueError, match=msg):
        DeviceSpace.from_numpy(panels, nb, dof, "cpu")


def test_upload_keeps_values_and_casts():
    a = np.arange(6, dtype=np.int32).reshape(2, 3)[:, ::2]  # non-contiguous
    t = upload(a, "cpu")
    assert t.dtype == torch.int32 and t.tolist() == [[0, 2], [3, 5]]
    f = upload([1.5, 2.5], "cpu", torch.float64)
    assert f.dtype == torch.float64 and f.tolist() == [1.5, 2.5]
    c = upload(np.array([1 + 2j]), "cpu")
    assert c.dtype == torch.complex128 and complex(c[0]) == 1 + 2j


def test_complex_pack_round_trip():
    """warp_tensor / unwarp_tensor (src/BEM_functions/utils/io.py:4-30):
    [..., 2] <-> complex, [..., 1] <-> real, anything else rejected."""
    from bem_b200.utils.io import unwarp_tensor, warp_tensor
    z = torch.randn(5, 3, dtype=torch.complex128)
    packed = unwarp_tensor(z)
    assert packed.shape == (5, 3, 2) and torch.equal(warp_tensor(packed), z)
    r = torch.randn(4, dtype=torch.float64)
    assert unwarp_tensor(r).shape == (4, 1) and torch.equal(warp_tensor(unwarp_tensor(r)), r)
    with pytest.raises(NotImplementedError):
        warp_tensor(torch.zeros(2, 3))


@pytest.mark.parametrize("quirk,honour,show,want", [
    (True, None, "Dirichlet", -1),    # reference behaviour: the parameter is stored, not read
    (False, None, "Dirichlet", 1),    # default follows quirk
    (True, True, "Neumann", 0),       # reference quadrature, show honoured
    (False, False, "Neumann", -1),    # corrected quadrature, reference colouring
])
def test_show_parameter_is_its_own_switch(quirk, honour, show, want):
    """`honour_show` decides whether `show` selects the splat and colouring,
    independently of the quadrature quirk flag (BEM_manager.py:28,43-50)."""
    from bem_b200.managers import CoreManager
    p = dict(dim=3, object="icosphere1", GaussQR=3, kernel="Laplace", boundary="Dirichlet", scope="Interior",
             show=show, quirk=quirk, device="cpu")
    if honour is not None:
        p["honour_show"] = honour
    b = CoreManager(p)._BEM_manager
    assert b._show == want
