"""The tcgen05 (TF32, three-product split) trailing update of the FP32 LU:
the factors reproduce P A = L U to FP32 accuracy, for real and complex
matrices whose sizes leave partial 128 x 128 tiles and a short last panel."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from bem_b200.engine import Engine
    e = Engine()
    yield e
    e.close()


def _unpack(LU, piv):
    n = LU.shape[0]
    L = np.tril(LU, -1) + np.eye(n)
    U = np.triu(LU)
    perm = np.arange(n)
    for i, p in enumerate(piv):
        perm[[i, p]] = perm[[p, i]]
    return L, U, perm


@pytest.mark.parametrize("n", [200, 453])
@pytest.mark.parametrize("cplx", [False, True])
def test_tiled_fp32_lu_residual(engine, n, cplx):
    rng = np.random.default_rng(n + cplx)
    A = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    A = A + 2 * n ** 0.5 * np.eye(n)
    dt = torch.complex64 if cplx else torch.float32
    LU = torch.as_tensor(A, device="cuda").to(dt).contiguous()
    piv, dinv, info = engine.lu_factor_tiled(LU)
    assert int(info.item()) == 0
    L, U, perm = _unpack(LU.cpu().numpy().astype(np.complex128 if cplx else np.float64), piv.cpu().numpy())
    res = np.abs(L @ U - A.astype(np.complex64 if cplx else np.float32)[perm]).max() / np.abs(A).max()
    # FP32 arithmetic (TF32 x 3 on the tensor cores): a few hundred ulps at most
    assert res < 5e-5


@pytest.mark.parametrize("n,cplx", [(1500, True), (2000, False), (1100, True)])
def test_tma_fed_update_lu_residual(engine, n, cplx):
    """The TMA-fed persistent trailing update (BEM_TUNE_LU_UPDATE = 2: TF32
    hi / lo operands split once per update, 128-byte-swizzled TMA stages,
    tcgen05 kind::tf32, TMEM double buffer) on sizes whose large updates
    cover more C tiles than SMs: P A = L U to FP32 accuracy, as the
    register-staged form."""
    from bem_b200 import _lib as L
    rng = np.random.default_rng(n + cplx)
    A = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    A = A + 2 * n ** 0.5 * np.eye(n)
    dt = torch.complex64 if cplx else torch.float32
    res = {}
    for form in (2, 1):
        LU = torch.as_tensor(A, device="cuda").to(dt).contiguous()
        engine.set_tuning(L.TUNE_LU_UPDATE, form)
        try:
            piv, dinv, info = engine.lu_factor_tiled(LU)
            torch.cuda.synchronize()
        finally:
            engine.set_tuning(L.TUNE_LU_UPDATE, 0)
        assert int(info.item()) == 0
        Lm, U, perm = _unpack(LU.cpu().numpy().astype(np.complex128 if cplx else np.float64), piv.cpu().numpy())
        res[form] = np.abs(Lm @ U - A.astype(np.complex64 if cplx else np.float32)[perm]).max() / np.abs(A).max()
    assert res[2] < 5e-5 and res[2] < 4 * res[1] + 1e-6, res
