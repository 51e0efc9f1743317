"""The other forms of the tensor-core normal matrix (BEM_TUNE_GRAM_PAIR = 2:
gram_tc2_kernel, tcgen05 cta_group::2 on 256 x 128 tiles; 3: one CTA with
sixteen epilogue warps) against the default one-CTA form and the FP64
product: the normal matrix of the least squares (bem_gram) and the Cholesky
whose trailing updates it forms (bem_chol_factor)."""
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


def _gram(engine, A, P, form, tensor_cores=True):
    from bem_b200 import _lib as L
    n = A.shape[0]
    out = torch.zeros(n, n, dtype=A.dtype, device=A.device)
    d = torch.empty(n, dtype=torch.float64, device=A.device)
    engine.set_tuning(L.TUNE_GRAM_PAIR, form)
    try:
        engine.gram(A, P, out, d, tensor_cores=tensor_cores)
    finally:
        engine.set_tuning(L.TUNE_GRAM_PAIR, 0)
    torch.cuda.synchronize()
    return out, d


@pytest.mark.parametrize("form", [2, 3])
@pytest.mark.parametrize("cplx", [True, False])
@pytest.mark.parametrize("n", [50, 130, 300, 1000])
def test_pair_gram_matches_single_and_fp64(engine, n, cplx, form):
    """Same products, different tile shape: the two tensor-core forms agree
    to the FP32 rounding of their TMEM sums, and both match the FP64 normal
    matrix to the split's accuracy."""
    g = torch.Generator(device="cuda").manual_seed(n)
    dt = torch.complex128 if cplx else torch.float64
    A = torch.randn(n, n, dtype=dt, device="cuda", generator=g)
    P = torch.randn(n, n, dtype=dt, device="cuda", generator=g)
    N2, d2 = _gram(engine, A, P, form)
    N1, d1 = _gram(engine, A, P, 1)
    N0, d0 = _gram(engine, A, P, 1, tensor_cores=False)
    assert torch.equal(d1, d2) and torch.equal(d0, d2)
    scale = float(N0.abs().max())
    assert float((N2 - N1).abs().max()) / scale < 2e-6
    assert float((N2 - N0).abs().max()) / scale < 2e-6
    # Hermitian, real diagonal
    assert float((N2 - N2.conj().T).abs().max()) / scale < 1e-12
    if cplx:
        assert float(torch.diagonal(N2).imag.abs().max()) == 0.0


@pytest.mark.parametrize("form", [2, 3])
@pytest.mark.parametrize("cplx", [True, False])
@pytest.mark.parametrize("n", [300, 1333])
def test_pair_cholesky_updates(engine, n, cplx, form):
    """The Cholesky's tcgen05 trailing updates in the pair form solve like the
    one-CTA form (FP64 Schur complement, split products)."""
    from bem_b200 import _lib as L
    rng = np.random.default_rng(n)
    G = rng.standard_normal((2 * n, n)) + (1j * rng.standard_normal((2 * n, n)) if cplx else 0)
    N = G.conj().T @ G / n
    d = 1.0 / np.sqrt(np.real(np.diag(N)))
    N = N * d[:, None] * d[None, :]
    dt = torch.complex128 if cplx else torch.float64
    b = rng.standard_normal(n) + (1j * rng.standard_normal(n) if cplx else 0)
    ref = np.linalg.solve(N, b)
    xs = []
    for fm in (form, 1):
        F = torch.as_tensor(N, dtype=dt, device="cuda").clone()
        engine.set_tuning(L.TUNE_GRAM_PAIR, fm)
        try:
            piv, dinv, info = engine.chol_factor(F, tensor_cores=True)
        finally:
            engine.set_tuning(L.TUNE_GRAM_PAIR, 0)
        assert int(info.item()) == 0
        x = torch.as_tensor(b, dtype=dt, device="cuda").contiguous()
        engine.lu_solve_tiled(F, piv, dinv, x)
        xs.append(x.cpu().numpy())
        assert np.linalg.norm(xs[-1] - ref) / np.linalg.norm(ref) < 1e-5
    assert np.linalg.norm(xs[0] - xs[1]) / np.linalg.norm(ref) < 1e-5
