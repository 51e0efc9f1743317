"""k-batched assembly (bem_assemble_batch) against the per-wavenumber
assembly (bem_assemble) and the oracle: every operator, P0 and P1 spaces,
FP64 and mixed precision, 2- and 4-wavenumber launches with padded tails; and
the batched transmission operators of the wavenumber sweep against the
per-k ones (get_augment_mat_A1_inv_norm's sequence, BEM_manager.py:952-988)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

KS = [1.0, 2.5, 3.75, 6.0, 7.5]  # five wavenumbers: full and padded groups of 2 and 4


def rel_err(a, b):
    a = a.cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = b.cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _engine(subdiv=2, Q=4):
    from bem_b200 import icosphere
    from bem_b200.engine import Engine
    v, f = icosphere(subdiv)
    eng = Engine("cuda:0")
    eng.set_mesh(v, f, Q)
    return eng, v, f


def _spaces(eng, f, nv, nbx, nby):
    from bem_b200.engine import DeviceSpace
    nt = len(f)
    panels = np.arange(nt, dtype=np.int32)
    out = []
    for nb in (nbx, nby):
        dof = panels.reshape(nt, 1) if nb == 1 else f.astype(np.int32)
        out.append((DeviceSpace.from_numpy(panels, nb, dof.reshape(-1), eng.device), nt if nb == 1 else nv))
    return out


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("op,nbx,nby", [(0, 1, 1), (0, 3, 3), (1, 1, 3), (1, 3, 3), (2, 3, 1), (3, 3, 3)])
@pytest.mark.parametrize("group", [0, 2, 4])
def test_batched_blocks_equal_per_k(prec, op, nbx, nby, group):
    from bem_b200 import _lib as L
    from bem_b200.engine import Engine
    eng, v, f = _engine()
    try:
        eng.set_tuning(L.TUNE_KBATCH_GROUP, group)
        (test, nr), (trial, nc) = _spaces(eng, f, len(v), nbx, nby)
        p = L.PREC_MIXED if prec == "mixed" else L.PREC_FP64
        desc = Engine.op_desc(op, True, 0.0, 0.0, quirk=True, precision=p)
        k2s = [k * k for k in KS]
        with_t = op == 1
        if with_t:  # out and its transposed copy share one leading dimension, as in the block system
            nr = nc = max(nr, nc)
        outs = [torch.zeros(nr, nc, dtype=torch.complex128, device=eng.device) for _ in KS]
        scales = [1.0 + 0.25 * i for i in range(len(KS))]
        outs_t = [torch.zeros(nc, nr, dtype=torch.complex128, device=eng.device) for _ in KS] if with_t else None
        scales_t = [-0.5 - i for i in range(len(KS))] if with_t else None
        eng.assemble_batch(desc, test, trial, KS, k2s, outs, scales, outs_t, scales_t)
        for i, (k, k2) in enumerate(zip(KS, k2s)):
            ref = torch.zeros_like(outs[i])
            ref_t = torch.zeros_like(outs_t[i]) if with_t else None
            eng.assemble(Engine.op_desc(op, True, k, k2, quirk=True, precision=p), test, trial, ref, scale=scales[i],
                         out_t=ref_t, scale_t=scales_t[i] if with_t else 0.0)
            # FP64: only the order of the sums differs; mixed: both are FP32 sums
            # of the same terms, rounded in different places
            tol = 1e-12 if prec == "fp64" else 2e-6
            assert rel_err(outs[i], ref) < tol, (i, rel_err(outs[i], ref))
            if with_t:
                assert rel_err(outs_t[i], ref_t) < tol
    finally:
        eng.close()


def test_batched_block_matches_oracle():
    """One batched FP64 single-layer block against the CPU restatement."""
    from bem_b200 import _lib as L
    from bem_b200.engine import Engine
    from oracle import oracle as O
    eng, v, f = _engine(subdiv=1, Q=4)
    try:
        (sp, n), _ = _spaces(eng, f, len(v), 1, 1)
        ks = [2.0, 5.0, 9.0]
        outs = [torch.zeros(n, n, dtype=torch.complex128, device=eng.device) for _ in ks]
        eng.assemble_batch(Engine.op_desc(0, True, 0.0, 0.0, quirk=True, precision=L.PREC_FP64), sp, sp, ks,
                           [k * k for k in ks], outs, [1.0] * len(ks))
        panels = np.arange(len(f), dtype=np.int32)
        for k, o in zip(ks, outs):
            ref = np.zeros((n, n), complex)
            O.assemble(v, f, O.OP_V, True, k, k * k, 4, True, (panels, 1, panels), (panels, 1, panels), out=ref)
            assert rel_err(o, ref) < 1e-12
    finally:
        eng.close()


def test_batch_rejects_bad_arguments():
    from bem_b200 import _lib as L
    from bem_b200.engine import Engine
    eng, v, f = _engine(subdiv=1, Q=3)
    try:
        (sp, n), _ = _spaces(eng, f, len(v), 1, 1)
        out = torch.zeros(n, n, dtype=torch.complex128, device=eng.device)
        with pytest.raises(L.BemError):  # Laplace has no wavenumber to batch
            eng.assemble_batch(Engine.op_desc(0, False, 0.0, 0.0, quirk=True), sp, sp, [1.0], [1.0], [out], [1.0])
        with pytest.raises(L.BemError):
            eng.assemble_batch(Engine.op_desc(0, True, 0.0, 0.0, quirk=True), sp, sp, [float("nan")], [1.0],
                               [out], [1.0])
    finally:
        eng.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("A_type", [1, 2])
def test_batched_transmission_operators(prec, A_type):
    """The sweep's batched [A(k); P(k)] equals the per-k assembly sequence."""
    from bem_b200.managers import CoreManager
    from bem_b200.managers.sweep import transmission_operator, transmission_operators
    from bem_b200 import icosphere
    from bem_b200.workloads import plane_wave
    v, f = icosphere(2)
    params = dict(dim=3, object="icosphere2", vertices=v, panels=f, GaussQR=3, n_i=3.0, n_o=1.0, k=0.0,
                  kernel="Helmholtz_Transmission", boundary="Full", scope="Interior", show="Default", Q_Neumann=1,
                  Q_Dirichlet=1, precision=prec, log_to_disk=False, make_video=False, show_wireframe=False, vis=False)
    fD, fN = plane_wave(1.0, [0.0, 0.0, 1.0])
    core = CoreManager(params)
    core.initialization(fD, fN)
    bm = core._BEM_manager
    ks = [1.5, 2.25, 4.0]
    got = transmission_operators(bm, ks, A_type)
    tol = 1e-12 if prec == "fp64" else 2e-6
    for k, G in zip(ks, got):
        R = transmission_operator(bm, k, A_type, augmented=True)
        assert rel_err(G, R) < tol, (k, rel_err(G, R))
    core.kill()
