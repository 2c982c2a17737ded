"""Descriptors and the proposal MLP on the GPU against the numpy restatement
(oracle/mlp.py): descriptors to FP32 accuracy, the BF16 forward pass and its training
gradient to the rounding of BF16 activations, and training that learns."""
import numpy as np
import pytest

from akmc_b200 import configs as cf
from akmc_b200.field import Field
from oracle import mlp as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eam_field(potdir):
    s = cf.fcc_vacancy_system(4)
    return Field().readPotential(str(potdir / "eam.pot")).setup(s.lat, None, 4000)


def test_descriptors_match_oracle(gpu, eam_field):
    from akmc_b200 import proposals as P
    systems = [cf.fcc_vacancy_system(4, seed=3), cf.fcc_vacancy_system(5, n_vacancies=2, seed=4)]
    d = P.descriptors(eam_field, systems).cpu().numpy()
    off = np.concatenate([[0], np.cumsum([s.n for s in systems])])
    for k, s in enumerate(systems):
        ref = M.descriptors(s.pos, s.box)
        got = d[off[k]:off[k + 1]]
        assert np.allclose(got, ref, rtol=2e-4, atol=2e-5), np.abs(got - ref).max()


def test_readout_basis_matches_oracle(gpu, eam_field):
    from akmc_b200 import proposals as P
    systems = [cf.fcc_vacancy_system(4, seed=5), cf.fcc_vacancy_system(5, n_vacancies=2, seed=6)]
    d, B = P.descriptors(eam_field, systems, with_basis=True)
    d2 = P.descriptors(eam_field, systems)
    assert np.array_equal(d.cpu().numpy(), d2.cpu().numpy())
    B = B.cpu().numpy()
    off = np.concatenate([[0], np.cumsum([s.n for s in systems])])
    for k, s in enumerate(systems):
        ref = M.basis(s.pos, s.box)
        got = B[off[k]:off[k + 1]]
        assert np.abs(got - ref).max() < 2e-5, np.abs(got - ref).max()
        # the readout vanishes on atoms whose environment has inversion symmetry and
        # not on the vacancy's neighbours
        assert np.abs(ref).max() > 0.1


def test_readout_forward_and_gradient_match_oracle(gpu):
    import torch
    from akmc_b200 import proposals as P
    rng = np.random.default_rng(5)
    n = 150
    X = rng.normal(1.0, 2.0, (n, 64)).astype(np.float32)
    B = rng.normal(0.0, 0.5, (n, 3, 3)).astype(np.float32)
    T = rng.normal(0.0, 0.3, (n, 3)).astype(np.float32)
    model = P.ProposalModel(seed=4)
    model.set_norm(X)
    norm = model.norm.cpu().numpy()
    p = model.params.cpu().numpy()
    Bt = torch.tensor(B, device=gpu)
    y = model.predict(torch.tensor(X, device=gpu), Bt).cpu().numpy()
    y_ref = M.readout(M.forward(X, (norm[:64], norm[64:]), p), B)
    assert np.abs(y - y_ref).max() < 2e-2
    assert np.abs(y - y_ref).mean() < 1e-3
    loss, g = model.loss_grad(torch.tensor(X, device=gpu), torch.tensor(T, device=gpu), lr=0.0, basis=Bt)
    loss_ref, g_ref = M.loss_and_grad(X, T, (norm[:64], norm[64:]), p, B=B)
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    g = g.cpu().numpy()
    assert np.linalg.norm(g - g_ref) <= 2e-2 * np.linalg.norm(g_ref)


def test_forward_and_gradient_match_oracle(gpu):
    import torch
    from akmc_b200 import proposals as P
    rng = np.random.default_rng(0)
    n = 200
    X = rng.normal(1.0, 2.0, (n, 64)).astype(np.float32)
    T = rng.normal(0.0, 0.3, (n, 3)).astype(np.float32)
    model = P.ProposalModel(seed=3)
    model.set_norm(X)
    norm = model.norm.cpu().numpy()
    p = model.params.cpu().numpy()
    y = model.predict(torch.tensor(X, device=gpu)).cpu().numpy()
    y_ref = M.forward(X, (norm[:64], norm[64:]), p)
    # BF16 activations: a rare one-ulp flip of a hidden value moves an output by ~1e-3
    assert np.abs(y - y_ref).max() < 2e-2
    assert np.abs(y - y_ref).mean() < 1e-3
    loss, g = model.loss_grad(torch.tensor(X, device=gpu), torch.tensor(T, device=gpu), lr=0.0)
    loss_ref, g_ref = M.loss_and_grad(X, T, (norm[:64], norm[64:]), p)
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    g = g.cpu().numpy()
    assert np.linalg.norm(g - g_ref) <= 2e-2 * np.linalg.norm(g_ref)


def test_training_learns(gpu):
    from akmc_b200 import proposals as P
    rng = np.random.default_rng(1)
    X = rng.normal(0.0, 1.0, (6000, 64)).astype(np.float32)
    A = rng.normal(0.0, 0.3, (64, 3)).astype(np.float32)
    T = np.tanh(X @ A).astype(np.float32)
    model = P.ProposalModel(seed=2)
    model.set_norm(X)
    hist = model.train(X, T, epochs=30, batch=2048, lr=3e-3)
    assert hist[-1] < 0.2 * hist[0]


@pytest.mark.parametrize("n,with_basis", [(1000, False), (4099, True), (127, True)])
def test_tensor_core_forward_matches_fp32_pipe(gpu, n, with_basis):
    """akmc_mlp_forward (tcgen05, FP32 accumulation in tensor memory) against the same
    network on the FP32 pipe and against the numpy restatement: equal up to BF16 flips of
    hidden activations, ragged last tile included."""
    import ctypes as C
    import torch
    from akmc_b200 import _lib
    from akmc_b200 import proposals as P
    rng = np.random.default_rng(n)
    X = rng.normal(0.5, 1.5, (n, 64)).astype(np.float32)
    model = P.ProposalModel(seed=7)
    model.set_norm(X)
    Xt = torch.tensor(X, device=gpu)
    B = rng.normal(0.0, 0.5, (n, 3, 3)).astype(np.float32) if with_basis else None
    Bt = torch.tensor(B, device=gpu) if with_basis else None
    y_tc = model.predict(Xt, Bt).cpu().numpy()
    out = torch.empty((n, 3), dtype=torch.float32, device=gpu)
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    lib = _lib.load()
    assert lib.akmc_mlp_forward_fp32pipe(n, ptr(Xt), ptr(model.norm), ptr(model.params), ptr(Bt), ptr(out),
                                         C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    torch.cuda.synchronize()
    assert lib.akmc_mlp_check() == 0
    y_fp = out.cpu().numpy()
    assert np.isfinite(y_tc).all()
    assert np.abs(y_tc - y_fp).max() < 2e-2
    assert np.abs(y_tc - y_fp).mean() < 1e-3
    norm = model.norm.cpu().numpy()
    y_ref = M.forward(X, (norm[:64], norm[64:]), model.params.cpu().numpy())
    if with_basis:
        y_ref = M.readout(y_ref, B)
    assert np.abs(y_tc - y_ref).mean() < 1e-3


@pytest.mark.parametrize("n,with_basis", [(300, False), (257, True)])
def test_tensor_core_gradient_matches_oracle(gpu, n, with_basis):
    """akmc_mlp_train_step (tcgen05 forward and backward) against the numpy restatement with
    the hidden-layer errors rounded to BF16 as the tensor core takes them, and against the
    FP32-pipe training step; ragged last tile included."""
    import torch
    from akmc_b200 import proposals as P
    rng = np.random.default_rng(n)
    X = rng.normal(1.0, 2.0, (n, 64)).astype(np.float32)
    T = rng.normal(0.0, 0.3, (n, 3)).astype(np.float32)
    B = rng.normal(0.0, 0.5, (n, 3, 3)).astype(np.float32) if with_basis else None
    model = P.ProposalModel(seed=5)
    model.set_norm(X)
    norm = model.norm.cpu().numpy()
    p = model.params.cpu().numpy()
    Xt, Tt = torch.tensor(X, device=gpu), torch.tensor(T, device=gpu)
    Bt = torch.tensor(B, device=gpu) if with_basis else None
    loss, g = model.loss_grad(Xt, Tt, lr=0.0, basis=Bt)
    loss_fp, g_fp = model.loss_grad(Xt, Tt, lr=0.0, basis=Bt, fp32pipe=True)
    from akmc_b200 import _lib
    assert _lib.load().akmc_mlp_check() == 0
    g, g_fp = g.cpu().numpy(), g_fp.cpu().numpy()
    loss_ref, g_ref = M.loss_and_grad(X, T, (norm[:64], norm[64:]), p, B=B, rnd_grad=M.bf16)
    assert np.isfinite(g).all()
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    assert np.linalg.norm(g - g_ref) <= 1e-2 * np.linalg.norm(g_ref)
    assert np.linalg.norm(g - g_fp) <= 2e-2 * np.linalg.norm(g_fp)
    # every block of the parameter vector is right, not only the large ones
    off = 0
    for fi, fo in M.SIZES:
        for size in (fi * fo, fo):
            a, r = g[off:off + size], g_ref[off:off + size]
            assert np.linalg.norm(a - r) <= 2e-2 * np.linalg.norm(r) + 1e-7, (off, size)
            off += size
