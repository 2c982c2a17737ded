"""Learned proposal directions for batched saddle searches.

The plain search seeds each Dimer walker with a random local displacement (the reference's
rule, SaddleSearch.cpp:390-415, with the workloads' N(0, 0.1 A)-within-4 A variant).  Here a
small MLP (akmc_mlp_*) maps per-atom descriptors (akmc_batch_descriptors) of the minimum to
three coefficients of the atom's readout vectors B_m (neighbour directions weighted by the
first three shells), whose combination is the atom's predicted displacement: the
displacement the atom had in the saddles the plain searches found where it moved most.  The
descriptors are invariant under rotation; the readout makes the prediction rotate with the
atom's surroundings (an atom of a perfect cubic environment gets zero).  A walker is seeded
along the predicted displacement of one chosen atom; walkers whose learned start does not
converge fall back to a random start.

* :func:`descriptors` -- (n_total, 64) descriptors of a set of systems;
* :func:`training_rows` -- (descriptor, target) rows from converged plain searches;
* :class:`ProposalModel` -- parameters, input standardisation, training, prediction;
* :func:`learned_seeds` -- starting displacements and modes for a walker set.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check

N_DESC = 64


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def descriptors(field, systems, pos=None, with_basis=False):
    """Descriptors of every atom of ``systems`` at ``pos`` (default: their positions):
    (n_total, 64) float32 CUDA tensor, rows in the systems' atom order; with ``with_basis``
    also the readout vectors, (n_total, 3, 3) float32 (vector, component)."""
    import torch
    b = field.batch([s.n for s in systems], np.array([s.box for s in systems]),
                    np.concatenate([s.labels for s in systems]),
                    np.concatenate([s.charge for s in systems]))
    x = np.concatenate([s.pos for s in systems]) if pos is None else pos
    p = torch.tensor(np.asarray(x, dtype=np.float64), device="cuda")
    F, E, S = b.alloc("cuda")
    b.forces_(p, F, E, S)
    d = torch.empty((b.n_total, N_DESC), dtype=torch.float32, device="cuda")
    B = torch.empty((b.n_total, 3, 3), dtype=torch.float32, device="cuda") if with_basis else None
    check(_lib.load().akmc_batch_descriptors(b._h, _ptr(d), _ptr(B) if with_basis else None, _stream()),
          "batch_descriptors")
    torch.cuda.synchronize()
    if int(S.max()) != 0:
        raise RuntimeError("force call before the descriptors reported an error")
    b.close()
    return (d, B) if with_basis else d


def _wrap(d, box):
    return d - box * np.rint(d / box)


def training_rows(desc_min, x_min, x_saddle, offsets, boxes, converged, radius=4.0, far=8,
                  rng=None):
    """Rows for the model from converged searches.  For every converged walker k (system
    rows offsets[k]:offsets[k+1]), the saddle displacement d = x_saddle - x_min is scaled to
    unit maximum; the atom that moves most and every atom within ``radius`` of it give rows
    (descriptor at the minimum, scaled displacement); ``far`` atoms farther than 2 radius
    give zero-target rows.  An atom seen in several saddles keeps the row of the saddle
    where it moved most.  Returns (desc rows (m, 64) float32, targets (m, 3) float32, row
    indices (m,) into desc_min)."""
    rng = rng or np.random.default_rng(0)
    desc_min = np.asarray(desc_min)
    best = {}
    rows_far = []
    for k in np.where(converged)[0]:
        a, b = int(offsets[k]), int(offsets[k + 1])
        box = np.asarray(boxes[k])
        d = _wrap(x_saddle[a:b] - x_min[a:b], box)
        mag = np.sqrt((d * d).sum(1))
        m = int(np.argmax(mag))
        if mag[m] <= 0:
            continue
        t = d / mag[m]
        dm = _wrap(x_min[a:b] - x_min[a + m], box)
        near = np.where(np.sqrt((dm * dm).sum(1)) < radius)[0]
        for i in near:
            key = a + int(i)
            if key not in best or mag[i] > best[key][0]:
                best[key] = (mag[i], t[i])
        farset = np.where(np.sqrt((dm * dm).sum(1)) > 2 * radius)[0]
        if len(farset):
            rows_far.extend(a + rng.choice(farset, size=min(far, len(farset)), replace=False))
    keys = np.array(sorted(best), dtype=np.int64)
    far_keys = np.array(sorted(set(rows_far) - set(best)), dtype=np.int64)
    idx = np.concatenate([keys, far_keys])
    X = desc_min[idx].astype(np.float32)
    T = np.concatenate([np.array([best[k][1] for k in keys]).reshape(-1, 3),
                        np.zeros((len(far_keys), 3))]).astype(np.float32)
    return X, T, idx


class ProposalModel:
    """The MLP's FP32 parameters and input standardisation, on the GPU."""

    def __init__(self, seed=0):
        import torch
        self.n_params = _lib.load().akmc_mlp_num_params()
        rng = np.random.default_rng(seed)
        sizes = ((64, 128), (128, 128), (128, 128), (128, 3))
        parts = []
        for fi, fo in sizes:
            parts.append(rng.normal(0.0, np.sqrt(1.0 / fi), fi * fo))
            parts.append(np.zeros(fo))
        p = np.concatenate(parts).astype(np.float32)
        assert p.size == self.n_params
        self.params = torch.tensor(p, device="cuda")
        self.norm = torch.cat([torch.zeros(N_DESC), torch.ones(N_DESC)]).cuda()
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0

    def set_norm(self, X):
        import torch
        Xt = torch.as_tensor(X, dtype=torch.float32, device="cuda")
        mean = Xt.mean(0)
        std = Xt.std(0)
        self.norm = torch.cat([mean, 1.0 / (std + 1e-3)]).contiguous()

    def loss_grad(self, X, T, lr=0.0, basis=None):
        """One step on rows (X, T) (CUDA tensors; ``basis`` (n, 3, 3) selects the readout);
        returns (loss, gradient tensor)."""
        import torch
        n = X.shape[0]
        tiles = (n + 31) // 32
        scratch = torch.empty(tiles * self.n_params, dtype=torch.float32, device="cuda")
        lpart = torch.empty(tiles, dtype=torch.float32, device="cuda")
        grad = torch.empty(self.n_params, dtype=torch.float32, device="cuda")
        if lr > 0:
            self.step += 1
        Bp = _ptr(basis) if basis is not None else None
        check(_lib.load().akmc_mlp_train_step(int(n), _ptr(X), _ptr(T), _ptr(self.norm), Bp, _ptr(self.params),
                                              _ptr(self.m), _ptr(self.v), _ptr(scratch), int(max(self.step, 1)),
                                              float(lr), _ptr(lpart), _ptr(grad), _stream()), "mlp_train_step")
        return float(lpart.sum().item()) / n, grad

    def train(self, X, T, epochs=200, batch=4096, lr=2e-3, seed=0, basis=None):
        """Adam on minibatches; returns the loss history (one value per step)."""
        import torch
        Xt = torch.as_tensor(X, dtype=torch.float32, device="cuda").contiguous()
        Tt = torch.as_tensor(T, dtype=torch.float32, device="cuda").contiguous()
        Bt = None if basis is None else torch.as_tensor(basis, dtype=torch.float32, device="cuda").contiguous()
        n = Xt.shape[0]
        g = torch.Generator(device="cpu").manual_seed(seed)
        hist = []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g).cuda()
            for s in range(0, n, batch):
                idx = perm[s:s + batch]
                loss, _ = self.loss_grad(Xt[idx].contiguous(), Tt[idx].contiguous(), lr,
                                         None if Bt is None else Bt[idx].contiguous())
                hist.append(loss)
        return hist

    def predict(self, desc, basis=None):
        """(n, 3) outputs; with ``basis`` the displacements sum_m y_m B_m."""
        import torch
        n = desc.shape[0]
        out = torch.empty((n, 3), dtype=torch.float32, device="cuda")
        Bp = _ptr(basis) if basis is not None else None
        check(_lib.load().akmc_mlp_forward(int(n), _ptr(desc), _ptr(self.norm), _ptr(self.params), Bp,
                                           _ptr(out), _stream()), "mlp_forward")
        return out


def learned_seeds(pred, x_min, offsets, boxes, radius=4.0, amplitude=0.3, noise=0.02, rng=None,
                  rank=0):
    """Starting displacements from predicted per-atom displacements.  In every walker the
    atom with the (rank+1)-th largest prediction is moved ``amplitude`` A along its
    prediction (its own hop: the model's target is the displacement an atom has in the
    saddle where it moves most), and the atoms within ``radius`` of it get N(0, noise).
    Returns (n_total, 3) float64."""
    rng = rng or np.random.default_rng(0)
    pred = np.asarray(pred, dtype=np.float64)
    out = np.zeros_like(pred)
    for k in range(len(offsets) - 1):
        a, b = int(offsets[k]), int(offsets[k + 1])
        p = pred[a:b]
        mag = np.sqrt((p * p).sum(1))
        m = int(np.argsort(-mag)[min(rank, b - a - 1)])
        box = np.asarray(boxes[k])
        dm = _wrap(x_min[a:b] - x_min[a + m], box)
        near = np.sqrt((dm * dm).sum(1)) < radius
        d = np.zeros_like(p)
        d[near] = rng.normal(0.0, noise, (int(near.sum()), 3))
        if mag[m] > 0:
            d[m] += amplitude * p[m] / mag[m]
        out[a:b] = d
    return out
