"""Learned proposal directions for batched saddle searches.

The plain search seeds each Dimer walker with a random local displacement (the reference's
rule, SaddleSearch.cpp:390-415, with the workloads' N(0, 0.1 A)-within-4 A variant).  Here two
small MLPs (akmc_mlp_*) read per-atom descriptors of the minimum (akmc_batch_descriptors):

* ``score``: how likely the atom is the one that moves most in a saddle the searches find
  (trained on 1 for the hop of each converged plain search, 0 for the atoms around it);
* ``direction``: the hop's displacement, as three coefficients of the atom's readout vectors
  B_m (neighbour directions weighted by the first three shells).  The descriptors are
  invariant under rotation; the readout makes the prediction rotate with the atom's
  surroundings (an atom with a centrosymmetric environment gets zero).

akmc_proposal_seeds then draws one candidate atom per walker among the best-scored ones and
moves it along its predicted displacement, with a little noise on its neighbourhood; walkers
without a candidate, and walkers whose learned start does not converge, fall back to a
random start.

* :func:`descriptors` -- (n_total, 64) descriptors of a set of systems;
* :func:`hop_rows` -- training rows from converged plain searches;
* :class:`ProposalModel` -- one MLP: parameters, input standardisation, training, prediction;
* :class:`Proposer` -- the two models and the device pipeline descriptors -> seeds;
* :func:`seeds` -- akmc_proposal_seeds.
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


def _take(a, idx):
    """Rows idx of a numpy array, or of a CUDA tensor (gathered on the device; only those rows
    come back)."""
    idx = np.asarray(idx, dtype=np.int64)
    if hasattr(a, "index_select"):
        import torch
        return a[torch.as_tensor(idx, device=a.device)].cpu().numpy()
    return np.asarray(a)[idx]


def hop_rows(desc, basis, x_min, x_saddle, offsets, boxes, usable, radius=4.0, far=8, rng=None):
    """Training rows from the saddles of walkers marked ``usable`` (walker k: atoms
    offsets[k]:offsets[k+1]; desc (n, 64) and basis (n, 3, 3) at the minimum x_min, numpy
    arrays or CUDA tensors).  In each saddle the atom that moves most (the hop) gives a
    direction row: its descriptor, its readout vectors and its displacement x_saddle - x_min
    (A).  Score rows: the hop (target 1) and every other atom within ``radius`` of it plus
    ``far`` random atoms of the walker (target 0); the score is the first model output.
    Returns dict(direction=(X, T, B), score=(X, T)), float32 arrays."""
    hops, TD, srows, TS = hop_picks(x_min, x_saddle, offsets, boxes, usable, radius, far, rng)
    f = lambda v, shape: np.asarray(v, np.float32).reshape(shape)  # noqa: E731
    XD = _take(desc, hops) if len(hops) else np.zeros((0, 64))
    BD = _take(basis, hops) if len(hops) else np.zeros((0, 3, 3))
    XS = _take(desc, srows) if len(srows) else np.zeros((0, 64))
    return dict(direction=(f(XD, (-1, 64)), TD, f(BD, (-1, 3, 3))), score=(f(XS, (-1, 64)), TS))


def hop_picks(x_min, x_saddle, offsets, boxes, usable, radius=4.0, far=8, rng=None):
    """The atoms :func:`hop_rows` takes its rows from, without the descriptors: (hops, TD,
    srows, TS) -- the hop of every usable walker (int64 atom numbers) with its displacement
    (float32 (n, 3)), then the score rows' atom numbers with their targets (float32 (m, 3)),
    walker by walker in the same order, so a caller can compute the descriptors of exactly
    these atoms."""
    rng = rng or np.random.default_rng(0)
    hops, TD, srows, TS = [], [], [], []
    for k in np.where(usable)[0]:
        a, b = int(offsets[k]), int(offsets[k + 1])
        box = np.asarray(boxes[k])
        d = _wrap(x_saddle[a:b] - x_min[a:b], box)
        mag = np.sqrt((d * d).sum(1))
        m = int(np.argmax(mag))
        if mag[m] <= 0:
            continue
        hops.append(a + m)
        TD.append(d[m])
        dm = _wrap(x_min[a:b] - x_min[a + m], box)
        near = np.where(np.sqrt((dm * dm).sum(1)) < radius)[0]
        pick = rng.choice(b - a, size=min(far, b - a), replace=False)
        idx = np.concatenate([near, pick])
        srows.append(a + idx)
        t = np.zeros((len(idx), 3), np.float32)
        t[idx == m, 0] = 1.0
        TS.append(t)
    srows = np.concatenate(srows).astype(np.int64) if srows else np.zeros(0, np.int64)
    TS = np.concatenate(TS) if TS else np.zeros((0, 3), np.float32)
    return np.asarray(hops, np.int64), np.asarray(TD, np.float32).reshape(-1, 3), srows, TS


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

    def loss_grad(self, X, T, lr=0.0, basis=None, fp32pipe=False):
        """One step on rows (X, T) (CUDA tensors; ``basis`` (n, 3, 3) selects the readout) by
        akmc_mlp_train_step (tensor cores), or its FP32-pipe cross-check; returns (loss,
        gradient tensor)."""
        import torch
        n = X.shape[0]
        tiles = (n + (31 if fp32pipe else 127)) // (32 if fp32pipe else 128)
        scratch = torch.empty(tiles * self.n_params, dtype=torch.float32, device="cuda")
        lpart = torch.empty(tiles, dtype=torch.float32, device="cuda")
        grad = torch.empty(self.n_params, dtype=torch.float32, device="cuda")
        if lr > 0:
            self.step += 1
        Bp = _ptr(basis) if basis is not None else None
        fn = _lib.load().akmc_mlp_train_step_fp32pipe if fp32pipe else _lib.load().akmc_mlp_train_step
        check(fn(int(n), _ptr(X), _ptr(T), _ptr(self.norm), Bp, _ptr(self.params), _ptr(self.m), _ptr(self.v),
                 _ptr(scratch), int(max(self.step, 1)), float(lr), _ptr(lpart), _ptr(grad), _stream()),
              "mlp_train_step")
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


def proposal_params(**kw):
    """akmc_proposal_params with the defaults of the metal workloads: candidates within half
    of the walker's best score, no proposal below score 0.02 (the score estimates the chance
    that the atom is the one that hops; the twelve neighbours of a vacancy share it, about
    1/12 each), the chosen atom moved by its predicted saddle displacement, N(0, 0.02 A) on the
    atoms within 4 A of it; atoms whose predicted displacement is shorter than 0.3 A (a hop
    is about 1.2 A; an atom between two vacancies gets opposite readout vectors that cancel)
    are not candidates."""
    p = _lib.ProposalParams(threshold=0.5, min_score=0.02, scale=1.0, noise=0.02, radius=4.0, min_disp=0.3,
                            region=0.0, group=0)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def seeds(begin, pos, box, pred, score, params=None, seed=0, counter=0, score_stride=3, stream=None,
          center=None):
    """akmc_proposal_seeds: (disp, mode, chosen) CUDA tensors for walkers whose atoms are
    rows begin[w]:begin[w+1] (CUDA int64 tensor) of pos (float64 (n, 3)); box float64
    (W, 3); pred float32 (n, 3); score float32 read with ``score_stride``; center (optional,
    float64 (W, 3)) with params.region > 0 limits each walker's candidates to its region."""
    import torch
    W = int(begin.numel()) - 1
    disp = torch.empty_like(pos)
    mode = torch.empty_like(pos)
    chosen = torch.empty(W, dtype=torch.int32, device=pos.device)
    p = params or proposal_params()
    check(_lib.load().akmc_proposal_seeds(W, _ptr(begin), _ptr(pos), _ptr(box),
                                          _ptr(center) if center is not None else None, _ptr(pred), _ptr(score),
                                          int(score_stride), C.byref(p), C.c_uint64(seed), C.c_uint64(counter),
                                          _ptr(disp), _ptr(mode), _ptr(chosen),
                                          C.c_void_p(stream if stream is not None else _stream().value)),
          "proposal_seeds")
    return disp, mode, chosen


def region_rows(begin, pos, box, center, radius):
    """Atom numbers (CUDA int32) of the atoms within ``radius`` of their walker's centre
    (minimum image): walker w holds rows begin[w]:begin[w+1] of pos, box[w] its cell."""
    import torch
    counts = begin[1:] - begin[:-1]
    wid = torch.repeat_interleave(torch.arange(counts.numel(), device=pos.device), counts)
    d = pos - center[wid]
    b = box[wid]
    d = d - b * torch.round(d / b)
    return torch.nonzero((d * d).sum(1) <= radius * radius).squeeze(1).to(torch.int32)


class Proposer:
    """The two models of the learned proposal: ``direction`` (readout on: the hop's
    displacement) and ``score`` (first output: how likely the atom is the one that hops)."""

    def __init__(self, seed=0):
        self.direction = ProposalModel(seed)
        self.score = ProposalModel(seed + 1)

    def fit(self, rows, dir_epochs=200, score_epochs=40, lr=2e-3, seed=0):
        XD, TD, BD = rows["direction"]
        XS, TS = rows["score"]
        if len(XD) == 0 or len(XS) == 0:
            raise ValueError("no training rows")
        self.direction.set_norm(XS)
        self.score.set_norm(XS)
        h1 = self.direction.train(XD, TD, epochs=dir_epochs, batch=1024, lr=lr, seed=seed, basis=BD)
        h2 = self.score.train(XS, TS, epochs=score_epochs, batch=4096, lr=lr, seed=seed)
        return h1, h2

    def predict(self, desc, basis):
        """(displacement (n, 3), score outputs (n, 3)) float32 CUDA tensors."""
        return self.direction.predict(desc, basis), self.score.predict(desc)

    def propose(self, walkers, x_min, params=None, seed=0, counter=0, fallback=None, center=None):
        """Starting displacements and modes for ``walkers`` (a :class:`Walkers`) from their
        minima x_min (CUDA float64 (n_total, 3)): (disp, mode, chosen), all on the device.
        Walkers without a proposal (chosen -1) take their rows of ``fallback`` (random
        starting displacements, CUDA float64 (n_total, 3)) as displacement and mode.  With
        ``center`` (CUDA float64 (W, 3)) and params.region > 0 the candidates are the atoms
        within params.region of their walker's centre, and only they get descriptors and
        predictions."""
        import torch
        begin, box = walkers.device_geometry()
        if center is not None and params is not None and params.region > 0:
            rows = region_rows(begin, x_min, box, center, params.region + 0.5)
            desc, basis = walkers.descriptors(x_min, with_basis=True, rows=rows)
            p_r, s_r = self.predict(desc, basis)
            n = x_min.shape[0]
            pred = torch.zeros((n, 3), dtype=torch.float32, device=x_min.device)
            score = torch.zeros((n, 3), dtype=torch.float32, device=x_min.device)
            pred[rows.long()] = p_r
            score[rows.long()] = s_r
        else:
            desc, basis = walkers.descriptors(x_min, with_basis=True)
            pred, score = self.predict(desc, basis)
        disp, mode, chosen = seeds(begin, x_min, box, pred, score, params, seed, counter, center=center)
        if fallback is not None:
            rows = (chosen < 0).repeat_interleave(begin[1:] - begin[:-1])[:, None]
            disp = torch.where(rows, fallback, disp)
            mode = torch.where(rows, fallback, mode)
        return disp, mode, chosen
