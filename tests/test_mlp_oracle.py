"""The numpy restatement of the proposal model (oracle/mlp.py) on its own: the analytic
gradient against central differences (rounding switched off), and the symmetry of the
descriptors and of the readout vectors."""
import numpy as np

from akmc_b200 import configs as cf
from oracle import mlp as M


def _fd_check(B):
    rng = np.random.default_rng(0)
    n = 12
    X = rng.normal(0.0, 1.0, (n, 64)).astype(np.float32)
    T = rng.normal(0.0, 0.3, (n, 3)).astype(np.float32)
    p = M.init_params(1).astype(np.float64)
    norm = (np.zeros(64, np.float32), np.ones(64, np.float32))
    ident = lambda a: np.asarray(a, dtype=np.float64)  # noqa: E731
    _, g = M.loss_and_grad(X, T, norm, p, rnd=ident, B=B)
    for k in rng.choice(p.size, 40, replace=False):
        e = np.zeros_like(p)
        e[k] = 1e-4
        lp, _ = M.loss_and_grad(X, T, norm, p + e, rnd=ident, B=B)
        lm, _ = M.loss_and_grad(X, T, norm, p - e, rnd=ident, B=B)
        fd = (lp - lm) / 2e-4
        assert abs(fd - g[k]) <= 2e-3 * max(1e-3, abs(fd)) + 1e-5, (k, fd, g[k])


def test_gradient_matches_central_differences():
    _fd_check(None)


def test_readout_gradient_matches_central_differences():
    B = np.random.default_rng(3).normal(0.0, 0.5, (12, 3, 3))
    _fd_check(B)


def test_readout_vanishes_in_perfect_crystal_and_rotates():
    s = cf.fcc_vacancy_system(3, n_vacancies=0, sigma=0.0, seed=1)
    B = M.basis(s.pos, s.box)
    assert np.abs(B).max() < 1e-9
    v = cf.fcc_vacancy_system(3, n_vacancies=1, seed=1)
    Bv = M.basis(v.pos, v.box)
    assert np.abs(Bv).max() > 0.1
    # a cubic rotation (x, y, z) -> (y, z, x) of the crystal permutes the components and
    # leaves the descriptors unchanged
    pr = v.pos[:, [1, 2, 0]]
    br = v.box[[1, 2, 0]]
    Br = M.basis(pr, br)
    assert np.allclose(Br, Bv[:, :, [1, 2, 0]], atol=1e-12)
    d0 = M.descriptors(v.pos, v.box)[:20]
    d1 = M.descriptors(pr, br)[:20]
    assert np.allclose(d0, d1, atol=1e-9)


def test_proposal_seeds_rules():
    rng = np.random.default_rng(2)
    n = 50
    begin = np.array([0, n])
    pos = rng.uniform(0.0, 12.0, (n, 3))
    box = np.full((1, 3), 12.0)
    pred = rng.normal(0.0, 1.0, (n, 3)).astype(np.float32)
    score = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
    kw = dict(min_score=0.2, scale=0.8, noise=0.05, radius=4.0, seed=3, counter=0)
    d, m, c = M.proposal_seeds(begin, pos, box, pred, score, threshold=1.0, **kw)
    best = int(np.argmax(score[:, 0]))
    assert c[0] == best
    assert np.array_equal(m[best], pred[best].astype(np.float64))
    assert np.count_nonzero(np.abs(m).sum(1)) == 1
    dd = pos - pos[best]
    dd -= 12.0 * np.rint(dd / 12.0)
    far = np.sqrt((dd * dd).sum(1)) >= 4.0
    assert np.all(d[far] == 0.0) and np.all(np.abs(d[~far]).sum(1) > 0)
    # the same key and counter give the same seeds; another counter, other noise
    d2, _, _ = M.proposal_seeds(begin, pos, box, pred, score, threshold=1.0, **kw)
    assert np.array_equal(d, d2)
    kw3 = dict(kw, counter=1)
    d3, _, _ = M.proposal_seeds(begin, pos, box, pred, score, threshold=1.0, **kw3)
    assert not np.array_equal(d, d3)
    # below min_score: no proposal
    _, _, c4 = M.proposal_seeds(begin, pos, box, pred, score * 0.1, threshold=0.5, **kw)
    assert c4[0] == -1


def _two_walkers():
    """Two FCC 3^3 vacancy walkers (107 atoms each) at a minimum and at a 'saddle' where one
    nearest neighbour of the vacancy has moved half way into it and the rest are jittered."""
    rng = np.random.default_rng(8)
    out_min, out_sad, hops = [], [], []
    for k in range(2):
        s = cf.fcc_vacancy_system(3, 3.615, 1, 0.0, 3 + k, vacancy_sites=[0])
        vac = np.zeros(3)
        d = s.pos - vac
        d -= s.box * np.rint(d / s.box)
        j = int(np.argsort((d * d).sum(1))[k])           # a nearest neighbour of the vacancy
        sad = s.pos + rng.normal(0.0, 0.01, s.pos.shape)
        sad[j] -= 0.5 * d[j]
        out_min.append(s.pos)
        out_sad.append(sad)
        hops.append(j)
    return np.concatenate(out_min), np.concatenate(out_sad), hops, s.box


def test_hop_picks_rows_and_targets():
    """The training-row picker of the learned proposal: the hop of each usable walker is its
    most displaced atom, with its minimum-image displacement as the direction target; the
    score rows are the atoms within the radius of the hop (the hop itself the only target 1)
    and `far` others of the walker; walkers not marked usable give no rows."""
    from akmc_b200 import proposals as P
    xm, xs, hops, box = _two_walkers()
    offs = np.array([0, 107, 214])
    H, TD, rows, TS = P.hop_picks(xm, xs, offs, [box, box], np.array([True, True]),
                                  radius=4.0, far=8, rng=np.random.default_rng(1))
    assert list(H) == [hops[0], 107 + hops[1]]
    for k in range(2):
        d = xs[H[k]] - xm[H[k]]
        assert np.allclose(TD[k], d - box * np.rint(d / box), atol=1e-6)
    assert TS.shape == (len(rows), 3) and np.all(TS[:, 1:] == 0)
    assert sorted(rows[TS[:, 0] == 1].tolist()) == sorted(H.tolist())
    for k in range(2):
        a, b = offs[k], offs[k + 1]
        mine = rows[(rows >= a) & (rows < b)]
        dm = xm[a:b] - xm[H[k]]
        dm -= box * np.rint(dm / box)
        near = a + np.where(np.sqrt((dm * dm).sum(1)) < 4.0)[0]
        assert set(near) <= set(mine.tolist()) and len(mine) == len(near) + 8
    H2, _, rows2, _ = P.hop_picks(xm, xs, offs, [box, box], np.array([False, True]), rng=np.random.default_rng(1))
    assert list(H2) == [107 + hops[1]] and (rows2 >= 107).all()


def test_hop_rows_gathers_the_picked_rows():
    """hop_rows = hop_picks plus the descriptors of the picked atoms, in the same order."""
    from akmc_b200 import proposals as P
    xm, xs, _, box = _two_walkers()
    offs = np.array([0, 107, 214])
    rng = np.random.default_rng(2)
    desc = rng.normal(size=(214, 64)).astype(np.float32)
    basis = rng.normal(size=(214, 3, 3)).astype(np.float32)
    u = np.array([True, True])
    H, TD, rows, TS = P.hop_picks(xm, xs, offs, [box, box], u, rng=np.random.default_rng(4))
    r = P.hop_rows(desc, basis, xm, xs, offs, [box, box], u, rng=np.random.default_rng(4))
    XD, TD2, BD = r["direction"]
    XS, TS2 = r["score"]
    assert np.array_equal(XD, desc[H]) and np.array_equal(BD, basis[H]) and np.array_equal(TD2, TD)
    assert np.array_equal(XS, desc[rows]) and np.array_equal(TS2, TS)
