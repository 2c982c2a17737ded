"""The learned-proposal pipeline on the GPU: the seeding kernel (akmc_proposal_seeds)
against its numpy restatement, Dimer runs of a walker subset, descriptors from a walker
set's own batch, and the trained proposal on vacancy hops."""
import numpy as np
import pytest

from akmc_b200 import configs as cf
from akmc_b200.field import Field
from akmc_b200.walkers import CONVERGED, SKIPPED, Walkers, dimer_params, fire_params
from oracle import mlp as M

pytestmark = pytest.mark.gpu


def _field(potdir, lat, n):
    return Field().readPotential(str(potdir / "eam.pot")).setup(lat, None, n)


@pytest.mark.parametrize("case", ["default", "all_candidates", "best_only", "no_noise", "min_disp", "region",
                                  "group"])
def test_seeds_match_oracle(gpu, case):
    import torch
    from akmc_b200 import proposals as P
    rng = np.random.default_rng(11)
    sizes = [37, 0, 300, 5, 1200, 64]
    begin = np.concatenate([[0], np.cumsum(sizes)])
    n = int(begin[-1])
    box = rng.uniform(9.0, 20.0, (len(sizes), 3))
    pos = np.concatenate([rng.uniform(0.0, 1.0, (k, 3)) * box[w] for w, k in enumerate(sizes)])
    pred = rng.normal(0.0, 1.0, (n, 3)).astype(np.float32)
    score = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
    score[begin[5]:begin[6], 0] *= 0.1                      # walker 5: below min_score
    kw = dict(threshold=0.5, min_score=0.2, scale=0.8, noise=0.02, radius=4.0, min_disp=0.0)
    if case == "all_candidates":
        kw.update(threshold=0.0)
    elif case == "best_only":
        kw.update(threshold=1.0)
    elif case == "no_noise":
        kw.update(noise=0.0)
    elif case == "min_disp":
        kw.update(min_disp=1.5)                              # about half the atoms ineligible
    if case == "group":
        kw.update(group=3)                                   # walkers 0-2 and 3-5 stratified
    center = None
    if case == "region":
        kw.update(region=4.0)
        center = pos[begin[:-1].clip(max=n - 1)] + 0.5       # a centre near each walker's first atom
    d, m, c = P.seeds(torch.tensor(begin, device=gpu), torch.tensor(pos, device=gpu),
                      torch.tensor(box, device=gpu), torch.tensor(pred, device=gpu),
                      torch.tensor(score, device=gpu), P.proposal_params(**kw), seed=123, counter=9,
                      center=None if center is None else torch.tensor(center, device=gpu))
    dr, mr, cr = M.proposal_seeds(begin, pos, box, pred, score, seed=123, counter=9, center=center, **kw)
    assert np.array_equal(c.cpu().numpy(), cr)
    if case == "group":
        # a group of walkers on one system draws from different slices of its candidates
        Wg = 6
        bg = np.arange(0, (Wg + 1) * 400, 400)
        pg = np.tile(pos[begin[4]:begin[4] + 400], (Wg, 1))
        qg = np.tile(pred[begin[4]:begin[4] + 400], (Wg, 1))
        sg = np.tile(score[begin[4]:begin[4] + 400], (Wg, 1))
        xg = np.tile(box[4], (Wg, 1))
        _, _, cg = P.seeds(torch.tensor(bg, device=gpu), torch.tensor(pg, device=gpu), torch.tensor(xg, device=gpu),
                           torch.tensor(qg, device=gpu), torch.tensor(sg, device=gpu), P.proposal_params(**kw),
                           seed=123, counter=9)
        _, _, cgr = M.proposal_seeds(bg, pg, xg, qg, sg, seed=123, counter=9, **kw)
        assert np.array_equal(cg.cpu().numpy(), cgr)
        assert len(set(cgr[:3].tolist())) == 3 and len(set(cgr[3:].tolist())) == 3
    assert cr[1] == -1 and cr[5] == -1 and (cr[[0, 2, 3, 4]] >= 0).all() or case == "region"
    if case == "region":
        for w in range(len(sizes)):
            if cr[w] >= 0:
                dc = pos[begin[w] + cr[w]] - center[w]
                dc -= box[w] * np.rint(dc / box[w])
                assert np.linalg.norm(dc) < 4.0
    assert np.array_equal(m.cpu().numpy(), mr)
    assert np.abs(d.cpu().numpy() - dr).max() < 1e-14
    if case == "min_disp":
        for w in (0, 2, 3, 4):
            assert np.linalg.norm(pred[begin[w] + cr[w]]) >= 1.5
    if case == "best_only":
        for w in (0, 2, 3, 4):
            sc = score[begin[w]:begin[w + 1], 0]
            assert cr[w] == int(np.argmax(sc))


def test_seeds_differ_per_walker_and_counter(gpu):
    import torch
    from akmc_b200 import proposals as P
    n, W = 100, 64
    begin = torch.arange(0, (W + 1) * n, n, dtype=torch.int64, device=gpu)
    pos = torch.rand((W * n, 3), dtype=torch.float64, device=gpu) * 12.0
    box = torch.full((W, 3), 12.0, dtype=torch.float64, device=gpu)
    pred = torch.randn((W * n, 3), device=gpu)
    score = torch.ones((W * n, 3), device=gpu)               # every atom a candidate
    _, _, c0 = P.seeds(begin, pos, box, pred, score, seed=5, counter=0)
    _, _, c1 = P.seeds(begin, pos, box, pred, score, seed=5, counter=1)
    c0, c1 = c0.cpu().numpy(), c1.cpu().numpy()
    assert len(set(c0.tolist())) > 30                        # replicas get different atoms
    assert (c0 != c1).mean() > 0.8


@pytest.fixture(scope="module")
def hop_set(potdir):
    """Eight jittered 4^3 vacancy systems, FIRE-relaxed on the GPU, with plain seeds."""
    import torch
    systems = [cf.fcc_vacancy_system(4, seed=40 + k, vacancy_sites=[int(k * 29 % 256)]) for k in range(8)]
    f = _field(potdir, systems[0].lat, systems[0].n)
    w = Walkers.from_systems(f, systems)
    x = torch.tensor(np.concatenate([s.pos for s in systems]), device="cuda")
    r = w.relax(x, fire_params(force_tol=1e-4))
    assert (r["status"] == CONVERGED).all()
    xm = x.cpu().numpy()
    sd = np.concatenate([cf.local_displacements(xm[w.offsets[k]:w.offsets[k + 1]], s.box,
                                                cf.fcc_sites(4, 3.615)[s.meta["vacancies"][0]], 1,
                                                seed=300 + k)[0] for k, s in enumerate(systems)])
    return f, systems, w, xm, r["energy"].copy(), sd


def test_dimer_subset(gpu, hop_set):
    import torch
    _, _, w, xm, _, sd = hop_set
    p = dimer_params(delta=0.005, rot_tol=0.1, max_iter=200)
    x_all = torch.tensor(xm + sd, device=gpu)
    m_all = torch.tensor(sd, device=gpu)
    full = w.dimer(x_all, m_all, p)
    mask = np.array([1, 0, 1, 0, 0, 1, 1, 0], dtype=np.int32)
    x_sub = torch.tensor(xm + sd, device=gpu)
    m_sub = torch.tensor(sd, device=gpu)
    sub = w.dimer_subset(x_sub, m_sub, torch.tensor(mask, device=gpu), p)
    xa, xs = x_all.cpu().numpy(), x_sub.cpu().numpy()
    for k in range(w.W):
        a, b = w.offsets[k], w.offsets[k + 1]
        if mask[k]:
            assert sub["status"][k] == full["status"][k]
            assert sub["iters"][k] == full["iters"][k]
            assert sub["energy"][k] == full["energy"][k]
            assert np.array_equal(xs[a:b], xa[a:b])
        else:
            assert sub["status"][k] == SKIPPED
            assert np.array_equal(xs[a:b], (xm + sd)[a:b])
            assert np.array_equal(m_sub.cpu().numpy()[a:b], sd[a:b])


def test_walker_descriptors_match_batch(gpu, hop_set):
    import torch
    from akmc_b200 import proposals as P
    f, systems, w, xm, _, _ = hop_set
    d, B = w.descriptors(torch.tensor(xm, device=gpu), with_basis=True)
    d2, B2 = P.descriptors(f, systems, xm, with_basis=True)
    assert np.allclose(d.cpu().numpy(), d2.cpu().numpy(), rtol=1e-5, atol=1e-6)
    assert np.allclose(B.cpu().numpy(), B2.cpu().numpy(), rtol=1e-5, atol=1e-6)


def test_descriptor_rows_match_every_atom(gpu, hop_set):
    """Descriptors of listed atoms only (a proposal's candidates) equal those rows of the
    every-atom call bit for bit; the rows are the atoms within 4.5 A of each vacancy site, in
    the order region_rows lists them, plus one row past the end (zeros)."""
    import torch
    from akmc_b200 import proposals as P
    _, systems, w, xm, _, _ = hop_set
    x = torch.tensor(xm, device=gpu)
    d, B = w.descriptors(x, with_basis=True)
    begin, box = w.device_geometry()
    centre = torch.tensor(np.array([cf.fcc_sites(4, 3.615)[s.meta["vacancies"][0]] for s in systems]), device=gpu)
    rows = P.region_rows(begin, x, box, centre, 4.5)
    assert 8 * 12 <= rows.numel() < w.n_total // 4
    rows = torch.cat([rows, torch.tensor([w.n_total], dtype=torch.int32, device=gpu)])
    dr, Br = w.descriptors(x, with_basis=True, rows=rows)
    r = rows[:-1].long()
    assert torch.equal(dr[:-1], d[r]) and torch.equal(Br[:-1], B[r])
    assert not dr[-1].any() and not Br[-1].any()


def test_learned_proposals_find_vacancy_hops(gpu, potdir, hop_set):
    """Train on plain searches of 4^3 and 6^3 systems, propose on other systems: the chosen
    atoms are nearest neighbours of a vacancy, the displacement points at it, and the
    searches converge to the vacancy hop."""
    import torch
    from akmc_b200 import proposals as P
    big = cf.fcc_vacancy_system(6)
    f = _field(potdir, big.lat, big.n)
    p = dimer_params(delta=0.005, rot_tol=0.1, max_iter=200)

    def make(seed, nsys):
        rng = np.random.default_rng(seed)
        systems = [cf.fcc_vacancy_system(int(rng.choice([4, 6])), n_vacancies=1, seed=int(rng.integers(1 << 30)),
                                         vacancy_sites=[int(rng.integers(256))]) for _ in range(nsys)]
        w = Walkers.from_systems(f, systems)
        x = torch.tensor(np.concatenate([s.pos for s in systems]), device=gpu)
        r = w.relax(x, fire_params(force_tol=1e-3))
        return systems, w, x, r["energy"].copy()

    rows = {"direction": [], "score": []}
    for seed in (1, 2):
        systems, w, x, em = make(seed, 96)
        xm = x.cpu().numpy()
        sd = np.concatenate([cf.local_displacements(xm[w.offsets[k]:w.offsets[k + 1]], s.box,
                                                    cf.fcc_sites(s.meta["ncell"], 3.615)[s.meta["vacancies"][0]], 1,
                                                    seed=seed * 1000 + k)[0] for k, s in enumerate(systems)])
        xs = torch.tensor(xm + sd, device=gpu)
        res = w.dimer(xs, torch.tensor(sd, device=gpu), p)
        desc, B = w.descriptors(x, with_basis=True)
        usable = (res["status"] == CONVERGED) & (res["energy"] - em < 2.0)
        r = P.hop_rows(desc.cpu().numpy(), B.cpu().numpy(), xm, xs.cpu().numpy(), w.offsets,
                       [s.box for s in systems], usable)
        rows["direction"].append(r["direction"])
        rows["score"].append(r["score"])
    cat = lambda parts: tuple(np.concatenate(z) for z in zip(*parts))  # noqa: E731
    rows = {k: cat(v) for k, v in rows.items()}
    prop = P.Proposer(seed=0)
    prop.fit(rows, dir_epochs=150, score_epochs=30)

    systems, w, x, em = make(3, 64)
    disp, mode, chosen = prop.propose(w, x, seed=9)
    xm = x.cpu().numpy()
    ch = chosen.cpu().numpy()
    dv = disp.cpu().numpy()
    near_vac, cosv = 0, []
    for k, s in enumerate(systems):
        assert ch[k] >= 0
        a = w.offsets[k]
        vac = cf.fcc_sites(s.meta["ncell"], 3.615)[s.meta["vacancies"][0]]
        d = vac - xm[a + ch[k]]
        d -= s.box * np.rint(d / s.box)
        r = np.linalg.norm(d)
        near_vac += r < 2.9
        g = mode.cpu().numpy()[a + ch[k]]
        cosv.append(g @ d / (np.linalg.norm(g) * r))
    assert near_vac >= 0.9 * len(systems)
    assert np.median(cosv) > 0.95
    res = w.dimer(x + disp, mode, p)
    conv = res["status"] == CONVERGED
    assert conv.mean() >= 0.9
    barrier = res["energy"][conv] - em[conv]
    assert (barrier < 2.0).mean() >= 0.9


def test_relax_subset(gpu, hop_set):
    """FIRE of a walker subset: the walkers run are bitwise the full call's, the others keep
    their positions and report skipped."""
    import torch
    from akmc_b200.walkers import SKIPPED
    _, _, w, xm, _, sd = hop_set
    start = xm + 0.3 * sd
    x_all = torch.tensor(start, device=gpu)
    full = w.relax(x_all, fire_params(force_tol=1e-4))
    mask = np.array([0, 1, 1, 0, 1, 0, 0, 1], dtype=np.int32)
    x_sub = torch.tensor(start, device=gpu)
    sub = w.relax_subset(x_sub, torch.tensor(mask, device=gpu), fire_params(force_tol=1e-4))
    xa, xs = x_all.cpu().numpy(), x_sub.cpu().numpy()
    for k in range(w.W):
        a, b = w.offsets[k], w.offsets[k + 1]
        if mask[k]:
            assert sub["status"][k] == full["status"][k] == CONVERGED
            assert sub["iters"][k] == full["iters"][k] and sub["energy"][k] == full["energy"][k]
            assert np.array_equal(xs[a:b], xa[a:b])
        else:
            assert sub["status"][k] == SKIPPED
            assert np.array_equal(xs[a:b], start[a:b])


def test_masked_first_call_on_fresh_walkers(gpu, potdir):
    """A walker set whose first call skips a walker between two others: the skipped walker's
    systems are never sorted, and the walkers that run still match a full call on another
    fresh set bit for bit (a system's last cell is measured against the next system's first
    cell start, valid before that system is ever sorted)."""
    import torch
    systems = [cf.fcc_vacancy_system(n, seed=70 + k, vacancy_sites=[int(k * 37 % 256)])
               for k, n in enumerate((6, 4, 6, 4))]
    f = _field(potdir, systems[0].lat, max(s.n for s in systems))
    start = np.concatenate([s.pos for s in systems])
    mask = np.array([1, 0, 1, 1], dtype=np.int32)
    # FIRE
    wa, wb = Walkers.from_systems(f, systems), Walkers.from_systems(f, systems)
    xa = torch.tensor(start, device=gpu)
    xb = torch.tensor(start, device=gpu)
    ra = wa.relax_subset(xa, torch.tensor(mask, device=gpu), fire_params(force_tol=1e-4))
    rb = wb.relax(xb, fire_params(force_tol=1e-4))
    xa_h, xb_h = xa.cpu().numpy(), xb.cpu().numpy()
    for k in range(len(systems)):
        a, b = wa.offsets[k], wa.offsets[k + 1]
        if mask[k]:
            assert ra["status"][k] == rb["status"][k] == CONVERGED
            assert ra["energy"][k] == rb["energy"][k] and ra["iters"][k] == rb["iters"][k]
            assert np.array_equal(xa_h[a:b], xb_h[a:b])
        else:
            assert ra["status"][k] == SKIPPED
    # Dimer from the relaxed minima of the full call, on two more fresh sets
    xm = xb_h
    sd = np.concatenate([cf.local_displacements(xm[wb.offsets[k]:wb.offsets[k + 1]], s.box,
                                                cf.fcc_sites(s.meta["ncell"], 3.615)[s.meta["vacancies"][0]], 1,
                                                seed=500 + k)[0] for k, s in enumerate(systems)])
    p = dimer_params(delta=0.005, rot_tol=0.1, max_iter=200)
    wc, wd = Walkers.from_systems(f, systems), Walkers.from_systems(f, systems)
    xc, mc = torch.tensor(xm + sd, device=gpu), torch.tensor(sd, device=gpu)
    xd, md = torch.tensor(xm + sd, device=gpu), torch.tensor(sd, device=gpu)
    rc = wc.dimer_subset(xc, mc, torch.tensor(mask, device=gpu), p)
    rd = wd.dimer(xd, md, p)
    xc_h, xd_h = xc.cpu().numpy(), xd.cpu().numpy()
    for k in range(len(systems)):
        a, b = wc.offsets[k], wc.offsets[k + 1]
        if mask[k]:
            assert rc["status"][k] == rd["status"][k]
            assert rc["energy"][k] == rd["energy"][k] and rc["iters"][k] == rd["iters"][k]
            assert np.array_equal(xc_h[a:b], xd_h[a:b])
        else:
            assert rc["status"][k] == SKIPPED
            assert np.array_equal(xc_h[a:b], (xm + sd)[a:b])
