"""EAM neighbour-list reuse (akmc_batch_create_skin): lists built for cutoff + skin serve
later calls until an atom moves more than skin/2, with the exact rsq <= cutoff^2 test kept,
so every call's forces equal a fresh cell scan's to the last bits of the sums."""
import numpy as np
import pytest

import oracle
from akmc_b200 import configs as cf
from akmc_b200.field import Field, PREC_FP64, PREC_MIXED
from akmc_b200.walkers import Walkers, dimer_params, CONVERGED
from oracle import walkers as W

pytestmark = pytest.mark.gpu

TOL = {PREC_FP64: (1e-12, 1e-10), PREC_MIXED: (1e-10, 1e-8)}   # energy rel, force abs


@pytest.mark.parametrize("prec", [PREC_FP64, PREC_MIXED])
def test_reused_lists_match_cell_scan(gpu, potdir, prec):
    import torch
    systems = [cf.fcc_vacancy_system(4, seed=1), cf.fcc_vacancy_system(6, seed=2),
               cf.fcc_vacancy_system(5, n_vacancies=2, seed=3)]
    f = Field().readPotential(str(potdir / "eam.pot")).setup(systems[1].lat, None, 900)
    f.setPrecision(prec)
    nat = [s.n for s in systems]
    boxes = np.array([s.box for s in systems])
    labs = np.concatenate([s.labels for s in systems])
    bs = f.batch(nat, boxes, labs, skin=0.4)
    b0 = f.batch(nat, boxes, labs)
    x = np.concatenate([s.pos for s in systems])
    rng = np.random.default_rng(9)
    off = np.concatenate([[0], np.cumsum(nat)])
    for step in range(14):
        if step > 0:
            x = x + rng.normal(0.0, 0.01, x.shape)          # a relaxation-sized step
        if step == 9:
            x[off[1] + 5] += np.array([0.25, 0.0, 0.0])     # one atom of system 1 jumps
        outs = []
        for b in (bs, b0):
            pos = torch.tensor(x, device=gpu)
            F, E, S = b.alloc(gpu)
            b.forces_(pos, F, E, S)
            torch.cuda.synchronize()
            assert int(S.max()) == 0
            outs.append((F.cpu().numpy(), E.cpu().numpy(), pos.cpu().numpy()))
        (Fs, Es, Ps), (F0, E0, P0) = outs
        assert np.array_equal(Ps, P0)                       # the same wrap
        et, ft = TOL[prec]
        assert np.all(np.abs(Es[:, 0] - E0[:, 0]) <= et * np.abs(E0[:, 0]))
        assert np.abs(Fs - F0).max() <= ft
        modes = bs.list_modes()
        if step == 0:
            assert list(modes) == [1, 1, 1]
        elif step == 9:
            assert modes[1] == 1                             # rebuilt: 0.25 A > skin / 2
        if step in (1, 2):
            assert list(modes) == [2, 2, 2]
        x = Ps
    # the last configuration against the FP64 oracle
    for k, s in enumerate(systems):
        Eo, Fo, _, _ = oracle.eam_forces(str(potdir / "eam.pot"), x[off[k]:off[k + 1]], s.labels, s.lat)
        assert abs(Es[k, 0] - Eo["total"]) <= 1e-6 * abs(Eo["total"])
        assert np.abs(Fs[off[k]:off[k + 1]] - Fo).max() <= 1e-5


def test_walkers_with_and_without_skin(gpu, potdir):
    import torch
    s = cf.fcc_vacancy_system(4, sigma=0.0)
    eo = W.EamOracle(str(potdir / "eam.pot"), s.lat, s.labels)
    r = W.fire_relax(eo, s.pos, p=W.FireParams(force_tol=1e-5, norm_tol=1e-6))
    xmin, emin = r["pos"], r["energy"]
    seeds = cf.local_displacements(xmin, s.box, [0.0, 0.0, 0.0], 6, seed=11)
    f = Field().readPotential(str(potdir / "eam.pot")).setup(s.lat, None, s.n)
    res = {}
    for skin in (0.4, 0.0):
        w = Walkers.from_systems(f, [s] * 6)
        w.set_skin(skin)
        assert abs(w.skin - skin) < 1e-15
        pos = torch.tensor(np.concatenate([xmin + d for d in seeds]), device=gpu)
        mode = torch.tensor(np.concatenate(list(seeds)), device=gpu)
        res[skin] = w.dimer(pos, mode, dimer_params(force_tol=1e-3))
        w.close()
    a, b = res[0.4], res[0.0]
    both = (a["status"] == CONVERGED) & (b["status"] == CONVERGED)
    assert both.sum() >= 3
    assert np.abs(a["energy"][both] - b["energy"][both]).max() < 1e-3
