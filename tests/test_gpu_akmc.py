"""An adaptive-KMC trajectory on the GPU (akmc_b200.akmc_loop): batched Dimer searches,
basin-2 relaxations, the FP64 event table and the KMC step, checked against the FP64 oracle
selection and the physics of a single vacancy in FCC."""
import numpy as np
import pytest

from akmc_b200 import configs as cf
from akmc_b200.akmc_loop import AkmcLoop
from akmc_b200.field import Field, PREC_MIXED
from oracle import kmc as K

pytestmark = pytest.mark.gpu


def test_vacancy_hops(gpu, potdir):
    s = cf.fcc_vacancy_system(4, sigma=0.0)
    f = Field().readPotential(str(potdir / "eam.pot")).setup(s.lat, None, s.n)
    f.setPrecision(PREC_MIXED)
    find = cf.fcc_vacancy_finder(4, 3.615)
    loop = AkmcLoop(f, s, find, n_walkers=16, seed=5)
    sites = [find(s.pos)[0]]
    last_t = 0.0
    for k in range(3):
        rec = loop.step()
        tab = loop.last_table
        assert rec.n_unique >= 1 and rec.chosen >= 0
        # every unique event is a nearest-neighbour hop: one barrier, basin 2 at E_min
        b = tab["e_saddle"][tab["unique"]] - tab["e_min"]
        assert np.ptp(b) < 1e-3 and abs(b[0] - 1.2522) < 5e-3
        assert np.all(np.abs(tab["e_basin2"][tab["unique"]] - tab["e_min"]) < 2e-3)
        # the device selection is the oracle's, in FP64
        r = K.rates(tab["e_saddle"], np.full(16, tab["e_min"]), tab["unique"], 1e13, 600.0)
        ch, tot, dt = K.select(r, tab["u"][0], tab["u"][1])
        assert ch == rec.chosen
        assert abs(rec.total_rate - tot) <= 1e-14 * tot and abs(rec.dt - dt) <= 1e-14 * dt
        # time advances; the vacancy moved by one nearest-neighbour distance
        assert rec.time > last_t
        last_t = rec.time
        v = find(loop.pos)
        assert len(v) == 1
        d = v[0] - sites[-1]
        d -= s.box * np.rint(d / s.box)
        assert abs(np.linalg.norm(d) - 3.615 / np.sqrt(2)) < 1e-6
        sites.append(v[0])


def test_restart_continues_the_trajectory(gpu, potdir, tmp_path):
    """Dump the basin after each step (the reference's archive layout), restart a new loop
    from the last block, and take the next step in both: the same event, to the rounding
    of the ten-decimal positions."""
    s = cf.fcc_vacancy_system(4, sigma=0.0)
    f = Field().readPotential(str(potdir / "eam.pot")).setup(s.lat, None, s.n)
    find = cf.fcc_vacancy_finder(4, 3.615)
    a = AkmcLoop(f, s, find, n_walkers=12, seed=9)
    arch = tmp_path / "archive"
    with open(arch, "w") as out:
        for k in range(2):
            a.step()
            a.dump(out, ["Cu"], header=(k == 0))
    b = AkmcLoop(f, s, find, n_walkers=12, seed=9)
    b.resume(str(arch), ["Cu"])
    assert b.iteration == a.iteration == 2
    assert abs(b.time - a.time) <= 1e-9 * a.time
    assert np.abs(b.pos - a.pos).max() < 1e-9
    ra, rb = a.step(), b.step()
    assert ra.chosen == rb.chosen
    assert abs(ra.barrier - rb.barrier) < 1e-5
    assert np.allclose(find(a.pos), find(b.pos))


def test_learned_proposals_in_the_loop(gpu, potdir):
    """A trajectory whose walkers learn where to start: the first step searches from random
    seeds, its saddles train the proposer, and the next steps start from learned proposals.
    Every step still finds the nearest-neighbour vacancy hop and moves the vacancy by one
    hop; the learned steps spend fewer force calls than the random one and cover several of
    the symmetry-equivalent hops."""
    from akmc_b200 import proposals as P
    s = cf.fcc_vacancy_system(4, sigma=0.0)
    f = Field().readPotential(str(potdir / "eam.pot")).setup(s.lat, None, s.n)
    f.setPrecision(PREC_MIXED)
    find = cf.fcc_vacancy_finder(4, 3.615)
    loop = AkmcLoop(f, s, find, n_walkers=16, seed=11, proposer=P.Proposer(seed=0))
    site = find(s.pos)[0]
    recs = []
    for k in range(4):
        rec = loop.step()
        recs.append(rec)
        tab = loop.last_table
        assert rec.chosen >= 0 and rec.n_unique >= 2
        b = tab["e_saddle"][tab["unique"]] - tab["e_min"]
        assert np.ptp(b) < 1e-3 and abs(b[0] - 1.2522) < 5e-3
        v = find(loop.pos)
        assert len(v) == 1
        d = v[0] - site
        d -= s.box * np.rint(d / s.box)
        assert abs(np.linalg.norm(d) - 3.615 / np.sqrt(2)) < 1e-6
        site = v[0]
    assert not recs[0].learned and all(r.learned for r in recs[1:])
    assert np.mean([r.force_calls for r in recs[1:]]) < recs[0].force_calls


def test_local_region_loop(gpu, potdir):
    """The loop with walkers over local regions (active radius 6 A) on a vacancy in the 10^3
    crystal (3999 atoms): each search walker holds under half of the crystal, the unique
    saddles within the polish window are polished in the crystal, the hops among them are
    nearest-neighbour hops whose barrier is the FP64 oracle's at the same crystal positions
    (the hop barrier of the free crystal, not the 0.15 eV higher one of the region's fixed
    shell); the vacancy moves one neighbour distance per step."""
    from oracle import walkers as W
    s = cf.fcc_vacancy_system(10, sigma=0.0)
    f = Field().readPotential(str(potdir / "eam.pot")).setup(s.lat, None, s.n)
    f.setPrecision(PREC_MIXED)
    find = cf.fcc_vacancy_finder(10, 3.615)
    loop = AkmcLoop(f, s, find, n_walkers=16, seed=5, active_radius=6.0, keep_saddles=3)
    site = find(s.pos)[0]
    for k in range(2):
        rec = loop.step()
        tab = loop.last_table
        assert rec.n_unique >= 1 and rec.chosen >= 0
        assert rec.atoms_per_walker < s.n // 2
        assert rec.polished + rec.unpolished >= rec.n_unique
        b = tab["e_saddle"][tab["unique"]] - tab["e_min"]
        hops = b[b < 2.0]              # saddles far above (concerted moves) stay at their region barrier
        assert len(hops) >= 1 and np.ptp(hops) < 1e-3 and abs(hops[0] - 1.2522) < 1e-2
        for sysq, xm, xs, bar in loop.last_saddles:
            eo = W.EamOracle(str(potdir / "eam.pot"), sysq.lat, sysq.labels)
            assert abs(bar - (eo(xs)[1] - eo(xm)[1])) < 1e-3      # the saddle bar, mixed against FP64
        v = find(loop.pos)
        assert len(v) == 1
        d = v[0] - site
        d -= s.box * np.rint(d / s.box)
        assert abs(np.linalg.norm(d) - 3.615 / np.sqrt(2)) < 1e-6
        site = v[0]


def test_local_region_loop_recycles_far_events(gpu, potdir):
    """Two vacancies 31 A apart in the 10^3 crystal: after the first step one of them has
    hopped, and the second step's crystal polish of the other vacancy's hops starts from
    the first step's polished saddles (carried into the new basin); the hops are still
    nearest-neighbour hops with the free crystal's barrier, and every kept saddle's barrier
    is the FP64 oracle's at the same positions."""
    from oracle import walkers as W
    sites = cf.fcc_sites(10, 3.615)
    far = int(np.argmin(np.abs(sites - 5 * 3.615).sum(1)))      # the site at (L/2, L/2, L/2)
    s = cf.fcc_vacancy_system(10, sigma=0.0, vacancy_sites=[0, far])
    f = Field().readPotential(str(potdir / "eam.pot")).setup(s.lat, None, s.n)
    f.setPrecision(PREC_MIXED)
    find = cf.fcc_vacancy_finder(10, 3.615)
    loop = AkmcLoop(f, s, find, n_walkers=32, seed=9, active_radius=6.0, keep_saddles=4)
    recs = [loop.step() for _ in range(2)]
    assert recs[0].recycled == 0
    assert recs[1].recycled >= 1, recs[1]
    tab = loop.last_table
    b = tab["e_saddle"][tab["unique"]] - tab["e_min"]
    hops = b[b < 2.0]                     # the searches may also find concerted moves far above
    assert len(hops) >= 2 and np.abs(hops - 1.2522).max() < 1e-2, (b, recs[1])
    for sysq, xm, xs, bar in loop.last_saddles:
        eo = W.EamOracle(str(potdir / "eam.pot"), sysq.lat, sysq.labels)
        assert abs(bar - (eo(xs)[1] - eo(xm)[1])) < 1e-3

