"""CPU checks of the walker oracle (oracle/walkers.py).

* FIRE: the restatement, driven by the reference's own forces, reproduces the
  reference's Relax::RelaxStructure "fire" (optim/Relax.cpp:44-315, compiled from the
  reference sources) to round-off, and with the oracle's own forces to the same minimum.
* Dimer (no reference implementation exists): the saddles it returns are first-order
  saddles of the vacancy hop -- zero force, one negative curvature, equal barriers for
  symmetry-equivalent hops -- and each connects the start minimum with a hopped minimum
  of the same energy.
"""
import numpy as np
import pytest

import oracle
from oracle import walkers as W
from akmc_b200 import configs as cf


def _wrapdiff(a, b, box):
    d = a - b
    return d - box * np.rint(d / box)


@pytest.fixture(scope="module")
def vacancy(potdir):
    # unjittered lattice: every nearest-neighbour hop of the vacancy is symmetry-equivalent
    s = cf.fcc_vacancy_system(4, sigma=0.0)
    eo = W.EamOracle(str(potdir / "eam.pot"), s.lat, s.labels)
    r = W.fire_relax(eo, s.pos, p=W.FireParams(force_tol=1e-5, norm_tol=1e-6))
    assert r["status"] == 1
    return s, eo, r


@pytest.mark.skipif(not oracle.reference_available("eam"), reason="reference not built")
def test_fire_restatement_matches_reference_fire(potdir):
    s = cf.fcc_vacancy_system(4)
    ref = oracle.ReferenceField("eam", str(potdir / "eam.pot"), s.lat, s.n)
    st, E, xr = ref.relax(s.pos, s.charge, s.labels)
    assert st == 0                                    # Status SUCCESS

    def ref_forces(p):
        e, F, w = ref.forces(p, s.charge, s.labels)
        return F, e["total"], w

    r = W.fire_relax(ref_forces, s.pos)
    assert r["status"] == 1
    assert np.abs(_wrapdiff(r["pos"], xr, s.box)).max() < 1e-10
    assert abs(r["energy"] - E["total"]) < 1e-9
    # the oracle's own forces reach the same minimum
    r2 = W.fire_relax(W.EamOracle(str(potdir / "eam.pot"), s.lat, s.labels), s.pos)
    assert np.abs(_wrapdiff(r2["pos"], xr, s.box)).max() < 1e-8
    assert abs(r2["energy"] - E["total"]) < 1e-8


@pytest.mark.skipif(not oracle.reference_available("eam"), reason="reference not built")
def test_fire_restatement_frozen_atoms_match_reference(potdir):
    s = cf.fcc_vacancy_system(4, seed=77)
    frozen = np.zeros(s.n, np.int32)
    frozen[::7] = 1
    ref = oracle.ReferenceField("eam", str(potdir / "eam.pot"), s.lat, s.n)
    st, E, xr = ref.relax(s.pos, s.charge, s.labels, frozen=frozen, max_iter=400)

    def ref_forces(p):
        e, F, w = ref.forces(p, s.charge, s.labels)
        return F, e["total"], w

    r = W.fire_relax(ref_forces, s.pos, frozen=frozen, p=W.FireParams(max_iter=400))
    assert (r["status"] == 1) == (st == 0)
    assert np.abs(_wrapdiff(r["pos"], xr, s.box)).max() < 1e-10
    # frozen atoms never move (up to the wrap)
    assert np.abs(_wrapdiff(r["pos"][frozen == 1], s.pos[frozen == 1], s.box)).max() < 1e-12


def test_dimer_finds_vacancy_hop_saddle(vacancy):
    s, eo, rmin = vacancy
    xmin, emin = rmin["pos"], rmin["energy"]
    seeds = cf.local_displacements(xmin, s.box, [0.0, 0.0, 0.0], 4, seed=11)
    p = W.DimerParams(force_tol=1e-3)
    found = []
    for d in seeds:
        o = W.dimer_search(eo, xmin + d, d, p)
        if o["status"] != 1:
            continue
        assert o["curvature"] < 0.0
        assert o["fmax"] < p.force_tol
        found.append(o)
    assert len(found) >= 2
    barriers = np.array([o["energy"] - emin for o in found])
    # every seed found a nearest-neighbour vacancy hop: symmetry-equivalent barriers
    assert np.ptp(barriers) < 1e-4
    assert 1.0 < barriers[0] < 1.5
    # the saddle connects the start minimum with a hopped minimum of the same energy
    o = found[0]
    ends = []
    for sgn in (+1.0, -1.0):
        r = W.fire_relax(eo, o["pos"] + sgn * 0.1 * o["mode"], p=W.FireParams(force_tol=1e-4))
        assert r["status"] == 1
        ends.append(r)
    assert abs(ends[0]["energy"] - emin) < 2e-3 and abs(ends[1]["energy"] - emin) < 2e-3
    moved = [np.sqrt((_wrapdiff(e["pos"], xmin, s.box) ** 2).sum(1)).max() for e in ends]
    assert min(moved) < 0.1 and max(moved) > 2.0     # one end is the start, one the hop


@pytest.mark.skipif(not oracle.reference_available("eam"), reason="reference not built")
def test_dimer_barrier_matches_reference_art(potdir, vacancy):
    """The reference's own ART (optim/ART.cpp unchanged, on the reference's EAM Field;
    oracle/ref_art.cpp) and the FP64 oracle Dimer, started from the same points near a
    vacancy hop, reach saddles whose barriers agree to 0.1 meV."""
    s, eo, rmin = vacancy
    xmin, emin = rmin["pos"], rmin["energy"]
    ref = oracle.ReferenceField("eam", str(potdir / "eam.pot"), s.lat, s.n)
    e_ref, _, _ = ref.forces(xmin, s.charge, s.labels)
    assert abs(e_ref["total"] - emin) <= 1e-9 * abs(emin)
    for sd in cf.vacancy_hop_starts(xmin, s.box, [0.0, 0.0, 0.0]):
        st, e_art, x_art = ref.art(xmin, s.charge, s.labels, sd, init_dt=0.0005, max_dt=0.001,
                                   max_par_iter=3000)
        assert st == 0
        F, _, _ = eo(x_art)
        assert np.sqrt((F * F).sum(1)).max() < 1e-3          # the reference ART's own criterion
        o = W.dimer_search(eo, xmin + sd, sd, W.DimerParams(force_tol=1e-3))
        assert o["status"] == 1
        assert abs((e_art - e_ref["total"]) - (o["energy"] - emin)) < 1e-4
        assert abs((e_art - e_ref["total"]) - 1.2522) < 1e-3


def test_dimer_rotation_recovers_lowest_mode():
    """On a quadratic surface the rotation turns any start mode to the lowest-curvature
    eigenvector, and the translation lands on the saddle exactly."""
    rng = np.random.default_rng(3)
    n = 4
    Q, _ = np.linalg.qr(rng.normal(size=(3 * n, 3 * n)))
    evals = np.concatenate([[-1.5], np.linspace(0.5, 4.0, 3 * n - 1)])   # one unstable mode
    H = Q @ np.diag(evals) @ Q.T
    x0 = rng.normal(size=3 * n) * 0.3

    def fn(p):
        d = p.reshape(-1) - x0
        return (-(H @ d)).reshape(-1, 3), 0.5 * float(d @ H @ d), p.copy()

    start = x0 + 0.2 * rng.normal(size=3 * n)
    mode = rng.normal(size=3 * n)
    o = W.dimer_search(fn, start.reshape(-1, 3), mode.reshape(-1, 3),
                       W.DimerParams(force_tol=1e-6, max_iter=3000, max_rise=1e9, rot_tol=1e-4))
    assert o["status"] == 1
    assert np.abs(o["pos"].reshape(-1) - x0).max() < 1e-5
    lowest = Q[:, 0]
    assert abs(abs(float(o["mode"].reshape(-1) @ lowest)) - 1.0) < 1e-6
    assert abs(o["curvature"] - evals[0]) < 1e-3
