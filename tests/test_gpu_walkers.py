"""Batched FIRE and Dimer walkers on the GPU (akmc_walkers_*) against the FP64 oracle.

Parity bars: FIRE minima to 1e-6 relative energy (the force-path bar) and 1e-3 A in
position; Dimer saddle energies and barriers to 1 meV (the saddle bar), each also
stated against the FP64 oracle run from the same start.
"""
import numpy as np
import pytest

from akmc_b200 import configs as cf
from akmc_b200.field import Field, PREC_FP64, PREC_MIXED
from akmc_b200.walkers import Walkers, dimer_params, fire_params, CONVERGED
import oracle
from oracle import walkers as W

pytestmark = pytest.mark.gpu


def _wrapdiff(a, b, box):
    d = a - b
    return d - box * np.rint(d / box)


def _field(path, lat, n, precision):
    f = Field().readPotential(str(path))
    f.setup(lat, None, n)
    f.setPrecision(precision)
    return f


def _stack(systems):
    return np.concatenate([s.pos for s in systems])


@pytest.fixture(scope="module")
def vacancy_min(potdir):
    """Unjittered 4x4x4 FCC with one vacancy, FIRE-relaxed by the oracle."""
    s = cf.fcc_vacancy_system(4, sigma=0.0)
    eo = W.EamOracle(str(potdir / "eam.pot"), s.lat, s.labels)
    r = W.fire_relax(eo, s.pos, p=W.FireParams(force_tol=1e-5, norm_tol=1e-6))
    assert r["status"] == 1
    return s, eo, r["pos"], r["energy"]


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_fire_batch_matches_oracle(gpu, potdir, precision):
    import torch
    systems = [cf.fcc_vacancy_system(4, seed=1234), cf.fcc_vacancy_system(4, seed=99),
               cf.fcc_vacancy_system(5, n_vacancies=2, seed=7)]
    f = _field(potdir / "eam.pot", systems[2].lat, max(s.n for s in systems), precision)
    w = Walkers.from_systems(f, systems)
    pos = torch.tensor(_stack(systems), device=gpu)
    res = w.relax(pos)
    out = pos.cpu().numpy()
    for k, s in enumerate(systems):
        r = W.fire_relax(W.EamOracle(str(potdir / "eam.pot"), s.lat, s.labels), s.pos)
        assert res["status"][k] == CONVERGED and r["status"] == 1
        assert abs(res["energy"][k] - r["energy"]) <= 1e-6 * abs(r["energy"])
        x = out[w.offsets[k]:w.offsets[k + 1]]
        assert np.abs(_wrapdiff(x, r["pos"], s.box)).max() < 1e-3
        if precision == PREC_FP64:
            assert abs(res["energy"][k] - r["energy"]) < 1e-9
            assert abs(int(res["iters"][k]) - r["iters"]) <= 2


def test_fire_frozen_atoms(gpu, potdir):
    import torch
    s = cf.fcc_vacancy_system(4, seed=77)
    frozen = np.zeros(s.n, np.int32)
    frozen[::7] = 1
    f = _field(potdir / "eam.pot", s.lat, s.n, PREC_FP64)
    w = Walkers.from_systems(f, [s], frozen=frozen)
    pos = torch.tensor(s.pos, device=gpu)
    res = w.relax(pos, fire_params(max_iter=400))
    x = pos.cpu().numpy()
    assert np.abs(_wrapdiff(x[frozen == 1], s.pos[frozen == 1], s.box)).max() < 1e-12
    r = W.fire_relax(W.EamOracle(str(potdir / "eam.pot"), s.lat, s.labels), s.pos, frozen=frozen,
                     p=W.FireParams(max_iter=400))
    assert (res["status"][0] == CONVERGED) == (r["status"] == 1)
    assert abs(res["energy"][0] - r["energy"]) < 1e-8
    assert np.abs(_wrapdiff(x, r["pos"], s.box)).max() < 1e-5


def test_fire_ionic_trajectory(gpu, potdir):
    """Rocksalt (510 ions): 40 FIRE steps on the GPU (FP64 terms) follow the oracle's."""
    import torch
    s = cf.rocksalt_schottky_system(4, seed=5)
    f = _field(potdir / "ion8_shell0.pot", s.lat, s.n, PREC_FP64)
    w = Walkers.from_systems(f, [s])
    pos = torch.tensor(s.pos, device=gpu)
    res = w.relax(pos, fire_params(max_iter=40))
    io = W.IonicOracle(str(potdir / "ion8_shell0.pot"), s.lat, s.charge, s.labels)
    r = W.fire_relax(io, s.pos, p=W.FireParams(max_iter=40))
    assert res["iters"][0] == r["iters"] == 40
    assert abs(res["energy"][0] - r["energy"]) <= 1e-9 * abs(r["energy"])
    assert np.abs(_wrapdiff(pos.cpu().numpy(), r["pos"], s.box)).max() < 1e-8


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_dimer_saddles_match_oracle(gpu, potdir, vacancy_min, precision):
    import torch
    s, eo, xmin, emin = vacancy_min
    nw = 6
    seeds = cf.local_displacements(xmin, s.box, [0.0, 0.0, 0.0], nw, seed=11)
    f = _field(potdir / "eam.pot", s.lat, s.n, precision)
    w = Walkers.from_systems(f, [s] * nw)
    pos = torch.tensor(np.concatenate([xmin + d for d in seeds]), device=gpu)
    mode = torch.tensor(np.concatenate(list(seeds)), device=gpu)
    p = dimer_params(force_tol=1e-3)                  # tight: isolates the precision effects
    res = w.dimer(pos, mode, p)
    out = pos.cpu().numpy()
    op = W.DimerParams(force_tol=1e-3)
    matched = 0
    for k in range(nw):
        o = W.dimer_search(eo, xmin + seeds[k], seeds[k], op)
        if precision == PREC_FP64:
            assert res["status"][k] == o["status"]
        if res["status"][k] != CONVERGED or o["status"] != 1:
            continue
        matched += 1
        # a saddle: small force, negative curvature, checked with the oracle's forces
        x = out[w.offsets[k]:w.offsets[k + 1]]
        F, E, _ = eo(x)
        assert np.sqrt((F * F).sum(1)).max() < 2 * p.force_tol
        assert res["curvature"][k] < 0.0
        assert abs(res["energy"][k] - E) <= 1e-7 * abs(E)
        # the saddle bar: energy and barrier against the FP64 oracle search
        assert abs(res["energy"][k] - o["energy"]) < 1e-3
        assert abs((res["energy"][k] - emin) - (o["energy"] - emin)) < 1e-3
        assert np.abs(_wrapdiff(x, o["pos"], s.box)).max() < 0.05
    assert matched >= 3


def test_dimer_is_deterministic(gpu, potdir, vacancy_min):
    import torch
    s, eo, xmin, emin = vacancy_min
    seeds = cf.local_displacements(xmin, s.box, [0.0, 0.0, 0.0], 4, seed=5)
    f = _field(potdir / "eam.pot", s.lat, s.n, PREC_MIXED)
    w = Walkers.from_systems(f, [s] * 4)
    runs = []
    for _ in range(2):
        pos = torch.tensor(np.concatenate([xmin + d for d in seeds]), device=gpu)
        mode = torch.tensor(np.concatenate(list(seeds)), device=gpu)
        res = w.dimer(pos, mode)
        runs.append((res, pos.cpu().numpy(), mode.cpu().numpy()))
    assert runs[0][0].tobytes() == runs[1][0].tobytes()
    assert np.array_equal(runs[0][1], runs[1][1]) and np.array_equal(runs[0][2], runs[1][2])


def test_dimer_uneven_walkers(gpu, potdir):
    """Walkers of 255 and 863 atoms in one set: every converged walker is a saddle of its
    own system by the oracle's forces, and the vacancy-hop barriers agree across sizes."""
    import torch
    small = cf.fcc_vacancy_system(4, sigma=0.0)
    big = cf.fcc_vacancy_system(6, sigma=0.0)
    mins, seeds, systems = [], [], []
    for s in (small, big):
        eo = W.EamOracle(str(potdir / "eam.pot"), s.lat, s.labels)
        r = W.fire_relax(eo, s.pos, p=W.FireParams(force_tol=1e-5, norm_tol=1e-6))
        mins.append((eo, r["pos"], r["energy"]))
    order = [0, 1, 1, 0, 1, 0]
    for j, k in enumerate(order):
        s = (small, big)[k]
        d = cf.local_displacements(mins[k][1], s.box, [0.0, 0.0, 0.0], 1, seed=100 + j)[0]
        seeds.append(d)
        systems.append(s)
    f = _field(potdir / "eam.pot", big.lat, big.n, PREC_MIXED)
    w = Walkers.from_systems(f, systems)
    pos = torch.tensor(np.concatenate([mins[k][1] + d for k, d in zip(order, seeds)]), device=gpu)
    mode = torch.tensor(np.concatenate(seeds), device=gpu)
    res = w.dimer(pos, mode, dimer_params(force_tol=1e-3))
    out = pos.cpu().numpy()
    barriers = {0: [], 1: []}
    for j, k in enumerate(order):
        if res["status"][j] != CONVERGED:
            continue
        eo, xm, em = mins[k]
        x = out[w.offsets[j]:w.offsets[j + 1]]
        F, E, _ = eo(x)
        assert np.sqrt((F * F).sum(1)).max() < 2e-3
        assert abs(E - res["energy"][j]) <= 1e-7 * abs(E)       # the 1e-6 relative bar, x10
        barriers[k].append(res["energy"][j] - em)
    assert len(barriers[0]) + len(barriers[1]) >= 4
    allb = np.array(barriers[0] + barriers[1])
    assert np.ptp(allb) < 5e-3          # the same hop, finite-size shift only


def test_ionic_dimer_mixed_vs_fp64(gpu, potdir):
    """The ionic configuration's 16 searches: rocksalt 5x5x5 with a Schottky pair (998 ions,
    10 A cutoff, eta 0.3), Dimer walkers started on the nearest-neighbour hops into both
    vacancies (8 cation, 8 anion).  FP32 pair terms with FP64 accumulation against an all-FP64
    run from the same starts: at least 14 of 16 reach the same saddle in both, and their
    barriers agree within the 1 meV bar."""
    import torch
    s = cf.rocksalt_schottky_system(5, seed=4321)
    pot = potdir / "ion10_shell0.pot"
    nw = 16
    out = {}
    for prec in (PREC_FP64, PREC_MIXED):
        f = _field(pot, s.lat, s.n, prec)
        one = Walkers.from_systems(f, [s])
        x = torch.tensor(s.pos, device=gpu)
        # both minima to 1e-4 eV/A: the barriers subtract them, and at 1e-3 where FIRE stops
        # moves the minimum energy by up to a meV
        r = one.relax(x, fire_params(force_tol=1e-4, norm_tol=1e-6, max_iter=4000))
        assert r["status"][0] == CONVERGED
        xmin, emin = x.cpu().numpy(), float(r["energy"][0])
        if prec == PREC_FP64:
            seeds = cf.rocksalt_hop_starts(xmin, s.labels, s.box, per_site=nw // 2, seed=31)
            x_ref = xmin
        w = Walkers.from_systems(f, [s] * nw)
        pos = torch.tensor(np.concatenate([x_ref + d for d in seeds]), device=gpu)
        mode = torch.tensor(np.concatenate(list(seeds)), device=gpu)
        res = w.dimer(pos, mode, dimer_params(max_iter=600, force_tol=1e-3))
        out[prec] = (res, emin, pos.cpu().numpy())
    (r64, e64, x64), (r32, e32, x32) = out[PREC_FP64], out[PREC_MIXED]
    assert abs(e64 - e32) <= 1e-6 * abs(e64)           # the minimum itself, to the energy bar
    n = s.n
    both = 0
    for k in range(nw):
        if r64["status"][k] != CONVERGED or r32["status"][k] != CONVERGED:
            continue
        d = _wrapdiff(x64[k * n:(k + 1) * n], x32[k * n:(k + 1) * n], s.box)
        if np.abs(d).max() > 0.05:
            continue                                  # the two runs reached different saddles
        both += 1
        assert r64["curvature"][k] < 0 and r32["curvature"][k] < 0
        assert abs((r64["energy"][k] - e64) - (r32["energy"][k] - e32)) < 1e-3
    assert both >= 14


@pytest.mark.skipif(not oracle.reference_available("eam"), reason="reference not built")
@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_dimer_barrier_matches_reference_art(gpu, potdir, vacancy_min, precision):
    """Barriers of the GPU Dimer against the reference's own saddle search: the reference's
    ART (optim/ART.cpp unchanged, on the reference's EAM Field) from the same starts near the
    vacancy hops.  The saddle bar is 1 meV; both agree to 0.2 meV."""
    import torch
    s, eo, xmin, emin = vacancy_min
    starts = cf.vacancy_hop_starts(xmin, s.box, [0.0, 0.0, 0.0], k=6)
    ref = oracle.ReferenceField("eam", str(potdir / "eam.pot"), s.lat, s.n)
    e_ref = ref.forces(xmin, s.charge, s.labels)[0]["total"]
    f = _field(potdir / "eam.pot", s.lat, s.n, precision)
    w = Walkers.from_systems(f, [s] * len(starts))
    pos = torch.tensor(np.concatenate([xmin + d for d in starts]), device=gpu)
    mode = torch.tensor(np.concatenate(starts), device=gpu)
    res = w.dimer(pos, mode, dimer_params(force_tol=1e-3))
    for k, sd in enumerate(starts):
        assert res["status"][k] == CONVERGED
        st, e_art, _ = ref.art(xmin, s.charge, s.labels, sd, init_dt=0.0005, max_dt=0.001, max_par_iter=3000)
        assert st == 0
        assert abs((res["energy"][k] - emin) - (e_art - e_ref)) < 2e-4

@pytest.mark.skipif(not oracle.reference_available("eam"), reason="reference not built")
@pytest.mark.parametrize("ncell", [6, 8])
def test_dimer_barrier_matches_reference_art_larger_cells(gpu, potdir, ncell):
    """The same check on the batched-walker configuration's larger size classes (6^3 and 8^3
    cells, 863 and 2047 atoms), mixed precision: GPU Dimer barriers against the reference's
    own ART from the same near-hop starts, within the 1 meV saddle bar."""
    import torch
    s = cf.fcc_vacancy_system(ncell, sigma=0.0)
    eo = W.EamOracle(str(potdir / "eam.pot"), s.lat, s.labels)
    r = W.fire_relax(eo, s.pos, p=W.FireParams(force_tol=1e-5, norm_tol=1e-6))
    assert r["status"] == 1
    xmin, emin = r["pos"], r["energy"]
    starts = cf.vacancy_hop_starts(xmin, s.box, [0.0, 0.0, 0.0], k=2)
    ref = oracle.ReferenceField("eam", str(potdir / "eam.pot"), s.lat, s.n)
    e_ref = ref.forces(xmin, s.charge, s.labels)[0]["total"]
    f = _field(potdir / "eam.pot", s.lat, s.n, PREC_MIXED)
    w = Walkers.from_systems(f, [s] * len(starts))
    pos = torch.tensor(np.concatenate([xmin + d for d in starts]), device=gpu)
    mode = torch.tensor(np.concatenate(starts), device=gpu)
    res = w.dimer(pos, mode, dimer_params(force_tol=1e-3))
    for k, sd in enumerate(starts):
        assert res["status"][k] == CONVERGED
        st, e_art, _ = ref.art(xmin, s.charge, s.labels, sd, init_dt=0.0005, max_dt=0.001, max_par_iter=3000)
        assert st == 0
        assert abs((res["energy"][k] - emin) - (e_art - e_ref)) < 1e-3


def test_dimer_frozen_atoms_local_region(gpu, potdir):
    """Walkers over local regions: the Dimer honours frozen atoms as FIRE does.  A vacancy hop
    in the 10^3 crystal (3999 atoms) searched twice from the same start -- in the whole crystal
    with every atom beyond 6 A of the vacancy frozen, and in the local region cut out of it
    (akmc_b200.configs.local_region: the free atoms and two cutoffs plus 1 A of fixed atoms
    around them) -- reaches the same saddle: frozen atoms keep their positions bit for bit and
    the two barriers agree far inside the 1 meV bar."""
    import torch
    s = cf.fcc_vacancy_system(10, sigma=0.0)
    site = cf.fcc_sites(10, 3.615)[s.meta["vacancies"][0]]
    f = _field(potdir / "eam.pot", s.lat, s.n, PREC_MIXED)
    one = Walkers.from_systems(f, [s])
    x = torch.tensor(s.pos, device=gpu)
    assert one.relax(x, fire_params(force_tol=1e-5, norm_tol=1e-6, max_iter=3000))["status"][0] == CONVERGED
    xmin = x.cpu().numpy()
    start = cf.vacancy_hop_starts(xmin, s.box, site, k=1)[0]
    reg = cf.local_region(xmin, s.labels, s.charge, s.box, site, 6.0, 5.0)
    frozen = np.ones(s.n, np.int32)
    frozen[reg.index[reg.frozen == 0]] = 0
    start[frozen == 1] = 0.0
    p = dimer_params(force_tol=1e-3)
    # the whole crystal, atoms beyond 6 A frozen
    wf = Walkers.from_systems(f, [s], frozen=frozen)
    e_min = f.forces(xmin, s.labels)[0]["total"]
    xs = torch.tensor(xmin + start, device=gpu)
    rf = wf.dimer(xs, torch.tensor(start, device=gpu), p)
    assert rf["status"][0] == CONVERGED and rf["curvature"][0] < 0
    xf = xs.cpu().numpy()
    # frozen atoms keep their positions (up to the wrap into the minimum-image cell)
    assert np.abs(_wrapdiff(xf[frozen == 1], xmin[frozen == 1], s.box)).max() < 1e-12
    # the local region alone
    fr = _field(potdir / "eam.pot", reg.system.lat, reg.system.n, PREC_MIXED)
    fr.set_list_density(s.n / float(np.prod(s.box)))   # the region is as dense as the crystal
    wr = Walkers.from_systems(fr, [reg.system], frozen=reg.frozen)
    e_min_r = fr.forces(reg.system.pos, reg.system.labels)[0]["total"]
    xr = torch.tensor(reg.system.pos + start[reg.index], device=gpu)
    rr = wr.dimer(xr, torch.tensor(start[reg.index], device=gpu), p)
    assert rr["status"][0] == CONVERGED
    assert np.abs(_wrapdiff(xr.cpu().numpy()[reg.frozen == 1], reg.system.pos[reg.frozen == 1],
                            reg.system.box)).max() < 1e-12
    assert abs((rf["energy"][0] - e_min) - (rr["energy"][0] - e_min_r)) < 2e-4
    d = (xr.cpu().numpy() - reg.shift) - xf[reg.index]
    d -= s.box * np.rint(d / s.box)
    assert np.abs(d).max() < 0.02


def test_dimer_patience_stops_stalled_walkers(gpu, potdir, vacancy_min):
    """The stall rule (akmc_dimer_params.patience): with it off a search runs as before; with a
    patience of a few steps, walkers whose max|F| stops falling end early with status
    MAX_ITER instead of running out the horizon, and converged walkers are unchanged."""
    import torch
    s, eo, xmin, emin = vacancy_min
    starts = cf.local_displacements(xmin, s.box, [0.0, 0.0, 0.0], 8, seed=21)
    f = _field(potdir / "eam.pot", s.lat, s.n, PREC_MIXED)
    w = Walkers.from_systems(f, [s] * len(starts))
    out = {}
    for pat in (0, 3):
        pos = torch.tensor(np.concatenate([xmin + d for d in starts]), device=gpu)
        mode = torch.tensor(np.concatenate(list(starts)), device=gpu)
        out[pat] = w.dimer(pos, mode, dimer_params(force_tol=1e-3, max_iter=200, patience=pat))
    r0, r3 = out[0], out[3]
    assert (r3["iters"] <= r0["iters"]).all()
    stopped = (r3["status"] == 2) & (r3["iters"] < 200)
    assert stopped.any()
    both = (r0["status"] == CONVERGED) & (r3["status"] == CONVERGED)
    assert np.array_equal(r0["iters"][both], r3["iters"][both])
    assert np.abs(r0["energy"][both] - r3["energy"][both]).max(initial=0.0) == 0.0
