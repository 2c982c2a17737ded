"""Parity of the CUDA force path with the reference (golden vectors) and the FP64 oracle.

Bars (stated per test):
* energies to 1e-6 relative, forces to 1e-5 eV/A in the default mixed precision
  (FP32 terms, FP64 geometry and accumulation);
* energies to 1e-11 relative and forces to 1e-9 eV/A with every term in FP64;
* wrapped positions (the reference mutates them in place) to 1e-12 A.
"""
import glob
import os

import numpy as np
import pytest

import oracle
from akmc_b200 import configs as cf
from akmc_b200 import Field, PREC_FP64, PREC_MIXED

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
E_REL = {PREC_MIXED: 1e-6, PREC_FP64: 1e-11}
F_ABS = {PREC_MIXED: 1e-5, PREC_FP64: 1e-9}


def make_field(path, lat, n, prec):
    f = Field().readPotential(str(path))
    f.setup(lat, None, n)
    f.setPrecision(prec)
    return f


@pytest.mark.parametrize("prec", [PREC_MIXED, PREC_FP64], ids=["mixed", "fp64"])
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))),
                         ids=lambda p: os.path.basename(p)[:-4])
def test_matches_reference_golden(gpu, potdir, path, prec):
    g = np.load(path)
    pot = potdir / (str(g["potential"]) + ".pot")
    f = make_field(pot, g["lat"], len(g["pos"]), prec)
    E, F, W = f.forces(g["pos"], g["labels"], g["charge"])
    ref = g["energies"].copy()
    if "embedding_pinned" in g.files and not bool(g["embedding_pinned"]):
        # a multi-species EAM: the reference's embedding energy reads a stale species label
        # (metal/Field.cpp:362-367); the FP64 oracle's, each atom's own species, stands in
        Eo, _, _, _ = oracle.eam_forces(str(pot), g["pos"], g["labels"], g["lat"])
        ref[0], ref[4] = Eo["total"], Eo["many"]
    assert abs(E["total"] - ref[0]) <= E_REL[prec] * abs(ref[0])
    for k, name in enumerate(["rcp", "real", "vdw", "many"]):
        assert abs(E[name] - ref[k + 1]) <= E_REL[prec] * abs(ref[0]), name
    assert np.abs(F - g["forces"]).max() <= F_ABS[prec]
    assert np.abs(W - g["wrapped"]).max() <= 1e-12


@pytest.mark.parametrize("prec", [PREC_MIXED, PREC_FP64], ids=["mixed", "fp64"])
def test_ionic_workload_vs_fp64_oracle(gpu, potdir, prec):
    """Rocksalt 5^3, one Schottky pair, eta = 0.3, cutoff 10 A.  With the default 1 A
    shell the reference's setup rejects this cell (cutoff + shell > L/2), and with
    `nbrlist` the reference takes a neighbour-list path whose arrays it never allocates,
    so the FP64 oracle is the check here (the 6^3 golden vectors cover the reference)."""
    s = cf.rocksalt_schottky_system(5, 4.21, 0.03, 4321)
    f = Field().readPotential(str(potdir / "ion10.pot"))
    with pytest.raises(Exception):
        f.setup(s.lat, None, s.n)          # the reference's image check, kept
    pot = potdir / "ion10_shell0.pot"
    S = oracle.ionic_setup(str(pot), s.lat)
    Eo, Fo, _ = oracle.ionic_forces(S, s.pos, s.charge, s.labels, s.lat)
    f = make_field(pot, s.lat, s.n, prec)
    assert abs(f.ewald()["eta"] - 0.3) < 1e-9
    assert f.ewald()["nk"] == S["nk"]
    E, F, _ = f.forces(s.pos, s.labels, s.charge)
    assert abs(E["total"] - Eo["total"]) <= E_REL[prec] * abs(Eo["total"])
    assert np.abs(F - Fo).max() <= F_ABS[prec]


def _rocksalt_variant(ncell, a0, drop, seed, sigma=0.03):
    """Rocksalt ncell^3 without the ions `drop` (indices of the perfect crystal), the anion
    charges scaled so that the cell stays neutral."""
    s = cf.rocksalt_schottky_system(ncell, a0, sigma, seed, remove_pair=False)
    keep = np.ones(s.n, bool)
    keep[list(drop)] = False
    lab, q = s.labels[keep], s.charge[keep].copy()
    q[lab == 1] *= q[lab == 0].sum() / -q[lab == 1].sum()
    return cf.System(pos=s.pos[keep], labels=lab, charge=q, lat=s.lat)


@pytest.mark.parametrize("case", ["below64", "odd_even"])
def test_whole_cell_sizes_vs_fp64_oracle(gpu, potdir, tmp_path, case):
    """The whole-cell kernel (every pair under the minimum image, the system staged whole in
    shared memory): odd and even atom counts, and systems of at most 64 atoms, where one CTA
    holds every atom and lanes past the end hold none."""
    if case == "below64":
        pot = tmp_path / "ion4.pot"
        cf.write_ionic_potentials(str(pot), 4.0, cf.ewald_precision_for_eta(0.8, 4.0), shell=0.0)
        ncell, drops = 2, [(), (0,), (0, 32), (0, 1, 32)]          # 64, 63, 62, 61 ions
    else:
        pot = potdir / "ion10_shell0.pot"
        ncell, drops = 5, [(), (0,), (0, 500), (0, 1, 500)]        # 1000, 999, 998, 997 ions
    for k, drop in enumerate(drops):
        s = _rocksalt_variant(ncell, 4.21, drop, 50 + k)
        S = oracle.ionic_setup(str(pot), s.lat)
        Eo, Fo, _ = oracle.ionic_forces(S, s.pos, s.charge, s.labels, s.lat)
        f = make_field(pot, s.lat, s.n, PREC_MIXED)
        E, F, _ = f.forces(s.pos, s.labels, s.charge)
        assert abs(E["total"] - Eo["total"]) <= E_REL[PREC_MIXED] * abs(Eo["total"]), s.n
        assert np.abs(F - Fo).max() <= F_ABS[PREC_MIXED], s.n


def test_whole_cell_ragged_batch_and_largest_system(gpu, potdir, tmp_path):
    """One batch of whole-cell systems of different atom counts (1000, 999, 998, 997: the
    kernel's grid is sized for the largest, CTAs past a system's end return), and a system at
    the whole-cell limit (rocksalt 8^3 = 4096 ions with a 12 A cutoff: two cells per side),
    each against the FP64 oracle."""
    import torch
    pot = potdir / "ion10_shell0.pot"
    systems = [_rocksalt_variant(5, 4.21, drop, 60 + k) for k, drop in enumerate([(), (0,), (0, 500), (0, 1, 500)])]
    f = make_field(pot, systems[0].lat, 1000, PREC_MIXED)
    b = f.batch([s.n for s in systems], np.array([s.box for s in systems]),
                np.concatenate([s.labels for s in systems]), np.concatenate([s.charge for s in systems]))
    pos = torch.tensor(np.concatenate([s.pos for s in systems]), device=gpu)
    force, energy, status = b.alloc()
    b.forces_(pos, force, energy, status)
    torch.cuda.synchronize()
    assert (status.cpu().numpy() == 0).all()
    F, E = force.cpu().numpy(), energy.cpu().numpy()
    S = oracle.ionic_setup(str(pot), systems[0].lat)
    for k, s in enumerate(systems):
        Eo, Fo, _ = oracle.ionic_forces(S, s.pos, s.charge, s.labels, s.lat)
        sl = slice(b.offsets[k], b.offsets[k + 1])
        assert abs(E[k, 0] - Eo["total"]) <= E_REL[PREC_MIXED] * abs(Eo["total"]), s.n
        assert np.abs(F[sl] - Fo).max() <= F_ABS[PREC_MIXED], s.n
    pot12 = tmp_path / "ion12.pot"
    cf.write_ionic_potentials(str(pot12), 12.0, cf.ewald_precision_for_eta(0.27, 12.0), shell=0.0)
    s = cf.rocksalt_schottky_system(8, 4.21, 0.03, 77, remove_pair=False)
    assert s.n == 4096
    f = make_field(pot12, s.lat, s.n, PREC_MIXED)
    E, F, _ = f.forces(s.pos, s.labels, s.charge)
    S = oracle.ionic_setup(str(pot12), s.lat)
    Eo, Fo, _ = oracle.ionic_forces(S, s.pos, s.charge, s.labels, s.lat)
    assert abs(E["total"] - Eo["total"]) <= E_REL[PREC_MIXED] * abs(Eo["total"])
    assert np.abs(F - Fo).max() <= F_ABS[PREC_MIXED]


@pytest.mark.parametrize("prec", [PREC_MIXED, PREC_FP64], ids=["mixed", "fp64"])
def test_ionic_cell_list_path_vs_fp64_oracle(gpu, potdir, prec):
    """Ionic systems the whole-cell kernel does not take: rocksalt 8^3 (4096 ions) at an 8 A
    cutoff (four cells per side) and rocksalt 9^3 (5832 ions, above the whole-cell limit) at
    10 A (three cells per side), through the cell-list ionic pass, against the FP64 oracle."""
    for ncell, pot in ((8, "ion8_shell0"), (9, "ion10_shell0")):
        s = cf.rocksalt_schottky_system(ncell, 4.21, 0.03, 90 + ncell)
        S = oracle.ionic_setup(str(potdir / (pot + ".pot")), s.lat)
        Eo, Fo, _ = oracle.ionic_forces(S, s.pos, s.charge, s.labels, s.lat)
        f = make_field(potdir / (pot + ".pot"), s.lat, s.n, prec)
        E, F, _ = f.forces(s.pos, s.labels, s.charge)
        assert abs(E["total"] - Eo["total"]) <= E_REL[prec] * abs(Eo["total"]), ncell
        for name in ("rcp", "real", "vdw"):
            assert abs(E[name] - Eo[name]) <= E_REL[prec] * abs(Eo["total"]), (ncell, name)
        assert np.abs(F - Fo).max() <= F_ABS[prec], ncell


def test_batch_of_uneven_systems(gpu, potdir):
    import torch
    systems = cf.uneven_fcc_batch(12, sizes=(4, 6, 8), seed=5)
    f = Field().readPotential(str(potdir / "eam.pot"))
    f.setup(systems[0].lat, None, 10)
    nat = [s.n for s in systems]
    boxes = np.array([s.box for s in systems])
    lab = np.concatenate([s.labels for s in systems])
    b = f.batch(nat, boxes, lab)
    pos = torch.tensor(np.concatenate([s.pos for s in systems]), device=gpu)
    force, energy, status = b.alloc()
    b.forces_(pos, force, energy, status)
    torch.cuda.synchronize()
    F = force.cpu().numpy()
    E = energy.cpu().numpy()
    assert (status.cpu().numpy() == 0).all()
    for k, s in enumerate(systems):
        Eo, Fo, _, _ = oracle.eam_forces(str(potdir / "eam.pot"), s.pos, s.labels, s.lat)
        sl = slice(b.offsets[k], b.offsets[k + 1])
        assert abs(E[k, 0] - Eo["total"]) <= 1e-6 * abs(Eo["total"])
        assert np.abs(F[sl] - Fo).max() <= 1e-5


def test_neighbour_sets_match_brute_force(gpu, potdir):
    """The cell list's neighbour sets equal the reference criterion (j != i, minimum
    image, rsq <= rc^2; NbrListPBC.cpp:41-125) evaluated by brute force in FP64, atom by
    atom, for cells that need the per-pair minimum image (4^3: 2 cells per side) and cells
    that use shifted neighbour cells (6^3, 8^3)."""
    import torch
    systems = [cf.fcc_vacancy_system(4, 3.615, 1, 0.05, 21),
               cf.fcc_vacancy_system(6, 3.615, 3, 0.05, 22),
               cf.fcc_vacancy_system(8, 3.615, 2, 0.05, 23)]
    f = Field().readPotential(str(potdir / "eam.pot"))
    f.setup(systems[0].lat, None, 10)
    b = f.batch([s.n for s in systems], np.array([s.box for s in systems]),
                np.concatenate([s.labels for s in systems]))
    pos = torch.tensor(np.concatenate([s.pos for s in systems]), device=gpu)
    force, energy, status = b.alloc()
    b.forces_(pos, force, energy, status)
    torch.cuda.synchronize()
    counts, rows = b.neighbours(128)
    flips = 0
    for k, s in enumerate(systems):
        off, nbr = oracle.neighbour_list(s.pos, s.lat, 5.0)
        a0 = b.offsets[k]
        for i in range(s.n):
            ref = nbr[off[i]:off[i + 1]]
            got = rows[a0 + i, :counts[a0 + i]] - a0
            if not np.array_equal(np.sort(ref), got):
                flips += 1
    assert flips == 0


def test_bitwise_deterministic(gpu, potdir):
    import torch
    s = cf.rocksalt_schottky_system(6, 4.21, 0.03, 8)
    f = make_field(potdir / "ion10.pot", s.lat, s.n, PREC_MIXED)
    b = f.batch([s.n] * 3, np.array([s.box] * 3), np.tile(s.labels, 3), np.tile(s.charge, 3))
    base = torch.tensor(np.tile(s.pos, (3, 1)), device=gpu)
    outs = []
    for _ in range(3):
        force, energy, status = b.alloc()
        b.forces_(base.clone(), force, energy, status)
        torch.cuda.synchronize()
        outs.append((force.cpu().numpy(), energy.cpu().numpy()))
    for F, E in outs[1:]:
        assert np.array_equal(F, outs[0][0]) and np.array_equal(E, outs[0][1])
    # the three identical systems of one batch agree bitwise too
    F = outs[0][0].reshape(3, s.n, 3)
    assert np.array_equal(F[0], F[1]) and np.array_equal(F[0], F[2])


def test_nan_position_sets_status(gpu, potdir):
    s = cf.fcc_vacancy_system(4, 3.615, 1, 0.02, 3)
    f = make_field(potdir / "eam.pot", s.lat, s.n, PREC_MIXED)
    pos = s.pos.copy()
    pos[7, 1] = np.nan
    from akmc_b200 import AkmcError, STATUS
    with pytest.raises(AkmcError) as e:
        f.forces(pos, s.labels)
    assert e.value.code == STATUS["ERR_NONFINITE"]
    # the field stays usable after the error
    E, F, _ = f.forces(s.pos, s.labels)
    assert np.isfinite(F).all()


def test_embedding_range_error(gpu, potdir):
    """A crystal compressed until rho leaves the embedding table: the reference exits
    (ManyBody.cpp:603-608); here the call reports ERR_EMBED_RANGE and returns."""
    s = cf.fcc_vacancy_system(6, 1.70, 1, 0.0, 3)     # a0 1.7 A, L 10.2 A: rho >> 50
    f = make_field(potdir / "eam.pot", s.lat, s.n, PREC_MIXED)
    from akmc_b200 import AkmcError, STATUS
    with pytest.raises(AkmcError) as e:
        f.forces(s.pos, s.labels)
    assert e.value.code == STATUS["ERR_EMBED_RANGE"]
