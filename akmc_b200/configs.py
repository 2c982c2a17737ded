"""Seeded synthetic configurations and potential files for the AKMC force path.

There is no public dataset for this path; every workload is generated here from a
recorded seed.  File formats follow the reference readers exactly:

* ``potentials`` keyword files: metal ``Field::readPotential``
  (potentials/metal/Field.cpp:122-205) and pair ``Field::readPotential``
  (potentials/pair/Field.cpp:215-317), species lines per ``Species::loadSpecies``
  (potentials/Species.cpp:31-70), Buckingham entries per ``TwoBody::loadPotential``
  (potentials/pair/TwoBody.cpp:56-266), EAM entries per ``ManyBody::loadPotential``
  (potentials/metal/ManyBody.cpp:287-296).
* EAM tables in the single-element LAMMPS setfl layout read by
  ``MetalPotential::readLEAM`` (potentials/metal/MetalPotential.cpp:276-361):
  four header lines, ``Nrho drho Nr dr cutoff``, one element line, then F(rho),
  rho(r) and r*phi(r).

Lattice vectors use the reference's row layout ``lat[0:3]`` = a, ``lat[3:6]`` = b,
``lat[6:9]`` = c (Common/Basis.cpp:356-570).  Only orthorhombic cells are supported,
as in the reference's Ewald half-space weighting (potentials/pair/Ewald.cpp:304-311).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

# --------------------------------------------------------------------------------------
# Finnis-Sinclair-type EAM of the small metal workload, tabulated on the reference mesh.
# phi(r) = 0.5 exp(-9 (r/2.556 - 1)) eV, rho(r) = exp(-3 (r/2.556 - 1)),
# F(rho) = -1.2 sqrt(rho) eV; phi and rho are multiplied by a C2 quintic switch that
# takes them smoothly from 1 at r = 4.5 A to 0 at the 5.0 A cutoff.
# --------------------------------------------------------------------------------------
FS_R0 = 2.556
FS_RC = 5.0
FS_RSW = 4.5
FS_NR = 5001
FS_NRHO = 5001
FS_DRHO = 0.01


def _switch(r: np.ndarray) -> np.ndarray:
    t = np.clip((r - FS_RSW) / (FS_RC - FS_RSW), 0.0, 1.0)
    return 1.0 - t * t * t * (10.0 - 15.0 * t + 6.0 * t * t)


def fs_phi(r):
    r = np.asarray(r, dtype=np.float64)
    return 0.5 * np.exp(-9.0 * (r / FS_R0 - 1.0)) * _switch(r)


def fs_rho(r):
    r = np.asarray(r, dtype=np.float64)
    return np.exp(-3.0 * (r / FS_R0 - 1.0)) * _switch(r)


def fs_embed(rho):
    return -1.2 * np.sqrt(np.asarray(rho, dtype=np.float64))


def write_setfl(path: str, nr: int = FS_NR, nrho: int = FS_NRHO, drho: float = FS_DRHO,
                rc: float = FS_RC, element: str = "Cu", mass: float = 63.546,
                a0: float = 3.615, scale=(1.0, 1.0, 1.0)) -> None:
    """Write the tabulated FS-type EAM in the setfl layout the reference reads; ``scale``
    multiplies its F, rho and r*phi tables (distinct tables for the entries of an alloy)."""
    dr = rc / (nr - 1)
    r = np.arange(nr, dtype=np.float64) * dr
    rh = np.arange(nrho, dtype=np.float64) * drho
    F = scale[0] * fs_embed(rh)
    rho = scale[1] * fs_rho(r)
    rphi = scale[2] * r * fs_phi(r)
    with open(path, "w") as f:
        f.write("Finnis-Sinclair-type EAM, tabulated by akmc_b200.configs\n")
        f.write("phi=0.5exp(-9(r/2.556-1)) rho=exp(-3(r/2.556-1)) F=-1.2sqrt(rho)\n")
        f.write("quintic switch 4.5-5.0 A\n")
        f.write(f"1 {element}\n")
        f.write(f"{nrho} {drho:.17g} {nr} {dr:.17g} {rc:.17g}\n")
        f.write(f"29 {mass} {a0} fcc\n")
        for arr in (F, rho, rphi):
            for k in range(0, len(arr), 5):
                f.write(" ".join(f"{v:.17e}" for v in arr[k:k + 5]) + "\n")


def write_eam_potentials(path: str, setfl_path: str, cutoff: float = FS_RC,
                         element: str = "Cu", mass: float = 63.546) -> None:
    """``potentials`` file for the metal Field: one species, one EAM entry."""
    with open(path, "w") as f:
        f.write(f"cutoff {cutoff}\n")
        f.write("species 1\n")
        f.write(f"{element} {mass} 0.0\n")
        f.write("manybody 1 ev\n")
        f.write("eam\n")
        f.write(f"{element} {element} {os.path.abspath(setfl_path)} lammps\n")
        f.write("close\n")


ALLOY_SCALES = {("Cu", "Cu"): (1.0, 1.0, 1.0), ("Ni", "Ni"): (1.15, 0.9, 1.1), ("Cu", "Ni"): (1.05, 0.95, 0.9)}


def write_eam_alloy_potentials(path: str, d: str, cutoff: float = FS_RC) -> None:
    """``potentials`` file of a two-species EAM (Cu, label 0; Ni, label 1) with one setfl
    table per species pair, each the FS-type table scaled by ALLOY_SCALES and written into
    directory d: the reference takes a neighbour's density from its own species' table, an
    atom's embedding from its own, and a pair's terms from the pair's (ManyBody.cpp:937-1000)."""
    with open(path, "w") as f:
        f.write(f"cutoff {cutoff}\n")
        f.write("species 2\n")
        f.write("Cu 63.546 0.0\n")
        f.write("Ni 58.693 0.0\n")
        f.write(f"manybody {len(ALLOY_SCALES)} ev\n")
        for (a, b), sc in ALLOY_SCALES.items():
            fn = os.path.join(os.path.abspath(d), f"alloy_{a}{b}.setfl")
            write_setfl(fn, element=a, scale=sc)
            f.write("eam\n")
            f.write(f"{a} {b} {fn} lammps\n")
        f.write("close\n")


def fcc_alloy_system(ncell: int = 4, a0: float = 3.615, fraction: float = 0.3, sigma: float = 0.02,
                     seed: int = 11) -> System:
    """FCC with one vacancy, a seeded random fraction of the atoms species 1 (the alloy)."""
    s = fcc_vacancy_system(ncell, a0, 1, sigma, seed)
    rng = np.random.default_rng(seed + 1)
    lab = (rng.random(s.n) < fraction).astype(np.int32)
    return System(pos=s.pos, labels=lab, charge=np.zeros(s.n), lat=s.lat,
                  meta=dict(s.meta, kind="fcc alloy", fraction=fraction))


# --------------------------------------------------------------------------------------
# Rocksalt oxide with Buckingham + Ewald.
# --------------------------------------------------------------------------------------
BUCK_MGO = (1284.4, 0.2997, 0.0)
BUCK_OO = (22764.0, 0.149, 27.88)
BUCK_MGMG = (0.0, 1.0, 0.0)   # listed explicitly: an unlisted pair would fall back to pot 0


def ewald_eta_from_precision(precis: float, rc: float) -> float:
    """eta as the reference derives it from ``ewald precis`` (pair/Field.cpp:129-133)."""
    eps = min(abs(precis), 0.5)
    tol = math.sqrt(abs(math.log(eps * rc)))
    return math.sqrt(abs(math.log(eps * rc * tol))) / rc


def ewald_precision_for_eta(eta: float, rc: float) -> float:
    """Inverse of :func:`ewald_eta_from_precision` (bisection in log space)."""
    lo, hi = math.log(1e-30), math.log(0.5 / max(rc, 1.0))
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if ewald_eta_from_precision(math.exp(mid), rc) > eta:
            lo = mid          # smaller precis -> larger eta
        else:
            hi = mid
    return math.exp(0.5 * (lo + hi))


def write_ionic_potentials(path: str, cutoff: float, precis: float,
                           q_cat: float = 2.0, q_an: float = -2.0, shell=None) -> None:
    """``potentials`` file for the pair Field: Mg/O, three Buckingham entries, Ewald.

    ``shell`` writes an ``nbrlist <shell>`` line.  The pair Field checks
    cutoff + shell <= L/2 with a 1.0 A default shell (pair/Field.cpp:98-107,
    pair/Field.h:66); the 10 A cutoff of the rocksalt 5x5x5 workload (L = 21.05 A) only
    passes with an explicit ``nbrlist 0.0``."""
    with open(path, "w") as f:
        f.write(f"cutoff {cutoff}\n")
        if shell is not None:
            f.write(f"nbrlist {shell}\n")
        f.write("species 2\n")
        f.write(f"Mg 24.305 {q_cat}\n")
        f.write(f"O 15.999 {q_an}\n")
        f.write("twobody 3 ev ev\n")
        for (a, b), (A, rho, C) in ((("Mg", "O"), BUCK_MGO), (("O", "O"), BUCK_OO),
                                    (("Mg", "Mg"), BUCK_MGMG)):
            f.write("buck\n")
            f.write(f"{a} {b} {A!r} {rho!r} {C!r}\n")
        f.write(f"ewald precis {precis!r}\n")
        f.write("close\n")


# --------------------------------------------------------------------------------------
# Lattices.
# --------------------------------------------------------------------------------------
@dataclass
class System:
    """One periodic system in the reference's SoA layout."""
    pos: np.ndarray            # (N, 3) float64, Angstrom
    labels: np.ndarray         # (N,) int32 species index (atmLabel)
    charge: np.ndarray         # (N,) float64 per-atom charge (Basis::charge)
    lat: np.ndarray            # (9,) float64 lattice vectors, rows a, b, c
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    @property
    def box(self) -> np.ndarray:
        return np.array([self.lat[0], self.lat[4], self.lat[8]])


def cubic_lat(L: float) -> np.ndarray:
    return np.array([L, 0, 0, 0, L, 0, 0, 0, L], dtype=np.float64)


def fcc_sites(ncell: int, a0: float) -> np.ndarray:
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(np.arange(ncell), np.arange(ncell), np.arange(ncell),
                             indexing="ij"), -1).reshape(-1, 3)
    return ((g[:, None, :] + basis[None, :, :]).reshape(-1, 3) * a0).astype(np.float64)


def fcc_vacancy_system(ncell: int = 4, a0: float = 3.615, n_vacancies: int = 1,
                       sigma: float = 0.02, seed: int = 1234,
                       vacancy_sites=None) -> System:
    """FCC metal with vacancies and seeded Gaussian jitter (the EAM workloads)."""
    rng = np.random.default_rng(seed)
    sites = fcc_sites(ncell, a0)
    if vacancy_sites is None:
        vacancy_sites = [0] if n_vacancies == 1 else \
            list(rng.choice(len(sites), size=n_vacancies, replace=False))
    keep = np.ones(len(sites), dtype=bool)
    keep[np.asarray(vacancy_sites, dtype=np.int64)] = False
    pos = sites[keep] + rng.normal(0.0, sigma, size=(int(keep.sum()), 3))
    n = pos.shape[0]
    return System(pos=pos, labels=np.zeros(n, np.int32), charge=np.zeros(n),
                  lat=cubic_lat(ncell * a0),
                  meta=dict(kind="fcc", ncell=ncell, a0=a0, vacancies=list(map(int, vacancy_sites)),
                            sigma=sigma, seed=seed))


def rocksalt_schottky_system(ncell: int = 5, a0: float = 4.21, sigma: float = 0.03,
                             seed: int = 4321, q_cat: float = 2.0, q_an: float = -2.0,
                             remove_pair: bool = True) -> System:
    """Rocksalt oxide (label 0 = cation Mg, 1 = anion O) with one Schottky pair removed:
    the cation at the origin and its nearest anion at (a0/2, 0, 0)."""
    rng = np.random.default_rng(seed)
    cat = fcc_sites(ncell, a0)
    an = cat + np.array([0.5 * a0, 0.0, 0.0])
    L = ncell * a0
    an = np.mod(an, L)
    pos = np.concatenate([cat, an])
    lab = np.concatenate([np.zeros(len(cat), np.int32), np.ones(len(an), np.int32)])
    if remove_pair:
        keep = np.ones(len(pos), bool)
        keep[0] = False                   # cation at the origin
        keep[len(cat)] = False            # anion at (a0/2, 0, 0)
        pos, lab = pos[keep], lab[keep]
    pos = pos + rng.normal(0.0, sigma, size=pos.shape)
    q = np.where(lab == 0, q_cat, q_an).astype(np.float64)
    return System(pos=pos, labels=lab.astype(np.int32), charge=q, lat=cubic_lat(L),
                  meta=dict(kind="rocksalt", ncell=ncell, a0=a0, sigma=sigma, seed=seed))


def doped_fluorite_system(ncell: int = 3, a0: float = 5.41, n_dopant_pairs: int = 1, sigma: float = 0.03,
                          seed: int = 31) -> System:
    """Fluorite dioxide with a trivalent dopant, three species: label 0 = anion (-2),
    1 = dopant cation (+3), 2 = host cation (+4).  Cations on the FCC sites, anions on the
    simple-cubic sublattice at (a0/4)(1, 1, 1) + a0/2 steps; each dopant pair replaces two host
    cations and removes one anion (the cell stays neutral).  Seeded choices and jitter."""
    rng = np.random.default_rng(seed)
    cat = fcc_sites(ncell, a0)
    g = np.stack(np.meshgrid(*[np.arange(2 * ncell)] * 3, indexing="ij"), -1).reshape(-1, 3)
    an = (g + 0.5) * (0.5 * a0)
    lab_c = np.full(len(cat), 2, np.int32)
    lab_c[rng.choice(len(cat), size=2 * n_dopant_pairs, replace=False)] = 1
    keep = np.ones(len(an), bool)
    keep[rng.choice(len(an), size=n_dopant_pairs, replace=False)] = False
    pos = np.concatenate([cat, an[keep]])
    lab = np.concatenate([lab_c, np.zeros(int(keep.sum()), np.int32)])
    pos = pos + rng.normal(0.0, sigma, size=pos.shape)
    q = np.choose(lab, [-2.0, 3.0, 4.0]).astype(np.float64)
    return System(pos=pos, labels=lab, charge=q, lat=cubic_lat(ncell * a0),
                  meta=dict(kind="fluorite", ncell=ncell, a0=a0, sigma=sigma, seed=seed))


def write_fluorite_potentials(path: str, cutoff: float = 7.0) -> None:
    """``potentials`` file for :func:`doped_fluorite_system`: three species, Buckingham for
    the two cation-anion pairs and the anion-anion pair only, no ``ewald`` line.  The
    reference then takes its default Ewald precision (madelungAcc 1e-6, pair/Field.h:54), and
    every cation-cation pair falls back to potential 0, the first entry (TwoBody.cpp:509)."""
    with open(path, "w") as f:
        f.write(f"cutoff {cutoff}\nspecies 3\nOx 16.0 -2.0\nDp 150.0 3.0\nHc 140.0 4.0\n")
        f.write("twobody 3 ev ev\n")
        for a, b, A, rho, C in (("Dp", "Ox", 1750.0, 0.345, 18.0), ("Hc", "Ox", 1650.0, 0.36, 16.0),
                                ("Ox", "Ox", 9000.0, 0.225, 30.0)):
            f.write(f"buck\n{a} {b} {A!r} {rho!r} {C!r}\n")
        f.write("close\n")


def vacancy_hop_starts(pos: np.ndarray, box, site, amplitude: float = 0.9, k: int = 4,
                       noise: float = 0.02, seed: int = 0) -> list:
    """Starting displacements inside the negative-curvature region of vacancy hops: for up to
    k nearest neighbours (closer than 2.9 A) of the vacancy at ``site``, that atom moved
    ``amplitude`` A towards the site and N(0, noise) on the atoms within 4 A of it (minimum
    image).  Returns a list of (N, 3) arrays."""
    box = np.asarray(box, dtype=np.float64)
    rng = np.random.default_rng(seed)
    dv = np.asarray(site, dtype=np.float64) - pos
    dv -= box * np.rint(dv / box)
    r = np.sqrt((dv * dv).sum(1))
    out = []
    for i in np.where(r < 2.9)[0][:k]:
        d = pos - pos[i]
        d -= box * np.rint(d / box)
        near = np.sqrt((d * d).sum(1)) < 4.0
        sd = np.zeros_like(pos)
        sd[near] = rng.normal(0.0, noise, (int(near.sum()), 3))
        sd[i] += amplitude * dv[i] / r[i]
        out.append(sd)
    return out


def rocksalt_hop_starts(pos: np.ndarray, labels, box, a0: float = 4.21, amplitude: float = 1.0,
                        per_site: int = 8, noise: float = 0.02, seed: int = 0) -> list:
    """Starting displacements of the ionic configuration's searches: for each vacancy of
    rocksalt_schottky_system -- the cation site at the origin and the anion site at
    (a0/2, 0, 0) -- up to ``per_site`` same-species nearest neighbours (a0/sqrt(2) away)
    moved ``amplitude`` A towards the vacancy, and N(0, noise) on the atoms within 4 A of the
    moving one (minimum image).  Returns a list of (N, 3) arrays, cation hops first."""
    box = np.asarray(box, dtype=np.float64)
    labels = np.asarray(labels)
    rng = np.random.default_rng(seed)
    out = []
    for species, site in ((0, (0.0, 0.0, 0.0)), (1, (0.5 * a0, 0.0, 0.0))):
        dv = np.asarray(site, dtype=np.float64) - pos
        dv -= box * np.rint(dv / box)
        r = np.sqrt((dv * dv).sum(1))
        cand = np.where((labels == species) & (r < 0.5 * a0 * np.sqrt(2.0) + 0.3))[0]
        cand = cand[np.argsort(r[cand], kind="stable")][:per_site]
        for i in cand:
            d = pos - pos[i]
            d -= box * np.rint(d / box)
            near = np.sqrt((d * d).sum(1)) < 4.0
            sd = np.zeros_like(pos)
            sd[near] = rng.normal(0.0, noise, (int(near.sum()), 3))
            sd[i] += amplitude * dv[i] / r[i]
            out.append(sd)
    return out


@dataclass
class LocalRegion:
    """A walker's local region cut out of a periodic crystal (see local_region)."""
    system: System                # the cut-out atoms in their own isolated cell
    index: np.ndarray             # their indices in the crystal
    frozen: np.ndarray            # 1 for the atoms outside the active radius
    shift: np.ndarray             # crystal position = region position - shift (then wrapped); the centre sits at 0


def local_region(pos: np.ndarray, labels, charge, box, centre, active_radius: float, cutoff: float,
                 margin: float = 1.0) -> LocalRegion:
    """The atoms of a search confined to a local region (the reference's active region,
    SaddleSearch::constructActiveRegion, optim/SaddleSearch.cpp:15-354): those within
    ``active_radius`` of ``centre`` move (the free atoms), those out to active_radius + 2
    cutoffs + margin stay fixed, and the rest of the crystal is left out.  Free atoms that
    move by less than ``margin`` interact only with atoms of the region, and every atom whose
    energy terms they change (within one cutoff) has its whole neighbourhood (a second
    cutoff) inside it; so energy differences and free-atom forces of the region equal those
    of the crystal -- for EAM, whose density reaches one cutoff and whose embedding another.
    The region sits, unwrapped around its centre, at the origin of an isolated cubic cell wide
    enough that it never meets its periodic image (2 (radius + cutoff)); wrapping into that
    cell (as every force call does) leaves it unchanged."""
    box = np.asarray(box, dtype=np.float64)
    d = pos - np.asarray(centre, dtype=np.float64)
    d -= box * np.rint(d / box)
    r = np.sqrt((d * d).sum(1))
    rs = active_radius + 2.0 * cutoff + margin
    if rs > 0.5 * box.min():
        raise ValueError("the local region is wider than half the crystal")
    idx = np.where(r <= rs)[0]
    L = 2.0 * (rs + cutoff)
    sub_pos = d[idx].copy()
    frozen = (r[idx] > active_radius).astype(np.int32)
    shift = -np.asarray(centre, dtype=np.float64)
    sub = System(pos=sub_pos, labels=np.asarray(labels)[idx].astype(np.int32),
                 charge=np.asarray(charge, dtype=np.float64)[idx], lat=cubic_lat(L),
                 meta=dict(kind="local_region", active_radius=active_radius, region_radius=rs))
    return LocalRegion(system=sub, index=idx, frozen=frozen, shift=shift)


def fcc_cluster_system(ncell: int = 20, a0: float = 3.615, cluster: int = 6, isolated: int = 10,
                       sigma: float = 0.02, seed: int = 2026) -> System:
    """FCC crystal with a compact vacancy cluster and isolated vacancies (the AKMC-loop
    configuration at scale: 20^3 cells, 32 000 sites, a 6-vacancy cluster and 10 isolated
    vacancies).  The cluster is a seeded site and its cluster - 1 nearest sites (distance,
    then site index); each isolated vacancy is a seeded site farther than 2 a0 from every
    vacancy chosen before it."""
    rng = np.random.default_rng(seed)
    sites = fcc_sites(ncell, a0)
    L = ncell * a0

    def dist(a, pts):
        d = pts - a
        d -= L * np.rint(d / L)
        return np.sqrt((d * d).sum(-1))
    c0 = int(rng.integers(len(sites)))
    dc = dist(sites[c0], sites)
    order = np.lexsort((np.arange(len(sites)), dc))
    vac = [int(i) for i in order[:cluster]]
    while len(vac) < cluster + isolated:
        k = int(rng.integers(len(sites)))
        if dist(sites[k], sites[np.asarray(vac)]).min() > 2.0 * a0:
            vac.append(k)
    s = fcc_vacancy_system(ncell, a0, sigma=sigma, seed=int(rng.integers(1 << 31)), vacancy_sites=vac)
    s.meta["cluster"] = vac[:cluster]
    return s


def uneven_fcc_batch(n_systems: int = 512, sizes=(4, 6, 8, 10), a0: float = 3.615,
                     sigma: float = 0.02, seed: int = 2024) -> list:
    """Batched walkers of uneven size: cells drawn uniformly from ``sizes``, each system
    with 1-3 random vacancies and its own jitter seed."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(n_systems):
        nc = int(rng.choice(sizes))
        nv = int(rng.integers(1, 4))
        out.append(fcc_vacancy_system(nc, a0, n_vacancies=nv, sigma=sigma,
                                      seed=int(rng.integers(0, 2**31 - 1)),
                                      vacancy_sites=None if nv > 1 else [int(rng.integers(0, 4 * nc ** 3))]))
    return out


def local_displacements(pos: np.ndarray, box, center, n_walkers: int, sigma: float = 0.1,
                        radius: float = 4.0, seed: int = 0) -> np.ndarray:
    """Dimer starting displacements of the metal workloads: Gaussian N(0, sigma) on every
    atom within ``radius`` of ``center`` (minimum image), zero elsewhere.  Returns
    (n_walkers, N, 3).  The reference's own seeding (SaddleSearch.cpp:390-415) draws
    uniform components on a chosen region; this is the workload's stated rule."""
    box = np.asarray(box, dtype=np.float64)
    d = pos - np.asarray(center, dtype=np.float64)
    d -= box * np.rint(d / box)
    near = np.where(np.sqrt((d * d).sum(1)) < radius)[0]
    rng = np.random.default_rng(seed)
    out = np.zeros((n_walkers,) + pos.shape)
    for w in range(n_walkers):
        out[w, near] = rng.normal(0.0, sigma, size=(len(near), 3))
    return out


def fcc_vacancy_finder(ncell: int, a0: float, tol: float = 1.0):
    """Seeding centres of an FCC crystal with vacancies: the lattice sites with no atom
    within ``tol`` (minimum image).  Returns a callable pos -> (k, 3).  Each atom is assigned
    to the nearest point of the half-lattice (spacing a0/2) and marks that point's site
    occupied when the point is an FCC site within ``tol`` of the atom: O(N) for the 32 000-site
    crystals of the AKMC loop."""
    sites = fcc_sites(ncell, a0)
    L = ncell * a0
    h = 0.5 * a0
    m = 2 * ncell
    # site index of half-lattice point (i, j, k) with i + j + k even, in fcc_sites order
    lut = np.full((m, m, m), -1, dtype=np.int64)
    ijk = np.rint(sites / h).astype(np.int64) % m
    lut[ijk[:, 0], ijk[:, 1], ijk[:, 2]] = np.arange(len(sites))

    def find(pos):
        pos = np.asarray(pos, dtype=np.float64)
        q = np.rint(pos / h).astype(np.int64)
        site = lut[q[:, 0] % m, q[:, 1] % m, q[:, 2] % m]
        ok = site >= 0
        d = pos[ok] - sites[site[ok]]
        d -= L * np.rint(d / L)
        hit = site[ok][(d * d).sum(1) <= tol * tol]
        occupied = np.zeros(len(sites), dtype=bool)
        occupied[hit] = True
        return sites[~occupied]
    return find
