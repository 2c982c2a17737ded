"""Generate the golden vectors of the force path from the reference's own Field.

The reference ships no tests or fixtures for this path, so its outputs are produced
here: the reference potential sources are compiled in place (oracle/Makefile ->
oracle/_ref/libref_{eam,pair}.so) and called through Field::readPotential / setup /
calculateForces exactly as the reference driver does.  Each fixture stores the inputs
(positions, labels, charges, lattice) and the reference outputs (energies, forces,
wrapped positions), so tests can check the oracle restatement and the CUDA path
without the reference tree.

    python tests/golden/make_golden.py          # needs the reference tree (this host)
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from akmc_b200 import configs as cf  # noqa: E402


def cases():
    """(name, family, potential file, system, min_dim_override, product potential file)."""
    out = []
    # EAM, the small metal workload: FCC 4x4x4, one vacancy, sigma 0.02, seed 1234
    out.append(("eam_fcc4_vac1", "eam", "eam", cf.fcc_vacancy_system(4, 3.615, 1, 0.02, 1234)))
    # ionic rocksalt 5^3, one Schottky pair, eta 0.3, cutoff 10 A: the ionic workload
    # itself.  The reference's setup guard (cutoff + 1 A shell <= L/2) rejects this cell,
    # so the harness passes a minimum dimension of 2 * (10 + 1) A to Field::setup; the
    # force loops are the reference's own.  The product reads the same potential with
    # `nbrlist 0.0` (its cell list has no Verlet shell).
    out.append(("ionic_rs5_rc10", "pair", "ion10", cf.rocksalt_schottky_system(5, 4.21, 0.03, 4321),
                22.000001, "ion10_shell0"))
    # EAM, 6x6x6 (864 sites, 2 vacancies): cell list with >= 3 cells per dimension
    out.append(("eam_fcc6_vac2", "eam", "eam",
                cf.fcc_vacancy_system(6, 3.615, 2, 0.02, 77, vacancy_sites=[0, 431])))
    # EAM, perfect crystal (known answer: zero forces)
    out.append(("eam_fcc5_perfect", "eam", "eam",
                cf.fcc_vacancy_system(5, 3.615, 1, 0.0, 5, vacancy_sites=[])))
    # ionic rocksalt 5^3 with one Schottky pair, cutoff 9.5 (the reference rejects 10 A
    # at this box size), Ewald precis 3.9e-6
    out.append(("ionic_rs5_rc95", "pair", "ion95", cf.rocksalt_schottky_system(5, 4.21, 0.03, 4321)))
    # ionic rocksalt 6^3 at the 10 A cutoff of the ionic workload, eta from precis at rc 10
    out.append(("ionic_rs6_rc10", "pair", "ion10", cf.rocksalt_schottky_system(6, 4.21, 0.03, 99)))
    # EAM alloy: two species, one table per species pair (Cu-Cu, Ni-Ni, Cu-Ni), FCC 4^3 with a
    # vacancy and 30 % of the atoms Ni.  Its forces and pair energy are pinned; its embedding
    # energy is not: the reference's embedding loop (metal/Field.cpp:362-367) reads a species
    # label left over from the loop before, which depends on the OpenMP thread count
    out.append(("eam_alloy_fcc4", "eam", "eam_alloy", cf.fcc_alloy_system(4, 3.615, 0.3, 0.02, 11)))
    # ionic, three species: doped fluorite 3^3 (323 ions, L = 16.23 A), cutoff 7 A with the
    # reference's default 1 A shell, no ewald line (default precision), cation-cation pairs
    # unlisted (potential 0 stands in for them)
    out.append(("ionic_fluorite3_rc7", "pair", "fluorite", cf.doped_fluorite_system(3, 5.41, 1, 0.03, 31)))
    return out


def write_potentials(d):
    cf.write_setfl(os.path.join(d, "fs.setfl"))
    cf.write_eam_potentials(os.path.join(d, "eam.pot"), os.path.join(d, "fs.setfl"))
    cf.write_ionic_potentials(os.path.join(d, "ion10.pot"), 10.0, cf.ewald_precision_for_eta(0.3, 10.0))
    cf.write_ionic_potentials(os.path.join(d, "ion10_shell0.pot"), 10.0,
                              cf.ewald_precision_for_eta(0.3, 10.0), shell=0.0)
    cf.write_ionic_potentials(os.path.join(d, "ion95.pot"), 9.5, 3.9e-6)
    cf.write_eam_alloy_potentials(os.path.join(d, "eam_alloy.pot"), d)
    cf.write_fluorite_potentials(os.path.join(d, "fluorite.pot"), 7.0)


def main():
    if not (oracle.reference_available("eam") and oracle.reference_available("pair")):
        oracle.build(reference=True)
    d = tempfile.mkdtemp(prefix="akmc_golden_")
    write_potentials(d)
    for case in cases():
        name, fam, pot, s = case[:4]
        override = case[4] if len(case) > 4 else 0.0
        product_pot = case[5] if len(case) > 5 else pot
        R = oracle.ReferenceField(fam, os.path.join(d, pot + ".pot"), s.lat, s.n, override)
        E, F, W = R.forces(s.pos, s.charge, s.labels)
        R.close()
        np.savez_compressed(os.path.join(HERE, name + ".npz"), pos=s.pos, labels=s.labels,
                            charge=s.charge, lat=s.lat, forces=F, wrapped=W, potential=product_pot,
                            energies=np.array([E["total"], E["rcp"], E["real"], E["vdw"], E["many"]]),
                            embedding_pinned=np.array(len(set(s.labels.tolist())) < 2 or fam != "eam"))
        print(f"{name}: N={s.n} E={E['total']:.10f} max|F|={np.abs(F).max():.6f}")


if __name__ == "__main__":
    main()
