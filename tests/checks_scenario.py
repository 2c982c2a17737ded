"""Run by tests/test_gpu_checks.py in a child process whose AKMC_LIB is the self-checking
library (libakmc_b200_checks.so): the call paths whose indices the checks cover, then the
hit counts of every check as one JSON line.  Not collected by pytest (test infrastructure)."""
import ctypes as C
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    import torch
    from akmc_b200 import Field, PREC_MIXED, _lib
    from akmc_b200 import configs as cf
    from akmc_b200.walkers import Walkers, dimer_params, fire_params
    lib = _lib.load()
    assert lib.akmc_checks_enabled() == 1, _lib.LIB_PATH
    d = tempfile.mkdtemp()
    cf.write_setfl(os.path.join(d, "fs.setfl"))
    cf.write_eam_potentials(os.path.join(d, "eam.pot"), os.path.join(d, "fs.setfl"))
    cf.write_ionic_potentials(os.path.join(d, "ion.pot"), 10.0, cf.ewald_precision_for_eta(0.3, 10.0), shell=0.0)
    out = {}
    # 1. uneven EAM walkers (4^3 and 6^3 cells): FIRE, then the Dimer on the three-image batch
    #    with neighbour-list reuse and work queues
    big = cf.fcc_vacancy_system(6)
    f = Field().readPotential(os.path.join(d, "eam.pot")).setup(big.lat, None, big.n)
    f.setPrecision(PREC_MIXED)
    rng = np.random.default_rng(1)
    systems = [cf.fcc_vacancy_system(int(rng.choice([4, 6])), n_vacancies=1, seed=int(rng.integers(1 << 30)),
                                     vacancy_sites=[int(rng.integers(256))]) for _ in range(96)]
    w = Walkers.from_systems(f, systems)
    x = torch.tensor(np.concatenate([s.pos for s in systems]), device="cuda")
    w.relax(x, fire_params(force_tol=1e-3))
    xm = x.cpu().numpy()
    sd = np.concatenate([cf.local_displacements(xm[w.offsets[k]:w.offsets[k + 1]], s.box,
                                                cf.fcc_sites(s.meta["ncell"], 3.615)[s.meta["vacancies"][0]], 1,
                                                seed=1000 + k)[0] for k, s in enumerate(systems)])
    res = w.dimer(torch.tensor(xm + sd, device="cuda"), torch.tensor(sd, device="cuda"),
                  dimer_params(delta=0.005, rot_tol=0.1, max_iter=200))
    out["dimer_converged"] = int((res["status"] == 1).sum())
    w.close()
    # 2. the ionic workload through the whole-cell kernel (16 x 998 ions) and the cell-list
    #    pass (8^3 rocksalt cells, L = 33.7 A: three cells per dimension)
    for ncell, nsys in ((5, 16), (8, 2)):
        sys_ = [cf.rocksalt_schottky_system(ncell, seed=40 + k) for k in range(nsys)]
        fi = Field().readPotential(os.path.join(d, "ion.pot")).setup(sys_[0].lat, None, sys_[0].n)
        b = fi.batch([s.n for s in sys_], np.array([s.box for s in sys_]), np.concatenate([s.labels for s in sys_]),
                     np.concatenate([s.charge for s in sys_]))
        pos = torch.tensor(np.concatenate([s.pos for s in sys_]), device="cuda")
        force, energy, status = b.alloc("cuda")
        b.forces_(pos, force, energy, status)
        torch.cuda.synchronize()
        out[f"ionic_{ncell}_status"] = int(status.max().item())
        b.close()
    hits = (C.c_int * (32 * 3))()
    first = (C.c_int * (32 * 3))()
    assert lib.akmc_checks_read(hits, first, 1) == 0
    out["hits"] = list(hits)
    out["first"] = list(first)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
