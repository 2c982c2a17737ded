"""Walkers over local regions (akmc_b200.configs.local_region), checked on the CPU with the
FP64 oracle: moving free atoms changes the region's energy exactly as it changes the
crystal's, and the free atoms' forces are the crystal's."""
import numpy as np

from akmc_b200 import configs as cf
from oracle import walkers as W


def test_region_energy_differences_and_forces_are_the_crystals(potdir):
    s = cf.fcc_vacancy_system(10, seed=3)                 # 3999 atoms, L = 36.15 A
    site = cf.fcc_sites(10, 3.615)[s.meta["vacancies"][0]]
    reg = cf.local_region(s.pos, s.labels, s.charge, s.box, site, 6.0, 5.0)
    assert reg.system.n < s.n // 2
    assert set(np.where(reg.frozen == 0)[0]) <= set(range(reg.system.n))
    full = W.EamOracle(str(potdir / "eam.pot"), s.lat, s.labels)
    part = W.EamOracle(str(potdir / "eam.pot"), reg.system.lat, reg.system.labels)
    F0, E0, _ = full(s.pos)
    f0, e0, _ = part(reg.system.pos)
    free = np.where(reg.frozen == 0)[0]
    assert np.abs(f0[free] - F0[reg.index[free]]).max() < 1e-9
    rng = np.random.default_rng(0)
    d = np.zeros_like(reg.system.pos)
    d[free] = rng.normal(0.0, 0.15, (len(free), 3))      # free atoms only, well under the margin
    x_full = s.pos.copy()
    x_full[reg.index] += d
    F1, E1, _ = full(x_full)
    f1, e1, _ = part(reg.system.pos + d)
    assert abs((e1 - e0) - (E1 - E0)) < 1e-9
    assert np.abs(f1[free] - F1[reg.index[free]]).max() < 1e-9
    # back to crystal coordinates
    back = reg.system.pos - reg.shift
    dd = back - s.pos[reg.index]
    dd -= s.box * np.rint(dd / s.box)
    assert np.abs(dd).max() < 1e-9
