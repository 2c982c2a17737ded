"""The C++ side of the drop-in boundary: the reference's own relaxation driver
(optim/Relax.cpp, compiled unchanged) on akmc_b200/cpp/Field.h.

CPU: the program builds and, with no GPU, fails loudly (exit 1 with the C-ABI status)
instead of falling back.  GPU: it relaxes the 255-atom vacancy workload to the minimum
the reference's FIRE reaches on the reference's own Field, within the force-path bars.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle
from akmc_b200 import configs as cf

needs_dropin = pytest.mark.skipif(not oracle.dropin_available(), reason="drop-in driver not built")


def _write_config(path, s):
    with open(path, "w") as f:
        f.write(f"{s.n}\n")
        f.write(" ".join(repr(float(v)) for v in s.lat) + "\n")
        for lab, (x, y, z) in zip(s.labels, s.pos):
            f.write(f"{int(lab)} {float(x)!r} {float(y)!r} {float(z)!r}\n")


def _read_out(path):
    with open(path) as f:
        st, e = f.readline().split()
        pos = np.loadtxt(f)
    return int(st), float(e), pos


@needs_dropin
def test_dropin_fails_loudly_without_gpu(potdir, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    s = cf.fcc_vacancy_system(4)
    _write_config(tmp_path / "cfg", s)
    r = subprocess.run([oracle.DROPIN_RELAX, str(potdir / "eam.pot"), str(tmp_path / "cfg"),
                        str(tmp_path / "out")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert "status 8" in r.stderr          # AKMC_ERR_CUDA: no device, no fallback


@needs_dropin
@pytest.mark.gpu
def test_reference_relax_on_dropin_field(gpu, potdir, tmp_path):
    s = cf.fcc_vacancy_system(4)
    _write_config(tmp_path / "cfg", s)
    r = subprocess.run([oracle.DROPIN_RELAX, str(potdir / "eam.pot"), str(tmp_path / "cfg"),
                        str(tmp_path / "out")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    st, e, x = _read_out(tmp_path / "out")
    assert st == 0                                     # Status SUCCESS
    # the reference's FIRE on the reference's own Field, from the same start
    ref = oracle.ReferenceField("eam", str(potdir / "eam.pot"), s.lat, s.n)
    rst, E, xr = ref.relax(s.pos, s.charge, s.labels)
    assert rst == 0
    assert abs(e - E["total"]) <= 1e-6 * abs(E["total"])
    d = x - xr
    d -= s.box * np.rint(d / s.box)
    assert np.abs(d).max() < 1e-3


@needs_dropin
@pytest.mark.gpu
def test_reference_relax_on_dropin_field_ionic(gpu, potdir, tmp_path):
    """Buckingham + Ewald through the same class: 30 reference FIRE steps on the 998-ion
    rocksalt follow the reference's own 30 steps on its pair Field."""
    s = cf.rocksalt_schottky_system(5, seed=4321)
    _write_config(tmp_path / "cfg", s)
    pot = str(potdir / "ion95.pot")
    r = subprocess.run([oracle.DROPIN_RELAX, pot, str(tmp_path / "cfg"), str(tmp_path / "out"),
                        "fire", "30"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    st, e, x = _read_out(tmp_path / "out")
    ref = oracle.ReferenceField("pair", pot, s.lat, s.n)
    rst, E, xr = ref.relax(s.pos, s.charge, s.labels, max_iter=30)
    assert st == rst
    assert abs(e - E["total"]) <= 1e-6 * abs(E["total"])
    d = x - xr
    d -= s.box * np.rint(d / s.box)
    assert np.abs(d).max() < 1e-5


needs_art_dropin = pytest.mark.skipif(not oracle.art_dropin_available(), reason="ART drop-in driver not built")


def _write_seed(path, d):
    np.savetxt(path, np.asarray(d, dtype=np.float64), fmt="%.17g")


@needs_art_dropin
def test_art_dropin_fails_loudly_without_gpu(potdir, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    s = cf.fcc_vacancy_system(4)
    _write_config(tmp_path / "cfg", s)
    _write_seed(tmp_path / "seed", np.zeros((s.n, 3)) + 0.01)
    r = subprocess.run([oracle.DROPIN_ART, str(potdir / "eam.pot"), str(tmp_path / "cfg"),
                        str(tmp_path / "seed"), str(tmp_path / "out")], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 1
    assert "status 8" in r.stderr          # AKMC_ERR_CUDA: no device, no fallback


@needs_art_dropin
@pytest.mark.gpu
def test_reference_art_on_dropin_field(gpu, potdir, tmp_path):
    """The reference's own saddle search (optim/ART.cpp, compiled unchanged) on the drop-in
    Field: from near-hop starts on a 4x4x4 vacancy, its saddle energies and barriers agree
    with the same ART on the reference's own Field within the 1 meV saddle bar."""
    from oracle import walkers as W
    s = cf.fcc_vacancy_system(4, sigma=0.0)
    eo = W.EamOracle(str(potdir / "eam.pot"), s.lat, s.labels)
    rr = W.fire_relax(eo, s.pos, p=W.FireParams(force_tol=1e-5, norm_tol=1e-6))
    assert rr["status"] == 1
    xmin = rr["pos"]
    starts = cf.vacancy_hop_starts(xmin, s.box, [0.0, 0.0, 0.0], k=3)
    ref = oracle.ReferenceField("eam", str(potdir / "eam.pot"), s.lat, s.n)
    e_ref_min = ref.forces(xmin, s.charge, s.labels)[0]["total"]
    from akmc_b200 import Field
    f = Field().readPotential(str(potdir / "eam.pot")).setup(s.lat, None, s.n)
    e_gpu_min = f.forces(xmin, s.labels)[0]["total"]
    m = cf.System(pos=xmin, labels=s.labels, charge=s.charge, lat=s.lat)
    _write_config(tmp_path / "cfg", m)
    for k, sd in enumerate(starts):
        _write_seed(tmp_path / f"seed{k}", sd)
        out = tmp_path / f"out{k}"
        r = subprocess.run([oracle.DROPIN_ART, str(potdir / "eam.pot"), str(tmp_path / "cfg"),
                            str(tmp_path / f"seed{k}"), str(out), "3000", "0.0005", "0.001"],
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        st, e_sad, _ = _read_out(out)
        rst, e_art, _ = ref.art(xmin, s.charge, s.labels, sd, init_dt=0.0005, max_dt=0.001, max_par_iter=3000)
        assert st == 0 and rst == 0
        assert abs(e_sad - e_art) < 1e-3
        assert abs((e_sad - e_gpu_min) - (e_art - e_ref_min)) < 1e-3
