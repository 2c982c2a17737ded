"""The reference's configuration and restart formats (Basis::inputBasis, Basis::dumpBasis,
Common/Basis.cpp:356-649): the reference's own example file, and dump/read round trips."""
import io
import os

import numpy as np
import pytest

from akmc_b200 import basis
from akmc_b200 import configs as cf

import oracle

GDC = os.path.join(oracle.REFERENCE, "docs", "examples", "gdc", "basis")


@pytest.mark.skipif(not os.path.exists(GDC), reason="reference tree absent")
def test_reads_the_reference_example():
    s = basis.read_basis(GDC, ["O", "Ce", "Gd"], [-2.0, 4.0, 3.0])
    assert s.n == 2549
    assert s.meta["iteration"] == 1 and s.meta["time"] == 0.0
    assert s.meta["energy"] == -87780.5106508483
    assert np.allclose(s.lat, [32.7232154959, 0, 0, 0, 32.7232154959, 0, 0, 0, 32.7232154959])
    assert np.allclose(s.pos[0], [1.4168603868, 1.3899782202, 1.3108695097])
    assert s.labels[0] == 0 and s.charge[0] == -2.0
    assert set(np.unique(s.labels)) <= {0, 1, 2}


def test_dump_round_trip_and_last_block(tmp_path):
    s = cf.rocksalt_schottky_system(3, seed=2)
    names = ["Mg", "O"]
    buf = io.StringIO()
    basis.dump(buf, s, names, 1.5e13, -123.456, 7, title="test")
    s2 = cf.System(pos=s.pos + 0.1, labels=s.labels, charge=s.charge, lat=s.lat)
    basis.dump(buf, s2, names, 3.0e13, -120.0, 8, header=False)
    path = str(tmp_path / "roundtrip")
    with open(path, "w") as f:
        f.write(buf.getvalue())
    a = basis.read_basis(path, names, [2.0, -2.0])
    assert a.meta["title"] == "test" and a.meta["iteration"] == 7
    assert np.abs(a.pos - s.pos).max() < 1e-10
    assert np.array_equal(a.labels, s.labels)
    z = basis.read_last(path, names)
    assert z.meta["iteration"] == 8 and z.meta["time"] == 3.0e13 and z.meta["energy"] == -120.0
    assert np.abs(z.pos - s2.pos).max() < 1e-10


def test_unknown_species_is_an_error(tmp_path):
    s = cf.fcc_vacancy_system(2, sigma=0.0)
    buf = io.StringIO()
    basis.dump(buf, s, ["Cu"], 0.0, 0.0, 0)
    path = str(tmp_path / "unknown")
    with open(path, "w") as f:
        f.write(buf.getvalue())
    with pytest.raises(basis.BasisError):
        basis.read_basis(path, ["Ni"])


def test_reads_velocity_and_force_lines(tmp_path):
    text = "t\n2 3 2\n5.0 0 0\n0 5.0 0\n0 0 5.0\nA 1\n1 2 3\n0 0 0\n9 9 9\nB 2\n4 5 6\n0 0 0\n9 9 9\n"
    path = str(tmp_path / "levcfg")
    with open(path, "w") as f:
        f.write(text)
    s = basis.read_basis(path, ["A", "B"])
    assert np.array_equal(s.pos, [[1, 2, 3], [4, 5, 6]]) and list(s.labels) == [0, 1]
