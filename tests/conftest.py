import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def potdir(tmp_path_factory):
    """Potential files of the workloads, written once per session."""
    from akmc_b200 import configs as cf
    d = tmp_path_factory.mktemp("potentials")
    cf.write_setfl(str(d / "fs.setfl"))
    cf.write_eam_potentials(str(d / "eam.pot"), str(d / "fs.setfl"))
    # ionic: Ewald eta = 0.3 at the 10 A cutoff (config 1), and the reference-runnable
    # variant at 9.5 A with precis 3.9e-6
    cf.write_ionic_potentials(str(d / "ion10.pot"), 10.0, cf.ewald_precision_for_eta(0.3, 10.0))
    cf.write_ionic_potentials(str(d / "ion10_shell0.pot"), 10.0,
                              cf.ewald_precision_for_eta(0.3, 10.0), shell=0.0)
    cf.write_ionic_potentials(str(d / "ion95.pot"), 9.5, 3.9e-6)
    # small rocksalt cells (4^3, L = 16.84 A) for the walker tests: 8 A cutoff, eta 0.35
    cf.write_ionic_potentials(str(d / "ion8_shell0.pot"), 8.0,
                              cf.ewald_precision_for_eta(0.35, 8.0), shell=0.0)
    # a two-species EAM with one table per species pair (the golden alloy case)
    cf.write_eam_alloy_potentials(str(d / "eam_alloy.pot"), str(d))
    # three ionic species, default Ewald precision, unlisted cation-cation pairs
    cf.write_fluorite_potentials(str(d / "fluorite.pot"), 7.0)
    return d


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from akmc_b200 import build
    build.build()
    return torch.device("cuda:0")
