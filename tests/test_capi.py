"""C-ABI library checks that need no GPU: it loads, exports every entry point that
include/akmc.h declares, and its potentials reader (pure host code) follows the
reference's keyword rules."""
import ctypes as C
import os
import re

import pytest

from akmc_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "akmc.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(akmc_[a-z_0-9]+)\s*\(", src)))


def test_every_declared_symbol_is_exported(lib):
    syms = declared_symbols()
    assert len(syms) >= 16
    for s in syms:
        assert hasattr(lib, s), s
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(syms) <= bound


def test_version(lib):
    assert b"sm_100a" in lib.akmc_version()


def _create(lib, path):
    h = C.c_void_p()
    st = lib.akmc_field_create(str(path).encode(), C.byref(h))
    return st, h


def test_reads_eam_file(lib, potdir):
    st, h = _create(lib, potdir / "eam.pot")
    assert st == 0
    assert lib.akmc_field_family(h) == 1
    assert lib.akmc_field_num_species(h) == 1
    assert lib.akmc_field_cutoff(h) == 5.0
    name = C.create_string_buffer(16)
    m, q = C.c_double(), C.c_double()
    assert lib.akmc_field_species(h, 0, name, C.byref(m), C.byref(q)) == 0
    assert name.value == b"Cu" and abs(m.value - 63.546) < 1e-12
    lib.akmc_field_destroy(h)


def test_reads_ionic_file(lib, potdir):
    st, h = _create(lib, potdir / "ion95.pot")
    assert st == 0
    assert lib.akmc_field_family(h) == 2
    assert lib.akmc_field_num_species(h) == 2
    q = C.c_double()
    lib.akmc_field_species(h, 1, None, None, C.byref(q))
    assert q.value == -2.0
    # Ewald parameters exist only after setup
    assert lib.akmc_field_ewald(h, None, None, None) == _lib.STATUS["ERR_STATE"]
    lib.akmc_field_destroy(h)


@pytest.mark.parametrize("body,code", [
    ("cutoff 5.0\nspecies 1\nCu 63.5 0.0\nfoo 1\nclose\n", "ERR_PARSE"),
    ("cutoff 5.0\nnoimage\nspecies 1\nCu 63.5 0.0\nmanybody 1 ev\neam\nCu Cu x lammps\nclose\n",
     "ERR_UNSUPPORTED"),
    ("cutoff 9.0\nspecies 1\nO 16 -2\ntwobody 1 ev ev\nmorse\nO O 1 2 3 4\nclose\n",
     "ERR_UNSUPPORTED"),
    ("cutoff 5.0\nspecies 1\nCu 63.5 0.0\nmanybody 1 ev\neam\nCu Cu /nonexistent.setfl\nclose\n",
     "ERR_IO"),
    ("cutoff 9.0\nspecies 1\nO 16 -2\nmaxNbrs 40\ntwobody 1 ev ev\nbuck\nO O 1 0.2 0\nclose\n",
     "ERR_PARSE"),   # the reference never matches maxNbrs after lower-casing
])
def test_rejects_bad_files(lib, tmp_path, body, code):
    p = tmp_path / "bad.pot"
    p.write_text(body)
    st, h = _create(lib, p)
    assert st == _lib.STATUS[code], lib.akmc_last_error()
    assert not h.value


def test_missing_file(lib):
    st, h = _create(lib, "/nonexistent/potentials")
    assert st == _lib.STATUS["ERR_IO"]


def test_batch_before_setup_is_state_error(lib, potdir):
    st, h = _create(lib, potdir / "eam.pot")
    n = (C.c_int * 1)(10)
    box = (C.c_double * 3)(10.0, 10.0, 10.0)
    lab = (C.c_int * 10)()
    b = C.c_void_p()
    assert lib.akmc_batch_create(h, 1, n, box, lab, None, C.byref(b)) == _lib.STATUS["ERR_STATE"]
    lib.akmc_field_destroy(h)


def test_checks_build_exports_and_reports(lib):
    """The default library compiles the kernel index checks away and says so; the
    self-checking build (build --checks) exports the same C ABI with the checks on."""
    assert lib.akmc_checks_enabled() == 0
    hits = (C.c_int * (32 * 3))()
    first = (C.c_int * (32 * 3))()
    assert lib.akmc_checks_read(hits, first, 0) == 7          # AKMC_ERR_UNSUPPORTED
    path = build.build(checks=True)
    chk = C.CDLL(path)
    assert chk.akmc_checks_enabled() == 1
    for s in declared_symbols():
        assert hasattr(chk, s), s
