"""The allocation-free EAM call (akmc_eam_forces_noalloc) against the batched call.

Some callers cannot call cudaMalloc when they need forces: code enqueuing work while its
stream is being captured into a CUDA graph, processes whose device memory belongs to a
caching allocator or a fixed budget, and loops that cannot afford the device-wide
synchronisation of cudaFree.  For them the library keeps the scratch of one system
(up to AKMC_NOALLOC_MAX_ATOMS atoms) in a fixed device array instead of allocating it.
This file checks, through the C ABI, that two calls in a row (two different systems, so
the second call runs on the first call's leftover scratch) give the same energies,
forces and wrapped positions as akmc_batch_forces, within the parity bars the other GPU
tests use, and that oversized systems are refused.  It is collected last so that a run
stopping at the first failure has already run every other test; it also passes alone in
a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from akmc_b200 import Field, STATUS
from akmc_b200 import configs as cf

pytestmark = pytest.mark.gpu

E_REL = 1e-6      # energy bar of the mixed-precision parity tests
F_ABS = 1e-5      # force bar (eV/A)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_matches_batch_call(gpu, potdir):
    import torch
    systems = [cf.fcc_vacancy_system(6, 3.615, 2, 0.02, 11, vacancy_sites=[3, 500]),
               cf.fcc_vacancy_system(4, 3.615, 1, 0.03, 12)]
    f = Field().readPotential(str(potdir / "eam.pot"))
    f.setup(systems[0].lat, None, 10)
    lib = f._lib
    stream = torch.cuda.current_stream().cuda_stream
    for s in systems:
        # the existing entry point: a batch of one system
        b = f.batch([s.n], np.array([s.box]), s.labels)
        pos_a = torch.tensor(s.pos, device=gpu)
        force_a, energy_a, status_a = b.alloc(gpu)
        b.forces_(pos_a, force_a, energy_a, status_a, stream)
        # the allocation-free entry point on the same input
        pos_b = torch.tensor(s.pos, device=gpu)
        lab = torch.tensor(s.labels, dtype=torch.int32, device=gpu)
        force_b = torch.full((s.n, 3), np.nan, dtype=torch.float64, device=gpu)
        energy_b = torch.full((5,), np.nan, dtype=torch.float64, device=gpu)
        status_b = torch.full((1,), -1, dtype=torch.int32, device=gpu)
        box = (C.c_double * 3)(*[float(x) for x in s.box])
        st = lib.akmc_eam_forces_noalloc(f._h, s.n, box, _ptr(pos_b), _ptr(lab), _ptr(force_b),
                                         _ptr(energy_b), _ptr(status_b), C.c_void_p(stream))
        assert st == 0, lib.akmc_last_error()
        torch.cuda.synchronize()
        assert int(status_a.item()) == 0 and int(status_b.item()) == 0
        Ea, Eb = energy_a.cpu().numpy()[0], energy_b.cpu().numpy()
        assert abs(Eb[0] - Ea[0]) <= E_REL * abs(Ea[0])
        assert np.abs(Eb - Ea).max() <= E_REL * abs(Ea[0])
        assert np.abs(force_b.cpu().numpy() - force_a.cpu().numpy()).max() <= F_ABS
        assert np.abs(pos_b.cpu().numpy() - pos_a.cpu().numpy()).max() <= 1e-12
        b.close()


def test_noalloc_refuses_oversized_system(gpu, potdir):
    import torch
    s = cf.fcc_vacancy_system(4, 3.615, 1, 0.02, 13)
    f = Field().readPotential(str(potdir / "eam.pot"))
    f.setup(s.lat, None, 10)
    lib = f._lib
    n = 4097                                   # one above AKMC_NOALLOC_MAX_ATOMS
    buf = torch.zeros((n, 3), dtype=torch.float64, device=gpu)
    lab = torch.zeros((n,), dtype=torch.int32, device=gpu)
    e = torch.zeros((5,), dtype=torch.float64, device=gpu)
    st_dev = torch.zeros((1,), dtype=torch.int32, device=gpu)
    box = (C.c_double * 3)(60.0, 60.0, 60.0)
    st = lib.akmc_eam_forces_noalloc(f._h, n, box, _ptr(buf), _ptr(lab), _ptr(buf), _ptr(e),
                                     _ptr(st_dev), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == STATUS["ERR_CAPACITY"]
    assert b"4096" in lib.akmc_last_error()


def test_noalloc_reports_out_of_range_label(gpu, potdir):
    """The labels of this call are read on the device only: one label outside the field's
    species sets AKMC_ERR_ARG in the status word instead of indexing the tables with it."""
    import torch
    s = cf.fcc_vacancy_system(4, 3.615, 1, 0.02, 14)
    f = Field().readPotential(str(potdir / "eam.pot"))
    f.setup(s.lat, None, 10)
    lib = f._lib
    stream = torch.cuda.current_stream().cuda_stream
    box = (C.c_double * 3)(*[float(x) for x in s.box])
    for bad in (1, -1):                        # the field has one species
        labels = s.labels.astype(np.int32).copy()
        labels[17] = bad
        pos = torch.tensor(s.pos, device=gpu)
        lab = torch.tensor(labels, device=gpu)
        force = torch.zeros((s.n, 3), dtype=torch.float64, device=gpu)
        energy = torch.zeros((5,), dtype=torch.float64, device=gpu)
        status = torch.zeros((1,), dtype=torch.int32, device=gpu)
        st = lib.akmc_eam_forces_noalloc(f._h, s.n, box, _ptr(pos), _ptr(lab), _ptr(force),
                                         _ptr(energy), _ptr(status), C.c_void_p(stream))
        assert st == 0, lib.akmc_last_error()
        torch.cuda.synchronize()
        assert int(status.item()) == STATUS["ERR_ARG"]
    # a clean call afterwards runs with a clean status
    pos = torch.tensor(s.pos, device=gpu)
    lab = torch.tensor(s.labels.astype(np.int32), device=gpu)
    st = lib.akmc_eam_forces_noalloc(f._h, s.n, box, _ptr(pos), _ptr(lab), _ptr(force),
                                     _ptr(energy), _ptr(status), C.c_void_p(stream))
    assert st == 0
    torch.cuda.synchronize()
    assert int(status.item()) == 0
