"""Host-side mirror of the reference's force-field interface over the C ABI.

The reference's optimisers see one object, ``Field`` (potentials/metal/Field.h:126-219,
potentials/pair/Field.h:658-748), created from a ``potentials`` file, set up for a cell
and called once per step through ``calculateForces``.  :class:`Field` keeps those
method names and argument meanings; :class:`Batch` is the device-resident path for
many independent systems (torch CUDA tensors as the memory, the kernels from
``libakmc_b200.so``).

Error behaviour: the reference exits the process on bad input; here every failure is
an :class:`AkmcError` carrying the C-ABI status code.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import AkmcError, Energy, check

PREC_MIXED = 0
PREC_FP64 = 1
FAMILY_EAM = 1
FAMILY_IONIC = 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


@dataclass
class Element:
    """Common/Element.h:5-32 (name, mass, charge)."""
    name: str
    mass: float
    charge: float


class Species:
    """potentials/Species.h:15-72: the element table the potentials file declares."""

    def __init__(self, elements=None):
        self.eleData = list(elements or [])

    def getNumSpecies(self):
        return len(self.eleData)

    def getSpecies(self, i):
        return self.eleData[i]

    def getMaxNumInteractions(self):
        return len(self.eleData) ** 2

    def getMass(self, i):
        return self.eleData[i].mass

    def index(self, name):
        return [e.name for e in self.eleData].index(name)


class Field:
    """Force field behind the reference's ``Field`` API, evaluated on the GPU."""

    def __init__(self):
        self._lib = _lib.load()
        self._h = C.c_void_p()
        self.species = Species()
        self._lat = None

    # --- reference-shaped lifecycle ----------------------------------------------------
    def readPotential(self, path, spec: Species | None = None):
        """Field::readPotential: parse the potentials file; fills ``spec`` like the
        reference's Species::loadSpecies."""
        check(self._lib.akmc_field_create(str(path).encode(), C.byref(self._h)), "readPotential")
        n = self._lib.akmc_field_num_species(self._h)
        els = []
        for i in range(n):
            name = C.create_string_buffer(16)
            m, q = C.c_double(), C.c_double()
            check(self._lib.akmc_field_species(self._h, i, name, C.byref(m), C.byref(q)), "species")
            els.append(Element(name.value.decode(), m.value, q.value))
        self.species = Species(els)
        if spec is not None:
            spec.eleData = list(els)
        return self

    def setup(self, latVector, rcpVector=None, maxAtoms=1):
        """Field::setup: cutoff check, Ewald k-set, device tables."""
        lat = np.ascontiguousarray(latVector, dtype=np.float64).reshape(9)
        rcp = None if rcpVector is None else np.ascontiguousarray(rcpVector, np.float64).reshape(9)
        check(self._lib.akmc_field_setup(self._h, _d(lat), None if rcp is None else _d(rcp),
                                         int(maxAtoms)), "setup")
        self._lat = lat
        return self

    def setPrecision(self, mode):
        check(self._lib.akmc_field_set_precision(self._h, int(mode)), "setPrecision")

    def calculateForces(self, posX, posY, posZ, forceX, forceY, forceZ, stress, latVector,
                        rcpVector, charge, atmLabel, frozen, numAtoms, eng: Energy | None = None):
        """Field::calculateForces (metal/Field.h:192-193) on host arrays.  As in the
        reference, forces and stress are overwritten and the positions are wrapped into
        the minimum-image cell in place.  ``frozen`` is ignored (callers zero frozen
        forces, Basis::freezeForces).  Returns the Energy record."""
        if self._lat is not None and not np.array_equal(np.asarray(latVector, np.float64).reshape(9),
                                                        self._lat):
            raise AkmcError(1, "calculateForces: lattice differs from the setup lattice")
        arrs = [posX, posY, posZ, forceX, forceY, forceZ]
        for a in arrs:
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
                raise TypeError("positions and forces must be contiguous float64 arrays")
        lab = np.ascontiguousarray(atmLabel, dtype=np.int32)
        q = None if charge is None else np.ascontiguousarray(charge, dtype=np.float64)
        st = stress if stress is not None else np.zeros(6)
        e = eng if eng is not None else Energy()
        check(self._lib.akmc_forces(self._h, int(numAtoms), _d(posX), _d(posY), _d(posZ), _i(lab),
                                    None if q is None else _d(q), _d(forceX), _d(forceY),
                                    _d(forceZ), _d(st), C.byref(e)), "calculateForces")
        return e

    # --- conveniences ------------------------------------------------------------------
    def forces(self, pos, labels, charge=None):
        """(N,3) positions -> (Energy dict, (N,3) forces, (N,3) wrapped positions)."""
        pos = np.asarray(pos, dtype=np.float64)
        n = len(pos)
        x, y, z = (np.ascontiguousarray(pos[:, k]).copy() for k in range(3))
        fx, fy, fz = (np.zeros(n) for _ in range(3))
        e = self.calculateForces(x, y, z, fx, fy, fz, np.zeros(6), self._lat, None, charge, labels,
                                 None, n)
        return e.as_dict(), np.stack([fx, fy, fz], 1), np.stack([x, y, z], 1)

    @property
    def family(self):
        return self._lib.akmc_field_family(self._h)

    @property
    def cutoff(self):
        return self._lib.akmc_field_cutoff(self._h)

    def ewald(self):
        eta, nk = C.c_double(), C.c_int()
        g = (C.c_int * 3)()
        check(self._lib.akmc_field_ewald(self._h, C.byref(eta), C.byref(nk), g), "ewald")
        return dict(eta=eta.value, nk=nk.value, gcell=list(g))

    def set_list_density(self, rho):
        """akmc_field_set_list_density: floor of the number density (atoms / A^3) that sizes
        the EAM neighbour lists of batches created afterwards (clustered atoms)."""
        check(self._lib.akmc_field_set_list_density(self._h, float(rho)), "set_list_density")
        return self

    def batch(self, natoms, boxes, labels, charges=None, skin=0.0):
        return Batch(self, natoms, boxes, labels, charges, skin)

    def close(self):
        if self._h:
            self._lib.akmc_field_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """akmc_batch: many independent systems, device-resident (torch CUDA tensors).

    Atoms of system s occupy rows ``offsets[s]:offsets[s+1]`` of the (n_total, 3) float64
    position and force tensors; energies are (nsys, 5): total, rcp, real, vdw, many."""

    def __init__(self, field: Field, natoms, boxes, labels, charges=None, skin=0.0):
        self.field = field
        self._lib = field._lib
        self.natoms = np.ascontiguousarray(natoms, dtype=np.int32)
        self.boxes = np.ascontiguousarray(boxes, dtype=np.float64).reshape(-1, 3)
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        q = None if charges is None else np.ascontiguousarray(charges, dtype=np.float64)
        self.nsys = len(self.natoms)
        self.n_total = int(self.natoms.sum())
        self.offsets = np.concatenate([[0], np.cumsum(self.natoms)]).astype(np.int64)
        self._h = C.c_void_p()
        self.skin = float(skin)
        check(self._lib.akmc_batch_create_skin(field._h, self.nsys, _i(self.natoms), _d(self.boxes),
                                               _i(lab), None if q is None else _d(q), self.skin,
                                               C.byref(self._h)), "batch_create")

    @property
    def launches(self):
        return self._lib.akmc_batch_launches(self._h)

    def forces_(self, pos, force, energy, status, stream=None):
        """Asynchronous device call on raw device pointers / torch tensors."""
        import torch
        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        ptr = lambda t: t.data_ptr() if hasattr(t, "data_ptr") else int(t)
        check(self._lib.akmc_batch_forces(self._h, C.c_void_p(ptr(pos)), C.c_void_p(ptr(force)),
                                          C.c_void_p(ptr(energy)), C.c_void_p(ptr(status)),
                                          C.c_void_p(int(stream))), "batch_forces")

    def forces_host(self, pos, force, energy, status, stream=None):
        """akmc_batch_forces_host on host numpy arrays or (pinned) CPU torch tensors:
        copies in, computes, copies wrapped positions, forces, energies, statuses back."""
        ptr = lambda a: a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data
        if stream is None:
            import torch
            stream = torch.cuda.current_stream().cuda_stream
        check(self._lib.akmc_batch_forces_host(self._h, C.c_void_p(ptr(pos)), C.c_void_p(ptr(force)),
                                               C.c_void_p(ptr(energy)), C.c_void_p(ptr(status)),
                                               C.c_void_p(int(stream))), "batch_forces_host")

    def autotune(self, pos, force, energy, status, stream=None):
        """Time the work-item sizes on these buffers and keep the fastest; returns it."""
        import torch
        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        ptr = lambda t: t.data_ptr() if hasattr(t, "data_ptr") else int(t)
        chosen = C.c_int(0)
        check(self._lib.akmc_batch_autotune(self._h, C.c_void_p(ptr(pos)), C.c_void_p(ptr(force)),
                                            C.c_void_p(ptr(energy)), C.c_void_p(ptr(status)),
                                            C.c_void_p(int(stream)), C.byref(chosen)), "autotune")
        return chosen.value

    def set_home_chunk(self, hc):
        check(self._lib.akmc_batch_set_home_chunk(self._h, int(hc)), "set_home_chunk")

    @property
    def home_chunk(self):
        return self._lib.akmc_batch_home_chunk(self._h)

    def neighbours(self, max_per_atom=256):
        """Neighbour sets of the last EAM force call: (counts (n,), rows (n, max) padded -1)."""
        counts = np.zeros(self.n_total, dtype=np.int32)
        rows = np.zeros((self.n_total, max_per_atom), dtype=np.int32)
        check(self._lib.akmc_batch_neighbours(self._h, _i(counts), _i(rows), int(max_per_atom)),
              "batch_neighbours")
        return counts, rows

    def list_modes(self):
        """Per system, what the last call did with its neighbour list: 0 no skin, 1 rebuilt,
        2 reused."""
        m = np.zeros(self.nsys, dtype=np.int32)
        check(self._lib.akmc_batch_list_modes(self._h, _i(m)), "batch_list_modes")
        return m

    def profile(self, enable=True):
        check(self._lib.akmc_batch_profile(self._h, int(bool(enable))), "batch_profile")

    def kernel_times(self):
        """{kernel name: (total ms, launches)} since the previous call."""
        ms = (C.c_double * 8)()
        cnt = (C.c_int * 8)()
        names = (C.c_char_p * 8)()
        n = self._lib.akmc_batch_kernel_times(self._h, ms, cnt, names, 8)
        return {names[k].decode(): (ms[k], cnt[k]) for k in range(n) if cnt[k] > 0}

    def alloc(self, device="cuda"):
        import torch
        return (torch.zeros((self.n_total, 3), dtype=torch.float64, device=device),
                torch.zeros((self.nsys, 5), dtype=torch.float64, device=device),
                torch.zeros((self.nsys,), dtype=torch.int32, device=device))

    def close(self):
        if self._h:
            self._lib.akmc_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
